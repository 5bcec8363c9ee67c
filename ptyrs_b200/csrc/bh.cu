// pty-chi BH on the GPU (reference engine/gpu/bh.rs:29-72; CPU twin `Bh::epoch`,
// engine/bh.rs:580-760): per batch the amplitude cost's gradient pass (the frame kernel's
// gradient mode on BH's residual, keeping each frame's detector field and exit-plane field),
// the gathers of 2·∂F/∂x*, the conjugate or steepest direction, ⟨g, D⟩ and the bilinear
// Hessian's H(·,·) per frame (bh.cuh), and the step α·D on object and probe.
#include "engine.cuh"

using namespace ptyb;

namespace ptyb::eng {
namespace {

// The batch's gradient pass, stack by stack in batch order: every frame's kept detector field
// U psi and exit-plane field Uᴴ(2·td) into psi_all / g_all at its batch slot, and
// 2·∂F/∂x* (engine/bh.rs:320-380) gathered into g_obj and g_probe with compensation.
void bh_grads(ptyb_handle* h, const int* frames, int n) {
  const size_t no = (size_t)h->nobj * h->nyo * h->nxo, np = (size_t)h->K * h->N * h->N;
  check(h, cudaMemsetAsync(h->g_obj, 0, no * sizeof(float2), h->stream), "memset");
  check(h, cudaMemsetAsync(h->g_obj_c, 0, no * sizeof(float2), h->stream), "memset");
  check(h, cudaMemsetAsync(h->g_probe, 0, np * sizeof(float2), h->stream), "memset");
  check(h, cudaMemsetAsync(h->g_probe_c, 0, np * sizeof(float2), h->stream), "memset");
  const int stack = std::min(n, h->slots);
  for (int s0 = 0; s0 < n; s0 += stack) {
    const int m = std::min(stack, n - s0);
    const int* fr = frames + s0;
    float2* gfield = h->g_all + (size_t)s0 * np;
    FrameArgs a = frame_args(h, fr);
    a.out = gfield;
    a.psi_out = h->psi_all + (size_t)s0 * np;
    check(h, launch_frame<kBhGrad>(h, a, m), "bh gradient pass");
    ++h->launches;
    GatherArgs g = gather_args(h, fr, m);
    g.upd = gfield;
    g.out = h->g_obj;
    g.comp = h->g_obj_c;
    timed(h, kKObjMl, [&] { object_tile_kernel<kGatherMl><<<ntiles(h), 1024, 0, h->stream>>>(g); }, m);
    launched(h, "bh object gradient");
    int nchunk = 0;
    const int chunk = probe_chunk(h, m, &nchunk);
    ProbeArgs pa = {};
    pa.object = h->object;
    pa.quad = h->quad;
    pa.upd = gfield;
    pa.frames = fr;
    pa.corners = h->corners;
    pa.omax = h->omax;
    pa.partial = h->partial;
    pa.nslot = m;
    pa.chunk = chunk;
    pa.nxo = h->nxo;
    pa.K = h->K;
    pa.N = h->N;
    pa.mode = 1;
    dim3 grid((h->N * h->N + 255) / 256, nchunk);
    timed(h, kKProbePartial, [&] { probe_partial_kernel<<<grid, 256, 0, h->stream>>>(pa); }, m);
    launched(h, "bh probe gradient");
    timed(h, kKProbeFinal, [&] {
      probe_finalize_kernel<<<(unsigned)((np + 255) / 256), 256, 0, h->stream>>>(
          h->partial, nchunk, (int)np, nullptr, h->g_probe, h->g_probe_c, 1.f, 2);
    });
    launched(h, "bh probe gradient sum");
  }
}

// H(u, v) over the batch (engine/bh.rs:500-575): every frame's share on the device, added in
// batch order on the host. Needs the batch's gradient pass (bh_grads) at the same state.
double bh_hessian(ptyb_handle* h, const int* frames, int n, const float2* uo, const float2* up,
                  const float2* vo, const float2* vp) {
  const size_t np = (size_t)h->K * h->N * h->N;
  BhArgs a = {};
  a.object = h->object;
  a.probe = h->probe;
  a.u_obj = uo;
  a.u_probe = up;
  a.v_obj = vo;
  a.v_probe = vp;
  a.same = uo == vo && up == vp;
  a.quad = h->quad;
  a.tw = h->tw;
  a.iobs = h->iobs;
  a.corners = h->corners;
  a.nyo = h->nyo;
  a.nxo = h->nxo;
  a.nprobe = h->nprobe;
  a.nobj = h->nobj;
  const int stack = std::min(n, h->slots);
  for (int s0 = 0; s0 < n; s0 += stack) {
    const int m = std::min(stack, n - s0);
    a.frames = frames + s0;
    a.psi = h->psi_all + (size_t)s0 * np;
    a.g = h->g_all + (size_t)s0 * np;
    a.out = h->gamma_sums + s0;
    cudaError_t e = cudaSuccess;
    timed(h, kKBhHessian, [&] { e = launch_bh_side(h->N, a, m, h->stream); }, m);
    check(h, e, "bh hessian");
    ++h->launches;
  }
  std::vector<double> v(n);
  check(h, copy_sync(h, v.data(), h->gamma_sums, n * sizeof(double), cudaMemcpyDeviceToHost),
        "bh hessian");
  double s = 0.0;
  for (double x : v) s += x;
  return s;
}

// ⟨a, b⟩ = Σ Re(conj(a)·b) over n elements, block partials added in order.
double dot_of(ptyb_handle* h, const float2* x, const float2* y, size_t n) {
  double out[2];
  array_sums(h, x, y, n, 2, out);
  return out[0];
}

// One BH epoch over the batches of `order` (device frames, lengths `sizes`): conjugate
// directions when `cg` (one batch of every frame after the first epoch), the steps into
// h->bh_steps.
void bh_epoch(ptyb_handle* h, const ptyb_bh_params& p, const int* order,
              const std::vector<int32_t>& sizes, bool cg) {
  const size_t no = (size_t)h->nobj * h->nyo * h->nxo, np = (size_t)h->K * h->N * h->N;
  const int size = std::min(p.batch_size, h->P);
  const double rho2 = p.probe_rho * p.probe_rho * ((double)h->N * h->N);
  h->bh_steps.clear();
  int off = 0;
  for (size_t b = 0; b < sizes.size(); ++b) {
    const int n = sizes[b];
    const int* frames = order + off;
    bh_grads(h, frames, n);
    // Pg: the probe part times ρ² (the object part is g itself)
    check(h, cudaMemcpyAsync(h->last_probe, h->g_probe, np * sizeof(float2),
                             cudaMemcpyDeviceToDevice, h->stream),
          "preconditioned gradient");
    timed(h, kKAxpy, [&] {
      scale_kernel<<<blocks_for(np), 256, 0, h->stream>>>(h->last_probe, (float)rho2, np);
    });
    launched(h, "preconditioned gradient");
    double beta = 0.0;
    if (cg) {
      const double hn =
          bh_hessian(h, frames, n, h->g_obj, h->last_probe, h->dir_obj, h->dir_probe);
      const double hd =
          bh_hessian(h, frames, n, h->dir_obj, h->dir_probe, h->dir_obj, h->dir_probe);
      beta = hn / hd;
    }
    // D = β·D′ − Pg (D = −Pg when β = 0)
    timed(h, kKAxpy, [&] {
      cg_direction_kernel<<<blocks_for(no), 256, 0, h->stream>>>(h->dir_obj, h->g_obj,
                                                                 (float)beta, no);
    });
    launched(h, "direction");
    timed(h, kKAxpy, [&] {
      cg_direction_kernel<<<blocks_for(np), 256, 0, h->stream>>>(h->dir_probe, h->last_probe,
                                                                 (float)beta, np);
    });
    launched(h, "direction");
    const double top =
        -(dot_of(h, h->g_obj, h->dir_obj, no) + dot_of(h, h->g_probe, h->dir_probe, np));
    const double bottom =
        bh_hessian(h, frames, n, h->dir_obj, h->dir_probe, h->dir_obj, h->dir_probe);
    const double alpha = top / bottom * n / size;
    timed(h, kKAxpy, [&] {
      axpy_kernel<<<blocks_for(no), 256, 0, h->stream>>>(h->object, h->dir_obj, (float)alpha, no);
    });
    launched(h, "step");
    timed(h, kKAxpy, [&] {
      axpy_kernel<<<blocks_for(np), 256, 0, h->stream>>>(h->probe, h->dir_probe, (float)alpha,
                                                         np);
    });
    launched(h, "step");
    ptyb_bh_step st;
    st.batch = (int32_t)b;
    st.count = n;
    st.beta = beta;
    st.alpha = alpha;
    st.top = top;
    st.bottom = bottom;
    h->bh_steps.push_back(st);
    off += n;
  }
}

}  // namespace
}  // namespace ptyb::eng

using namespace ptyb::eng;

extern "C" {

int ptyb_bh(ptyb_handle* h, const ptyb_bh_params* p, int32_t nepoch, int32_t calc_llk) {
  if (!h || !p) return PTYB_INVALID;
  if (p->batch_size <= 0 || nepoch < 0) {
    h->err = "BH batch_size must be >= 1";
    return PTYB_INVALID;
  }
  if (h->nslice > 1 || h->have_offsets) {
    h->err = "BH runs on a single-slice object without the position model";
    return PTYB_INVALID;
  }
  return guarded(h, true, [&]() -> int {
    const int size = std::min(p->batch_size, h->P);
    ensure_slots(h, std::min(h->P, h->stack));
    ensure_ml(h);
    std::vector<std::vector<int32_t>> sizes;
    // a fresh run: epoch e's batches from random_batches(nframe, size, seed, e)
    upload_orders(h, nepoch, size, p->seed, 0, &sizes, nullptr);
    begin_call(h);
    for (int ic = 0; ic < nepoch; ++ic) {
      bh_epoch(h, *p, h->order_all + (size_t)ic * h->P, sizes[ic], size == h->P && ic > 0);
      if (llk_due(calc_llk, ic, nepoch)) record(h, kAlgBh, llk_pass(h));
      ++h->cycle;
    }
    end_call(h, "bh");
    return PTYB_OK;
  });
}

int ptyb_bh_steps_len(ptyb_handle* h) { return h ? (int)h->bh_steps.size() : 0; }

int ptyb_bh_steps(ptyb_handle* h, ptyb_bh_step* dst, int32_t cap) {
  if (!h || (!dst && cap > 0)) return PTYB_INVALID;
  const int n = std::min<int>(cap, (int)h->bh_steps.size());
  std::copy(h->bh_steps.begin(), h->bh_steps.begin() + n, dst);
  return PTYB_OK;
}

}  // extern "C"
