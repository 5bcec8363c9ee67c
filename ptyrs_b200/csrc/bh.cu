// pty-chi BH on the GPU (reference engine/gpu/bh.rs:29-72; CPU twin `Bh::epoch`,
// engine/bh.rs:580-760): per batch the amplitude cost's gradient pass (the frame kernel's
// gradient mode on BH's residual, keeping each frame's detector field and exit-plane field),
// the gathers of 2·∂F/∂x*, the conjugate or steepest direction, ⟨g, D⟩ and the bilinear
// Hessian's H(·,·) per frame (bh.cuh), and the step α·D on object and probe. Under the position
// model (Patch sampling, engine/bh.rs:92-275) every frame reads its probe moved by its offset:
// the gradient pass and the object gather take the moved probes, the probe gradient goes back
// through each frame's move, and with refined offsets the offsets are variables (their
// gradient from the position sums of the gradient field, their parts of the directions and
// steps kept on the host, 0.3·α·D_d added to them).
#include "engine.cuh"

using namespace ptyb;

namespace ptyb::eng {
namespace {

constexpr double kPositionStep = 0.3;  // engine/bh.rs POSITION_STEP

// A displacement of the batch: object and probe on the device, the offsets' part [n][2] of
// the batch frames on the host (null without refined offsets).
struct BhVec {
  const float2* obj;
  const float2* probe;
  const double* d;
};

// The batch's gradient pass, stack by stack in batch order: every frame's kept detector field
// U psi and exit-plane field Uᴴ(2·td) into psi_all / g_all at its batch slot, and
// 2·∂F/∂x* (engine/bh.rs:320-380) gathered into g_obj and g_probe with compensation; with
// refined offsets ∂F/∂d per frame into ml_pos_sums ([frame][4], num_y and num_x).
void bh_grads(ptyb_handle* h, const int* frames, int n) {
  const size_t no = (size_t)h->nobj * h->nyo * h->nxo, np = (size_t)h->K * h->N * h->N;
  const bool pos = h->have_offsets, refine = pos && h->refine_offsets;
  check(h, cudaMemsetAsync(h->g_obj, 0, no * sizeof(float2), h->stream), "memset");
  check(h, cudaMemsetAsync(h->g_obj_c, 0, no * sizeof(float2), h->stream), "memset");
  check(h, cudaMemsetAsync(h->g_probe, 0, np * sizeof(float2), h->stream), "memset");
  check(h, cudaMemsetAsync(h->g_probe_c, 0, np * sizeof(float2), h->stream), "memset");
  if (pos) check(h, cudaMemsetAsync(h->g_probe_spec, 0, np * sizeof(float2), h->stream), "memset");
  const int stack = std::min(n, h->slots);
  for (int s0 = 0; s0 < n; s0 += stack) {
    const int m = std::min(stack, n - s0);
    const int* fr = frames + s0;
    float2* gfield = h->g_all + (size_t)s0 * np;
    FrameArgs a = frame_args(h, fr);
    if (pos) {
      // each frame's moved probe conj(q)·T_d(q·P) from the probe's spectra
      move_frames(h, fr, m, h->spec, h->wave);
      a.probe = h->wave;
      a.probe_stride = (int)np;
    }
    a.out = gfield;
    a.psi_out = h->psi_all + (size_t)s0 * np;
    check(h, launch_frame<kBhGrad>(h, a, m), "bh gradient pass");
    ++h->launches;
    GatherArgs g = gather_args(h, fr, m);
    g.upd = gfield;
    g.out = h->g_obj;
    g.comp = h->g_obj_c;
    if (pos) {
      g.probe = h->wave;
      g.probe_stride = (int)np;
    }
    timed(h, kKObjMl, [&] { object_tile_kernel<kGatherMl><<<ntiles(h), 1024, 0, h->stream>>>(g); }, m);
    launched(h, "bh object gradient");
    if (pos) {
      // DFT(conj(O_win)·g)·exp(+2πi f·d) per frame, summed in frame order (the moves' adjoint)
      MoveArgs mb = move_args(h, fr, h->wave2);
      mb.c = gfield;
      check(h, launch_move<kBackSpectrum>(h, mb, m), "bh probe gradient spectra");
      ++h->launches;
      timed(h, kKProbeFinal, [&] {
        probe_finalize_kernel<<<(unsigned)((np + 255) / 256), 256, 0, h->stream>>>(
            h->wave2, m, (int)np, nullptr, h->g_probe_spec, h->g_probe_c, 1.f, 2);
      }, m);
      launched(h, "bh probe gradient sum");
      if (refine) {
        // Σ_m Re⟨g, ∂_a M(P)·O·q⟩ per frame and axis: ∂F/∂d (engine/bh.rs:380-420)
        MoveArgs md = move_args(h, fr, nullptr);
        md.spec = h->spec;
        md.c = gfield;
        md.sums = h->ml_pos_sums;
        check(h, launch_move<kDerivSums>(h, md, m), "bh offsets gradient");
        ++h->launches;
      }
      continue;
    }
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
  if (pos) {
    // g_P = conj(q)·IDFT(Σ_frames spectra)
    MoveArgs mi = move_args(h, h->iota, h->g_probe);
    mi.spec = h->g_probe_spec;
    check(h, launch_move<kPlainInverse>(h, mi, 1), "bh probe gradient");
    ++h->launches;
  }
}

// The per-slot planes of the position model's Hessian for the stack `fr` of m frames:
// M(P), M(u_P) (and M(v_P) unless `same`), with refined offsets their derivatives.
void bh_planes(ptyb_handle* h, const int* fr, int m, bool same, bool refine) {
  auto mv = [&](const float2* spec, float2* out, int deriv) {
    MoveArgs a = move_args(h, fr, out);
    a.spec = spec;
    a.deriv = deriv;
    if (deriv == 0)
      check(h, launch_move<kFromSpectrum>(h, a, m), "bh moved planes");
    else
      check(h, launch_move<kDerivMove>(h, a, m), "bh moved plane derivatives");
    ++h->launches;
  };
  float2** p = h->bh_planes;
  mv(h->spec, p[0], 0);
  mv(h->bh_spec_u, p[1], 0);
  if (!same) mv(h->bh_spec_v, p[2], 0);
  if (!refine) return;
  mv(h->spec, p[3], 1);
  mv(h->spec, p[4], 2);
  mv(h->bh_spec_u, p[5], 1);
  mv(h->bh_spec_u, p[6], 2);
  if (!same) {
    mv(h->bh_spec_v, p[7], 1);
    mv(h->bh_spec_v, p[8], 2);
  }
  mv(h->spec, p[9], 3);
  mv(h->spec, p[10], 4);
  mv(h->spec, p[11], 5);
}

void ensure_bh_planes(ptyb_handle* h) {
  if (h->bh_slots >= h->slots) return;
  const size_t np = (size_t)h->K * h->N * h->N;
  for (auto& p : h->bh_planes) p = alloc<float2>(h, (size_t)h->slots * np);
  h->bh_ud = alloc<double>(h, (size_t)h->slots * 2);
  h->bh_vd = alloc<double>(h, (size_t)h->slots * 2);
  if (!h->bh_spec_u) {
    h->bh_spec_u = alloc<float2>(h, np);
    h->bh_spec_v = alloc<float2>(h, np);
  }
  h->bh_slots = h->slots;
}

// H(u, v) over the batch (engine/bh.rs:500-575): every frame's share on the device, added in
// batch order on the host. Needs the batch's gradient pass (bh_grads) at the same state, and
// under the position model the probe's spectra in h->spec.
double bh_hessian(ptyb_handle* h, const int* frames, int n, const BhVec& u, const BhVec& v) {
  const size_t np = (size_t)h->K * h->N * h->N;
  const bool pos = h->have_offsets, refine = pos && h->refine_offsets;
  const bool same = u.obj == v.obj && u.probe == v.probe && u.d == v.d;
  BhArgs a = {};
  a.object = h->object;
  a.probe = h->probe;
  a.u_obj = u.obj;
  a.u_probe = u.probe;
  a.v_obj = v.obj;
  a.v_probe = v.probe;
  a.same = same;
  a.quad = h->quad;
  a.tw = h->tw;
  a.iobs = h->iobs;
  a.corners = h->corners;
  a.nyo = h->nyo;
  a.nxo = h->nxo;
  a.nprobe = h->nprobe;
  a.nobj = h->nobj;
  if (pos) {
    ensure_bh_planes(h);
    spectrum_of(h, u.probe, h->bh_spec_u);
    if (!same) spectrum_of(h, v.probe, h->bh_spec_v);
    float2** p = h->bh_planes;
    a.w = p[0];
    a.tu = p[1];
    a.tv = same ? p[1] : p[2];
    if (refine) {
      a.dwy = p[3];
      a.dwx = p[4];
      a.dtuy = p[5];
      a.dtux = p[6];
      a.dtvy = same ? p[5] : p[7];
      a.dtvx = same ? p[6] : p[8];
      a.dwyy = p[9];
      a.dwyx = p[10];
      a.dwxx = p[11];
      a.ud = h->bh_ud;
      a.vd = same ? h->bh_ud : h->bh_vd;
    }
  }
  const int stack = std::min(n, h->slots);
  for (int s0 = 0; s0 < n; s0 += stack) {
    const int m = std::min(stack, n - s0);
    a.frames = frames + s0;
    a.psi = h->psi_all + (size_t)s0 * np;
    a.g = h->g_all + (size_t)s0 * np;
    a.out = h->gamma_sums + s0;
    if (pos) {
      bh_planes(h, a.frames, m, same, refine);
      if (refine) {
        check(h, copy_sync(h, h->bh_ud, u.d + 2 * s0, 2 * m * sizeof(double),
                           cudaMemcpyHostToDevice),
              "bh offsets parts");
        if (!same)
          check(h, copy_sync(h, h->bh_vd, v.d + 2 * s0, 2 * m * sizeof(double),
                             cudaMemcpyHostToDevice),
                "bh offsets parts");
      }
    }
    cudaError_t e = cudaSuccess;
    timed(h, kKBhHessian, [&] { e = launch_bh_side(h->N, a, m, h->stream); }, m);
    check(h, e, "bh hessian");
    ++h->launches;
  }
  std::vector<double> out(n);
  check(h, copy_sync(h, out.data(), h->gamma_sums, n * sizeof(double), cudaMemcpyDeviceToHost),
        "bh hessian");
  double s = 0.0;
  for (double x : out) s += x;
  return s;
}

// ⟨a, b⟩ = Σ Re(conj(a)·b) over n elements, block partials added in order.
double dot_of(ptyb_handle* h, const float2* x, const float2* y, size_t n) {
  double out[2];
  array_sums(h, x, y, n, 2, out);
  return out[0];
}

// BH through a multislice object (no position model): Q(w) = H(w, w) over the batch from the
// second-order expansion of the exit waves along w through the slices (multislice.cuh
// `slice_gamma_kernel` in its BH mode), per frame on the device, added in batch order.
double bh_slice_quad(ptyb_handle* h, const int* frames, int n, const float2* w_obj,
                     const float2* w_probe) {
  SliceGammaArgs g = {};
  g.d_obj = w_obj;
  g.d_probe = w_probe;
  g.bh = 1;
  const int stack = std::min(n, h->slots);
  for (int s0 = 0; s0 < n; s0 += stack) {
    const int m = std::min(stack, n - s0);
    g.sa.f = frame_args(h, frames + s0);
    g.sa.f.nslot = m;
    g.sa.tf = h->tf;
    g.sa.nslice = h->nslice;
    g.sa.obj_plane = (size_t)h->nyo * h->nxo;
    g.out = h->gamma_sums + (size_t)s0 * 2;
    cudaError_t e = cudaSuccess;
    timed(h, kKBhHessian, [&] { e = launch_slice_gamma_side(h->N, g, m, h->K, h->stream); }, m);
    check(h, e, "bh quadratic form through slices");
    ++h->launches;
  }
  std::vector<double> out((size_t)n * 2);
  check(h, copy_sync(h, out.data(), h->gamma_sums, out.size() * sizeof(double),
                     cudaMemcpyDeviceToHost),
        "bh quadratic form");
  double s = 0.0;
  for (int k = 0; k < n; ++k) s += out[2 * (size_t)k];
  return s;
}

// H(u, v) through the slices by polarization, (Q(u + v) − Q(u − v))/4, exact for the
// symmetric bilinear H; Q(u) when v is u.
double bh_slice_hessian(ptyb_handle* h, const int* frames, int n, const BhVec& u,
                        const BhVec& v) {
  if (u.obj == v.obj && u.probe == v.probe) return bh_slice_quad(h, frames, n, u.obj, u.probe);
  const size_t no = (size_t)h->nslice * h->nyo * h->nxo, np = (size_t)h->K * h->N * h->N;
  float2 *to = h->bh_tmp, *tp = h->bh_tmp + no;
  double q[2];
  for (int k = 0; k < 2; ++k) {
    const float sgn = k == 0 ? 1.f : -1.f;
    check(h, cudaMemcpyAsync(to, u.obj, no * sizeof(float2), cudaMemcpyDeviceToDevice,
                             h->stream),
          "bh polarization");
    check(h, cudaMemcpyAsync(tp, u.probe, np * sizeof(float2), cudaMemcpyDeviceToDevice,
                             h->stream),
          "bh polarization");
    timed(h, kKAxpy, [&] {
      axpy_kernel<<<blocks_for(no), 256, 0, h->stream>>>(to, v.obj, sgn, no);
    });
    launched(h, "bh polarization");
    timed(h, kKAxpy, [&] {
      axpy_kernel<<<blocks_for(np), 256, 0, h->stream>>>(tp, v.probe, sgn, np);
    });
    launched(h, "bh polarization");
    q[k] = bh_slice_quad(h, frames, n, to, tp);
  }
  return (q[0] - q[1]) / 4.0;
}

// One BH epoch through the slices (the multislice counterpart of bh_epoch): the gradients
// through the slices on BH's amplitude cost, the probe part preconditioned by ρ², β from the
// polarized Hessian, α·D on every slice and the probe.
void bh_epoch_slices(ptyb_handle* h, const ptyb_bh_params& p, const int* order,
                     const std::vector<int32_t>& sizes, bool cg) {
  const size_t no = (size_t)h->nslice * h->nyo * h->nxo, np = (size_t)h->K * h->N * h->N;
  const int size = std::min(p.batch_size, h->P);
  const double rho2 = p.probe_rho * p.probe_rho * ((double)h->N * h->N);
  h->bh_steps.clear();
  int off = 0;
  for (size_t b = 0; b < sizes.size(); ++b) {
    const int n = sizes[b];
    const int* frames = order + off;
    slice_gradients(h, true, true, frames, n, kCostBh);
    check(h, cudaMemcpyAsync(h->last_probe, h->g_probe, np * sizeof(float2),
                             cudaMemcpyDeviceToDevice, h->stream),
          "preconditioned gradient");
    timed(h, kKAxpy, [&] {
      scale_kernel<<<blocks_for(np), 256, 0, h->stream>>>(h->last_probe, (float)rho2, np);
    });
    launched(h, "preconditioned gradient");
    const BhVec pg = {h->g_slices, h->last_probe, nullptr};
    const BhVec dir = {h->dir_slices, h->dir_probe, nullptr};
    double beta = 0.0;
    if (cg) beta = bh_slice_hessian(h, frames, n, pg, dir) / bh_slice_hessian(h, frames, n, dir, dir);
    timed(h, kKAxpy, [&] {
      cg_direction_kernel<<<blocks_for(no), 256, 0, h->stream>>>(h->dir_slices, h->g_slices,
                                                                 (float)beta, no);
    });
    launched(h, "direction");
    timed(h, kKAxpy, [&] {
      cg_direction_kernel<<<blocks_for(np), 256, 0, h->stream>>>(h->dir_probe, h->last_probe,
                                                                 (float)beta, np);
    });
    launched(h, "direction");
    const double top =
        -(dot_of(h, h->g_slices, h->dir_slices, no) + dot_of(h, h->g_probe, h->dir_probe, np));
    const double bottom = bh_slice_hessian(h, frames, n, dir, dir);
    const double alpha = top / bottom * n / size;
    timed(h, kKAxpy, [&] {
      axpy_kernel<<<blocks_for(no), 256, 0, h->stream>>>(h->object, h->dir_slices, (float)alpha,
                                                         no);
    });
    launched(h, "step");
    timed(h, kKAxpy, [&] {
      axpy_kernel<<<blocks_for(np), 256, 0, h->stream>>>(h->probe, h->dir_probe, (float)alpha,
                                                         np);
    });
    launched(h, "step");
    ptyb_bh_step s;
    s.batch = (int32_t)b;
    s.count = n;
    s.beta = beta;
    s.alpha = alpha;
    s.top = top;
    s.bottom = bottom;
    h->bh_steps.push_back(s);
    off += n;
  }
}

// The run's state on the host: the offsets and, for CG, the direction's offsets part by frame.
struct BhHost {
  std::vector<double> offsets;  // [P][2]
  std::vector<double> dir_d;    // [P][2]
};

// One BH epoch over the batches of `order` (device frames, lengths `sizes`; `order_h` the same
// on the host): conjugate directions when `cg` (one batch of every frame after the first
// epoch), the steps into h->bh_steps.
void bh_epoch(ptyb_handle* h, const ptyb_bh_params& p, const int* order, const int* order_h,
              const std::vector<int32_t>& sizes, bool cg, BhHost& st) {
  const size_t no = (size_t)h->nobj * h->nyo * h->nxo, np = (size_t)h->K * h->N * h->N;
  const int size = std::min(p.batch_size, h->P);
  const double rho2 = p.probe_rho * p.probe_rho * ((double)h->N * h->N);
  const double pos_rho2 = p.position_rho * p.position_rho;
  const bool pos = h->have_offsets, refine = pos && h->refine_offsets;
  h->bh_steps.clear();
  int off = 0;
  for (size_t b = 0; b < sizes.size(); ++b) {
    const int n = sizes[b];
    const int* frames = order + off;
    const int* frames_h = order_h + off;
    if (pos) spectrum_of(h, h->probe, h->spec);
    bh_grads(h, frames, n);
    // the offsets' gradient of the batch frames, [n][2], and Pg's part of it
    std::vector<double> g_d, pg_d, prev_d, dir_d;
    if (refine) {
      std::vector<double> sums((size_t)h->P * 4);
      check(h, copy_sync(h, sums.data(), h->ml_pos_sums, sums.size() * sizeof(double),
                         cudaMemcpyDeviceToHost),
            "bh offsets gradient");
      g_d.resize(2 * n);
      pg_d.resize(2 * n);
      prev_d.resize(2 * n);
      dir_d.resize(2 * n);
      for (int k = 0; k < n; ++k)
        for (int ax = 0; ax < 2; ++ax) {
          const int f = frames_h[k];
          g_d[2 * k + ax] = sums[(size_t)f * 4 + ax];
          pg_d[2 * k + ax] = pos_rho2 * g_d[2 * k + ax];
          prev_d[2 * k + ax] = st.dir_d[2 * (size_t)f + ax];
        }
    }
    // Pg: the probe part times ρ² (the object part is g itself)
    check(h, cudaMemcpyAsync(h->last_probe, h->g_probe, np * sizeof(float2),
                             cudaMemcpyDeviceToDevice, h->stream),
          "preconditioned gradient");
    timed(h, kKAxpy, [&] {
      scale_kernel<<<blocks_for(np), 256, 0, h->stream>>>(h->last_probe, (float)rho2, np);
    });
    launched(h, "preconditioned gradient");
    const BhVec pg = {h->g_obj, h->last_probe, refine ? pg_d.data() : nullptr};
    const BhVec prev = {h->dir_obj, h->dir_probe, refine ? prev_d.data() : nullptr};
    double beta = 0.0;
    if (cg) {
      const double hn = bh_hessian(h, frames, n, pg, prev);
      const double hd = bh_hessian(h, frames, n, prev, prev);
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
    double top = -(dot_of(h, h->g_obj, h->dir_obj, no) + dot_of(h, h->g_probe, h->dir_probe, np));
    if (refine)
      for (int i = 0; i < 2 * n; ++i) {
        dir_d[i] = (cg ? beta * prev_d[i] : 0.0) - pg_d[i];
        top -= g_d[i] * dir_d[i];
      }
    const BhVec dir = {h->dir_obj, h->dir_probe, refine ? dir_d.data() : nullptr};
    const double bottom = bh_hessian(h, frames, n, dir, dir);
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
    if (refine) {
      // the direction's offsets part by frame (zero off the batch), and 0.3·α·D_d on the
      // batch's offsets (engine/bh.rs:735-745)
      std::fill(st.dir_d.begin(), st.dir_d.end(), 0.0);
      for (int k = 0; k < n; ++k)
        for (int ax = 0; ax < 2; ++ax) {
          const size_t i = 2 * (size_t)frames_h[k] + ax;
          st.dir_d[i] = dir_d[2 * k + ax];
          st.offsets[i] += kPositionStep * alpha * dir_d[2 * k + ax];
        }
      check(h, copy_sync(h, h->offsets, st.offsets.data(), st.offsets.size() * sizeof(double),
                         cudaMemcpyHostToDevice),
            "offsets");
    }
    ptyb_bh_step s;
    s.batch = (int32_t)b;
    s.count = n;
    s.beta = beta;
    s.alpha = alpha;
    s.top = top;
    s.bottom = bottom;
    h->bh_steps.push_back(s);
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
  if (h->nslice > 1 && h->have_offsets) {
    h->err = "BH through slices runs without the position model";
    return PTYB_INVALID;
  }
  if (h->nslice > 1 && slice_gamma_bytes(h->N, h->K) > 227 * 1024) {
    h->err = "BH through slices: the frame's modes do not fit one cluster's shared memory";
    return PTYB_INVALID;
  }
  if (!std::isfinite(p->position_rho) || !std::isfinite(p->probe_rho)) {
    h->err = "BH probe_rho and position_rho must be finite";
    return PTYB_INVALID;
  }
  return guarded(h, true, [&]() -> int {
    const int size = std::min(p->batch_size, h->P);
    ensure_slots(h, std::min(h->P, h->stack));
    ensure_ml(h);
    const bool pos = h->have_offsets, slices = h->nslice > 1;
    if (slices) {
      const size_t no = (size_t)h->nslice * h->nyo * h->nxo;
      if (!h->last_slices) {
        h->last_slices = alloc<float2>(h, no);
        h->dir_slices = alloc<float2>(h, no);
      }
      if (!h->bh_tmp) h->bh_tmp = alloc<float2>(h, no + (size_t)h->K * h->N * h->N);
    }
    BhHost st;
    if (pos) {
      ensure_spec(h);
      if (h->wave2_slots < h->slots) {
        h->wave2 = alloc<float2>(h, (size_t)h->slots * h->K * h->N * h->N);
        h->wave2_slots = h->slots;
      }
      if (!h->ml_pos_sums) h->ml_pos_sums = alloc<double>(h, (size_t)h->P * 4);
      st.offsets.resize((size_t)h->P * 2);
      st.dir_d.assign((size_t)h->P * 2, 0.0);
      check(h, copy_sync(h, st.offsets.data(), h->offsets, st.offsets.size() * sizeof(double),
                         cudaMemcpyDeviceToHost),
            "offsets");
    }
    std::vector<std::vector<int32_t>> sizes;
    // a fresh run: epoch e's batches from random_batches(nframe, size, seed, e), on the device
    // and (for the offsets' parts) on the host
    upload_orders(h, nepoch, size, p->seed, 0, &sizes, nullptr);
    std::vector<int32_t> order_h, order, sz;
    for (int e = 0; e < nepoch; ++e) {
      random_batches(h->P, size, p->seed, (uint64_t)e, &order, &sz);
      order_h.insert(order_h.end(), order.begin(), order.end());
    }
    begin_call(h);
    for (int ic = 0; ic < nepoch; ++ic) {
      if (slices)
        bh_epoch_slices(h, *p, h->order_all + (size_t)ic * h->P, sizes[ic],
                        size == h->P && ic > 0);
      else
        bh_epoch(h, *p, h->order_all + (size_t)ic * h->P, order_h.data() + (size_t)ic * h->P,
                 sizes[ic], size == h->P && ic > 0, st);
      if (llk_due(calc_llk, ic, nepoch)) {
        if (pos) {
          // every frame's moved probe at the epoch's end, for the LLK
          if (!h->wave_all) h->wave_all = alloc<float2>(h, (size_t)h->P * h->K * h->N * h->N);
          spectrum_of(h, h->probe, h->spec);
          const int stack = std::min(h->P, h->stack);
          for (int s0 = 0; s0 < h->P; s0 += stack)
            move_frames(h, h->iota + s0, std::min(stack, h->P - s0), h->spec,
                        h->wave_all + (size_t)s0 * h->K * h->N * h->N);
        }
        record(h, kAlgBh, llk_pass(h, pos ? h->wave_all : nullptr));
      }
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
