// rPIE on the GPU (reference engine/gpu/rpie.rs:31-63, 198-529; CPU twin
// engine/ptycho.rs:874-1085): per batch the frame pass, the overlap weights, the object and
// probe updates and, under the position model, pty-chi's position step.
#include "engine.cuh"

using namespace ptyb;

namespace ptyb::eng {
namespace {

// One rPIE batch (engine/ptycho.rs:904-1085; GPU launch sequence engine/gpu/rpie.rs:239-345).
void rpie_batch(ptyb_handle* h, const ptyb_rpie_params& p, const int* frames, int nslot) {
  FrameArgs a = frame_args(h, frames);
  GatherArgs g = gather_args(h, frames, nslot);
  const int pstride = h->K * h->N * h->N;
  const bool moved = h->have_offsets, refine = h->have_offsets && h->refine_offsets;
  if (moved) {
    // every frame's probe moved by its offset from the batch-start probe (engine/ptycho.rs:
    // 920-935); the views' waves in the frame pass and the object gathers
    ensure_spec(h);
    spectrum_of(h, h->probe, h->spec);
    move_frames(h, frames, nslot, h->spec, h->wave);
    a.probe = h->wave;
    a.probe_stride = pstride;
    g.probe = h->wave;
    g.probe_stride = pstride;
  }
  check(h, launch_frame<kRpie>(h, a, nslot), "rpie frame pass");
  ++h->launches;
  if (p.update_object) {
    check(h, cudaMemsetAsync(h->scal, 0, sizeof(float), h->stream), "memset");
    timed(h, kKObjOverlap, [&] { object_tile_kernel<kGatherOverlap><<<ntiles(h), 1024, 0, h->stream>>>(g); }, nslot);
    launched(h, "overlap max");
  }
  if (refine) {
    // pty-chi's position sums from mode 0 of the batch-start state (engine/ptycho.rs:1037-1064)
    check(h, launch_move<kDerivWindow>(h, move_args(h, frames, h->field), nslot), "window derivative");
    ++h->launches;
    timed(h, kKPositionSums, [&] {
      position_sums_kernel<<<nslot, 256, 0, h->stream>>>(h->field, h->wave, pstride, h->quad,
                                                          h->upd, h->K, h->N, h->pos_sums);
    }, nslot);
    launched(h, "position sums");
  }
  const int count = h->K * h->N * h->N;
  int nchunk = 0;
  if (p.update_probe && moved) {
    // each frame's rPIE probe direction moved back by −d (engine/ptycho.rs:1007-1035)
    timed(h, kKProbePartial, [&] {
      probe_terms_kernel<<<dim3((h->N * h->N + 255) / 256, nslot), 256, 0, h->stream>>>(
          h->object, h->quad, h->upd, frames, h->corners, h->nxo, h->K, h->N, h->field, h->omax,
          (float)p.probe_alpha);
    }, nslot);
    launched(h, "probe terms");
    check(h, launch_move<kMoveBack>(h, move_args(h, frames, h->field), nslot), "probe move back");
    ++h->launches;
  } else if (p.update_probe) {
    // Reads the batch-start object, so it runs before the object update.
    const int chunk = probe_chunk(h, nslot, &nchunk);
    ProbeArgs pa = {};
    pa.object = h->object;
    pa.quad = h->quad;
    pa.upd = h->upd;
    pa.frames = frames;
    pa.corners = h->corners;
    pa.omax = h->omax;
    pa.partial = h->partial;
    pa.alpha = (float)p.probe_alpha;
    pa.nslot = nslot;
    pa.chunk = chunk;
    pa.nxo = h->nxo;
    pa.K = h->K;
    pa.N = h->N;
    pa.mode = 0;
    dim3 grid((h->N * h->N + 255) / 256, nchunk);
    timed(h, kKProbePartial, [&] { probe_partial_kernel<<<grid, 256, 0, h->stream>>>(pa); }, pa.nslot);
    launched(h, "probe partial");
  }
  if (p.update_object) {
    g.alpha = (float)p.obj_alpha;
    g.step = (float)p.obj_step;
    timed(h, kKObjRpie, [&] { object_tile_kernel<kGatherRpie><<<ntiles(h), 1024, 0, h->stream>>>(g); }, g.nslot);
    launched(h, "object update");
  }
  if (p.update_probe) {
    // P += step/nbatch · Σ (frames in order); the gathers above read the batch-start probe
    timed(h, kKProbeFinal, [&] {
      probe_finalize_kernel<<<(count + 255) / 256, 256, 0, h->stream>>>(
          moved ? h->field : h->partial, moved ? nslot : nchunk, count, h->probe, nullptr,
          nullptr, (float)(p.probe_step / nslot), 0);
    });
    launched(h, "probe update");
  }
  if (refine) {
    const double eps = 1e-6 * ((double)h->N * h->N);
    timed(h, kKSolve, [&] {
      position_step_kernel<<<1, 32, 0, h->stream>>>(h->pos_sums, nslot, h->P, eps, frames,
                                                    h->offsets);
    });
    launched(h, "position step");
  }
}

}  // namespace
}  // namespace ptyb::eng

using namespace ptyb::eng;

extern "C" {

int ptyb_rpie(ptyb_handle* h, const ptyb_rpie_params* p, int32_t nepoch) {
  if (!h || !p) return PTYB_INVALID;
  if (p->batch_size <= 0 || nepoch < 0) {
    h->err = "rPIE batch_size must be >= 1";
    return PTYB_INVALID;
  }
  if (h->nobj != 1) {
    h->err = "rPIE needs exactly one object mode";
    return PTYB_INVALID;
  }
  if (h->nslice > 1) {
    h->err = "rPIE runs on a single-slice object";
    return PTYB_INVALID;
  }
  return guarded(h, true, [&]() -> int {
    const int bs = std::min(p->batch_size, h->P);
    ensure_slots(h, std::max(bs, std::min(h->P, h->stack)));
    std::vector<std::vector<int32_t>> sizes;
    upload_orders(h, nepoch, p->batch_size, p->seed, h->cycle, &sizes, nullptr);
    begin_call(h);
    for (int ic = 0; ic < nepoch; ++ic) {
      const int* order = h->order_all + (size_t)ic * h->P;
      int off = 0;
      for (int n : sizes[ic]) {
        rpie_batch(h, *p, order + off, n);
        off += n;
      }
      if (llk_due(p->calc_llk, ic, nepoch)) record(h, kAlgRpie, llk_pass(h));
      ++h->cycle;
    }
    end_call(h, "rpie");
    return PTYB_OK;
  });
}

}  // extern "C"
