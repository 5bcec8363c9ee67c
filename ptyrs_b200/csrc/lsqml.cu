// LSQML on the GPU (reference engine/gpu/lsqml.rs:75-126; CPU twin engine/lsqml.rs:581-714):
// per batch the frame passes with the far-field step, the object and probe directions, the
// FP64 step sizes and the updates; pty-chi's multislice object; the OPR probe variation
// (engine/opr.rs) and pty-chi's position step.
#include <utility>

#include "engine.cuh"

using namespace ptyb;

namespace ptyb::eng {
namespace {

__global__ void fill_kernel(float* x, float v, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = v;
}

// The preconditioner over every view on pty-chi's schedule (engine/lsqml.rs:676-700).
void lsqml_preconditioner(ptyb_handle* h, bool init) {
  GatherArgs g = gather_args(h, h->iota, h->P);
  g.pre_scale = init ? (float)(h->max_power / (4.0 * h->N * h->N * ((double)h->N * h->N))) : -1.f;
  timed(h, kKIllum, [&] { object_tile_kernel<kGatherIllum><<<ntiles(h), 1024, 0, h->stream>>>(g); });
  launched(h, "illumination");
  check(h, cudaMemsetAsync(h->scal + 1, 0, sizeof(float), h->stream), "memset");
  const size_t n = (size_t)h->nyo * h->nxo;
  timed(h, kKMax, [&] { max_kernel<<<296, 256, 0, h->stream>>>(h->pre, n, h->scal + 1); });
  launched(h, "pre max");
}

// Every slot's own probe planes of the batch into h->wave, or nullptr for the shared probe:
// the probe variation's planes (engine/opr.rs:88-120), each moved by its frame's offset under
// the position model (engine/lsqml.rs:500-523), or the shared probe moved.
const float2* frame_probes(ptyb_handle* h, const int* frames, int nslot);

// The batch's probe direction into h->d_probe (engine/lsqml.rs:200-229): each frame's
// conj(q·O_0)·χ_0 over its slice-0 window into h->field, moved back through the frame's move
// under the position model, and their frame mean. Returns the per-frame directions the mean
// was taken over (the moved-back ones; h->field keeps the raw ones the OPR step also reads).
const float2* probe_directions(ptyb_handle* h, const int* frames, int nslot,
                               const float2* quad, const float2* chi) {
  const int pstride = h->K * h->N * h->N;
  timed(h, kKProbePartial, [&] {
    probe_terms_kernel<<<dim3((h->N * h->N + 255) / 256, nslot), 256, 0, h->stream>>>(
        h->object, quad, chi, frames, h->corners, h->nxo, h->K, h->N, h->field);
  });
  launched(h, "probe terms");
  const float2* dirs = h->field;
  if (h->have_offsets) {
    float2* moved = h->field;
    if (h->opr_on) {
      // the OPR step reads both the raw and the moved-back directions
      moved = h->opr_moved;
      check(h, cudaMemcpyAsync(moved, h->field, (size_t)nslot * pstride * sizeof(float2),
                               cudaMemcpyDeviceToDevice, h->stream),
            "directions");
    }
    check(h, launch_move<kMoveBack>(h, move_args(h, frames, moved), nslot), "probe move back");
    ++h->launches;
    dirs = moved;
  }
  timed(h, kKProbeFinal, [&] {
    probe_finalize_kernel<<<(pstride + 255) / 256, 256, 0, h->stream>>>(
        dirs, nslot, pstride, h->probe, h->d_probe, nullptr, 1.0f / nslot, 1);
  });
  launched(h, "probe direction");
  return dirs;
}

void opr_step(ptyb_handle* h, const int* frames, int count, const float2* moved);

// One LSQML step through pty-chi's multislice object (engine/lsqml.rs:581-643 with
// SliceWaves, engine/multislice.rs): forward through the slices, backward χ per slice, every
// slice's object direction from its incident wave, the probe direction from χ of slice 0,
// slice 0's step sizes jointly with the probe and Eq. 23b on the others. Under the position
// model every frame's probe enters slice 0 moved by its offset (no phase on slice 0), the
// probe directions go back through the moves before their frame mean, and refinement takes
// pty-chi's position step from the middle slice (engine/lsqml.rs:231-270, 500-523).
void lsqml_batch_slices(ptyb_handle* h, const ptyb_lsqml_params& p, const int* frames, int nslot,
                        double* log, int log_stride) {
  const int S = h->nslice;
  const size_t plane = (size_t)h->N * h->N, fplanes = (size_t)h->K * plane;
  const size_t slice_stride = (size_t)nslot * fplanes, no = (size_t)h->nyo * h->nxo;
  const bool refine = h->have_offsets && h->refine_offsets;
  SliceArgs sa = {};
  sa.f = frame_args(h, frames);
  const float2* own = frame_probes(h, frames, nslot);
  if (own) {
    sa.f.probe = own;
    sa.f.probe_stride = (int)fplanes;
  }
  sa.f.cost = p.cost;
  sa.f.nslot = nslot;
  sa.f.a_prev = h->afar_all;
  sa.f.a_prev_by_frame = 1;
  sa.f.a_out = h->afar1;
  sa.tf = h->tf;
  sa.incident = h->incident;
  sa.chi = h->chi_slices;
  sa.nslice = S;
  sa.obj_plane = no;
  check(h, launch_slice<kSliceForward>(h, sa, nslot), "multislice forward");
  ++h->launches;
  sa.f.a_mid = h->afar1;
  sa.f.a_out = h->afar2;
  check(h, launch_slice<kSliceBackward>(h, sa, nslot), "multislice backward");
  ++h->launches;
  for (int s = 0; s < S; ++s) {
    GatherArgs g = gather_args(h, frames, nslot);
    g.upd = h->chi_slices + s * slice_stride;
    g.out = h->d_obj + s * no;
    g.quad = s + 1 == S ? h->quad : h->ones;
    if (s > 0) {
      g.probe = h->incident + (s - 1) * slice_stride;
      g.probe_stride = (int)fplanes;
    } else if (own) {
      g.probe = own;
      g.probe_stride = (int)fplanes;
    }
    timed(h, kKObjLsqml, [&] { object_tile_kernel<kGatherLsqml><<<ntiles(h), 1024, 0, h->stream>>>(g); }, nslot);
    launched(h, "slice object direction");
  }
  // probe direction from χ of slice 0 through slice 0's windows (no phase when S > 1)
  const float2* dirs = nullptr;
  if (own)
    dirs = probe_directions(h, frames, nslot, h->ones, h->chi_slices);
  else
    probe_pass(h, frames, nslot, 1, 0.f, 1.0f / nslot, h->ones, h->chi_slices);
  const double lambda0 = 1.2e-7 * ((double)h->N * h->N) / ((double)h->N * h->N);
  timed(h, kKDots, [&] {
    lsqml_dots_kernel<<<nslot * kDotParts, 512, 0, h->stream>>>(
        h->object, h->d_obj, own ? own : h->probe, h->d_probe, h->ones, h->chi_slices,
        frames, h->corners, h->nxo, h->K, h->N, lambda0, h->sums, own ? (int)fplanes : 0);
  }, nslot);
  launched(h, "step sums");
  // the eigenmodes and the refined weights on slice 0 from the state on entry, before the
  // window derivatives below take h->field, where the frame directions are
  if (h->opr_on) opr_step(h, frames, nslot, dirs);
  if (refine) {
    // pty-chi's position sums on slice S/2 (`slice_for_correction`) from the state on entry:
    // the wave entering it at mode 0 times its phase, its χ and its window's derivatives
    const int sc = S / 2;
    MoveArgs md = move_args(h, frames, h->field);
    md.object = h->object + sc * no;
    check(h, launch_move<kDerivWindow>(h, md, nslot), "window derivative");
    ++h->launches;
    const float2* in = sc == 0 ? own : h->incident + (sc - 1) * slice_stride;
    const float2* q = sc + 1 == S ? h->quad : h->ones;
    timed(h, kKPositionSums, [&] {
      position_sums_kernel<<<nslot, 256, 0, h->stream>>>(h->field, in, (int)fplanes, q,
                                                          h->chi_slices + sc * slice_stride,
                                                          h->K, h->N, h->pos_sums);
    }, nslot);
    launched(h, "position sums");
  }
  const double scale = (double)(S * h->K);
  for (int s = 1; s < S; ++s) {
    timed(h, kKDots, [&] {
      slice_dots_kernel<<<nslot, 512, 0, h->stream>>>(
          h->d_obj + s * no, h->incident + (s - 1) * slice_stride,
          s + 1 == S ? h->quad : nullptr, h->chi_slices + s * slice_stride, frames, h->corners,
          h->nxo, h->K, h->N, h->slice_sums);
    }, nslot);
    launched(h, "slice sums");
    timed(h, kKSolve, [&] {
      slice_solve_kernel<<<1, 1024, 0, h->stream>>>(h->slice_sums, nslot, scale, log + 2 + s,
                                                    log_stride, h->scal + 3 + s);
    });
    launched(h, "slice solve");
  }
  timed(h, kKSolve, [&] {
    lsqml_solve_kernel<<<1, 1024, 0, h->stream>>>(h->sums, nslot, scale, h->afar2, frames,
                                                   h->afar_all, log, h->scal + 2, log_stride);
  });
  launched(h, "step solve");
  for (int s = 0; s < S; ++s) {
    const int which = s == 0 ? 0 : 1 + s;  // relative to scal + 2: so_0, sp, so_1, so_2, …
    timed(h, kKAxpy, [&] {
      axpy_scal_kernel<<<(unsigned)((no + 255) / 256), 256, 0, h->stream>>>(
          h->object + s * no, h->d_obj + s * no, h->scal + 2, which, no);
    });
    launched(h, "slice step");
  }
  timed(h, kKAxpy, [&] {
    axpy_scal_kernel<<<(unsigned)((fplanes + 255) / 256), 256, 0, h->stream>>>(
        h->probe, h->d_probe, h->scal + 2, 1, fplanes);
  });
  launched(h, "probe step");
  if (refine) {
    const double eps = 1e-6 * ((double)h->N * h->N);
    timed(h, kKSolve, [&] {
      position_step_kernel<<<1, 32, 0, h->stream>>>(h->pos_sums, nslot, h->P, eps, frames,
                                                    h->offsets);
    });
    launched(h, "position step");
  }
}

// One LSQML step on a batch (engine/lsqml.rs:581-643), with the position model when offsets
// are set: each frame's probe moved by its offset, the probe directions moved back before
// their frame mean, and with refinement pty-chi's position step after the update.
// The probe variation's batch scratch for h->slots frames and the planes of every frame.
void ensure_opr(ptyb_handle* h) {
  const size_t plane = (size_t)h->N * h->N;
  if (h->opr_slots < h->slots) {
    h->opr_r = alloc<float2>(h, (size_t)h->slots * plane);
    h->opr_sums = alloc<double>(h, (size_t)h->slots * (4 * kOprParts + 2));
    h->opr_p = alloc<double>(h, h->slots);
    h->wave = alloc<float2>(h, (size_t)h->slots * h->K * plane);
    h->opr_moved = alloc<float2>(h, (size_t)h->slots * h->K * plane);
    h->opr_slots = h->slots;
  }
  if (!h->opr_e) {
    h->opr_e = alloc<float2>(h, plane);
    h->opr_scal = alloc<double>(h, 4);
    h->opr_count = alloc<unsigned>(h, 1);
    check(h, cudaMemsetAsync(h->opr_count, 0, sizeof(unsigned), h->stream), "memset");
  }
  if (!h->wave_all) h->wave_all = alloc<float2>(h, (size_t)h->P * h->K * plane);
}

// Every slot's own probe planes under the probe variation into `out` ([slot][K][N][N]).
void opr_planes(ptyb_handle* h, const int* frames, int nslot, float2* out) {
  const int plane = h->N * h->N;
  timed(h, kKOprStep, [&] {
    opr_planes_kernel<<<dim3((plane + 255) / 256, nslot), 256, 0, h->stream>>>(
        h->probe, h->opr_u, h->opr_w, h->opr_has_c ? h->opr_c : nullptr, frames, h->K, h->opr_k,
        plane, out);
  });
  launched(h, "opr planes");
}

const float2* frame_probes(ptyb_handle* h, const int* frames, int nslot) {
  if (h->opr_on) {
    opr_planes(h, frames, nslot, h->wave);
    if (h->have_offsets) {
      check(h, launch_move<kMoveOwn>(h, move_args(h, frames, h->wave), nslot), "planes move");
      ++h->launches;
    }
    return h->wave;
  }
  if (!h->have_offsets) return nullptr;
  ensure_spec(h);
  spectrum_of(h, h->probe, h->spec);
  move_frames(h, frames, nslot, h->spec, h->wave);
  return h->wave;
}

// The OPR step of the batch (engine/opr.rs:122-224) from its frame probe directions, mode-0
// plane of each slot of h->field (the main-mode weights and the weights) and of `moved` (the
// same taken back through the frames' moves, h->field without offsets: the residues), and the
// probe's mode 0 on entry. Two launches for the batch and four per eigenmode: each per-frame
// pass (kOprParts blocks per frame) finishes its batch-wide step (coefficients, weights) in its
// last block, and the Gram–Schmidt step of the residues against an eigenmode runs inside the
// next eigenmode's dots.
void opr_step(ptyb_handle* h, const int* frames, int count, const float2* moved) {
  const int plane = h->N * h->N, k = h->opr_k;
  const size_t dstride = (size_t)h->K * plane;
  const unsigned pb32 = (unsigned)((plane + 31) / 32);
  double* part = h->opr_sums;                                  // [count][parts][≤ 4]
  double* proj = h->opr_sums + (size_t)count * 4 * kOprParts;  // [count][2]
  double* uu = h->opr_scal;
  const dim3 per_frame(count, kOprParts);
  // the batch's frames counted once, on its first launch
  int64_t frames_left = count;
  auto units = [&] { return std::exchange(frames_left, 0); };
  if (h->opr_has_c && h->opr_refine_c) {
    timed(h, kKOprStep, [&] {
      opr_intensity_kernel<<<per_frame, 256, 0, h->stream>>>(h->probe, h->field, dstride,
                                                             h->object, frames, h->corners,
                                                             h->nxo, h->N, h->opr_count, part,
                                                             h->opr_c);
    }, units());
    launched(h, "opr intensity");
  }
  if (k == 0 || count < 2) return;
  timed(h, kKOprStep, [&] {
    opr_residue_kernel<<<pb32, 256, 0, h->stream>>>(moved, dstride, count, plane, h->opr_r);
  }, units());
  launched(h, "opr residues");
  const double a_u = std::min(0.1, (double)count / h->P);
  for (int i = 0; i < k; ++i) {
    float2* u = h->opr_u + (size_t)i * plane;
    const float2* prev = i ? u - plane : nullptr;
    timed(h, kKOprStep, [&] {
      opr_dots_kernel<<<per_frame, 256, 0, h->stream>>>(u, h->opr_r, h->N, prev, proj, uu,
                                                        h->opr_w, frames, k, i, h->opr_count,
                                                        part, h->opr_p);
    });
    launched(h, i ? "opr orthogonalisation and dots" : "opr dots");
    timed(h, kKOprStep, [&] {
      opr_e_kernel<<<pb32, 256, 0, h->stream>>>(h->opr_r, h->opr_p, count, plane, h->opr_e);
    });
    launched(h, "opr e");
    timed(h, kKOprStep, [&] {
      opr_u_kernel<<<1, 1024, 0, h->stream>>>(u, h->opr_e, a_u, plane, uu);
    });
    launched(h, "opr eigenmode step");
    const bool next = i + 1 < k;
    if (h->opr_refine_w || next) {
      timed(h, kKOprStep, [&] {
        opr_weight_proj_kernel<<<per_frame, 256, 0, h->stream>>>(
            u, h->opr_refine_w ? h->field : nullptr, dstride, next ? h->opr_r : nullptr,
            h->object, frames, h->corners, h->nxo, h->N, k, i, h->opr_count, part, proj,
            h->opr_w);
      });
      launched(h, h->opr_refine_w ? "opr weights" : "opr projections");
    }
  }
}

void lsqml_batch(ptyb_handle* h, const ptyb_lsqml_params& p, const int* frames, int nslot,
                 double* log) {
  const int pstride = h->K * h->N * h->N;
  FrameArgs a = frame_args(h, frames);
  a.cost = p.cost;
  const bool opr = h->opr_on;
  const float2* own = frame_probes(h, frames, nslot);
  if (own) {
    a.probe = own;
    a.probe_stride = pstride;
  }
  if (p.cost == PTYB_COST_POISSON) {
    // Forward pass with the xi solver's first pass, backward pass with its second.
    a.nslot = nslot;
    a.icalc = nullptr;
    a.a_prev = h->afar_all;
    a.a_prev_by_frame = 1;
    a.a_out = h->afar1;
    check(h, launch_frame<kStore>(h, a, nslot), "lsqml forward");
    ++h->launches;
    a.a_mid = h->afar1;
    a.a_out = h->afar2;
    check(h, launch_frame<kFromStore>(h, a, nslot), "lsqml backward");
    ++h->launches;
  } else {
    timed(h, kKMisc, [&] {
      fill_kernel<<<(nslot + 255) / 256, 256, 0, h->stream>>>(h->afar2, 0.5f, nslot);
    });
    launched(h, "a_far");
    check(h, launch_frame<kLsqmlFused>(h, a, nslot), "lsqml pass");
    ++h->launches;
  }
  GatherArgs g = gather_args(h, frames, nslot);
  if (own) {
    g.probe = own;
    g.probe_stride = pstride;
  }
  timed(h, kKObjLsqml, [&] { object_tile_kernel<kGatherLsqml><<<ntiles(h), 1024, 0, h->stream>>>(g); }, nslot);
  launched(h, "object direction");
  const float2* dirs = nullptr;
  if (own)
    dirs = probe_directions(h, frames, nslot, h->quad, h->upd);
  else
    probe_pass(h, frames, nslot, 1, 0.f, 1.0f / nslot);
  const double lambda0 = 1.2e-7 * ((double)h->N * h->N) / ((double)h->N * h->N);
  const float2* fprobe = own ? own : h->probe;
  const int fstride = own ? pstride : 0;
  timed(h, kKDots, [&] {
    lsqml_dots_kernel<<<nslot * kDotParts, 512, 0, h->stream>>>(h->object, h->d_obj, fprobe, h->d_probe,
                                                     h->quad, h->upd, frames, h->corners,
                                                     h->nxo, h->K, h->N, lambda0, h->sums,
                                                     fstride);
  }, nslot);
  launched(h, "step sums");
  // the eigenmodes and the refined weights from the state on entry (engine/lsqml.rs:620-621),
  // before the window derivatives below take h->field, where the frame directions are
  if (opr) opr_step(h, frames, nslot, dirs);
  const bool refine = h->have_offsets && h->refine_offsets;
  if (refine) {
    // position directions from the state on entry (engine/lsqml.rs:237-270)
    check(h, launch_move<kDerivWindow>(h, move_args(h, frames, h->field), nslot), "window derivative");
    ++h->launches;
    timed(h, kKPositionSums, [&] {
      position_sums_kernel<<<nslot, 256, 0, h->stream>>>(h->field, h->wave, pstride, h->quad,
                                                          h->upd, h->K, h->N, h->pos_sums);
    }, nslot);
    launched(h, "position sums");
  }
  timed(h, kKSolve, [&] {
    lsqml_solve_kernel<<<1, 1024, 0, h->stream>>>(h->sums, nslot, (double)(1 * h->K), h->afar2,
                                                   frames, h->afar_all, log, h->scal + 2, 3);
  });
  launched(h, "step solve");
  const size_t no = (size_t)h->nyo * h->nxo, np = (size_t)h->K * h->N * h->N;
  timed(h, kKAxpy, [&] {
    axpy_scal_kernel<<<(unsigned)((no + 255) / 256), 256, 0, h->stream>>>(h->object, h->d_obj,
                                                                         h->scal + 2, 0, no);
  });
  launched(h, "object step");
  timed(h, kKAxpy, [&] {
    axpy_scal_kernel<<<(unsigned)((np + 255) / 256), 256, 0, h->stream>>>(h->probe, h->d_probe,
                                                                         h->scal + 2, 1, np);
  });
  launched(h, "probe step");
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

int ptyb_lsqml_slice_steps(ptyb_handle* h, double* dst) {
  if (!h || !dst) return PTYB_INVALID;
  std::copy(h->slice_steps.begin(), h->slice_steps.end(), dst);
  return PTYB_OK;
}

int ptyb_lsqml(ptyb_handle* h, const ptyb_lsqml_params* p, int32_t nepoch, int32_t calc_llk) {
  if (!h || !p) return PTYB_INVALID;
  if (p->batch_size <= 0 || nepoch < 0 ||
      !(p->cost == PTYB_COST_POISSON || p->cost == PTYB_COST_AMPLITUDE)) {
    h->err = "LSQML batch_size must be >= 1 and cost poisson or amplitude";
    return PTYB_INVALID;
  }
  if (std::min(p->batch_size, h->P) > 1024) {
    h->err = "LSQML batches of more than 1024 frames are not supported";
    return PTYB_INVALID;
  }
  return guarded(h, true, [&]() -> int {
    const int size = std::min(p->batch_size, h->P);
    ensure_slots(h, std::max(size, std::min(h->P, h->stack)));
    if (h->opr_on) ensure_opr(h);
    std::vector<std::vector<int32_t>> sizes;
    std::vector<int32_t> last;
    // A fresh run: epochs from 0 (engine/gpu/lsqml.rs:97-105).
    upload_orders(h, nepoch, size, p->seed, 0, &sizes, &last);
    begin_call(h);
    timed(h, kKMisc, [&] {
      fill_kernel<<<(h->P + 255) / 256, 256, 0, h->stream>>>(h->afar_all, 0.5f, h->P);
    });
    launched(h, "a_far");
    for (int ic = 0; ic < nepoch; ++ic) {
      if (ic < 10 || ic % 10 == 0) lsqml_preconditioner(h, ic == 0);
      const int* order = h->order_all + (size_t)ic * h->P;
      int off = 0;
      const int stride = h->log_stride;
      for (int n : sizes[ic]) {
        if (h->nslice > 1)
          lsqml_batch_slices(h, *p, order + off, n, h->steplog + (size_t)off * stride, stride);
        else
          lsqml_batch(h, *p, order + off, n, h->steplog + (size_t)off * stride);
        off += n;
      }
      if (llk_due(calc_llk, ic, nepoch)) {
        if (h->opr_on) {
          // the LLK of every frame's own probe (engine/lsqml.rs:537-551)
          const int stack = std::min(h->P, h->stack);
          for (int s0 = 0; s0 < h->P; s0 += stack) {
            const int n = std::min(stack, h->P - s0);
            float2* planes = h->wave_all + (size_t)s0 * h->K * h->N * h->N;
            opr_planes(h, h->iota + s0, n, planes);
            if (h->have_offsets) {
              check(h, launch_move<kMoveOwn>(h, move_args(h, h->iota + s0, planes), n),
                    "planes move");
              ++h->launches;
            }
          }
          record(h, kAlgLsqml, llk_pass(h, h->wave_all));
        } else {
          record(h, kAlgLsqml, llk_pass(h));
        }
      }
      ++h->cycle;
    }
    end_call(h, "lsqml");
    // The last epoch's steps, for `ptyb_lsqml_steps`.
    h->steps.clear();
    h->slice_steps.clear();
    if (nepoch > 0) {
      const int stride = h->log_stride;
      std::vector<double> log((size_t)h->P * stride);
      check(h, copy_sync(h, log.data(), h->steplog, log.size() * sizeof(double),
                          cudaMemcpyDeviceToHost),
            "steps");
      int b = 0, o = 0;
      for (int n : sizes.back()) {
        for (int i = 0; i < n; ++i) {
          const double* row = log.data() + (size_t)(o + i) * stride;
          ptyb_lsqml_step st;
          st.batch = b;
          st.frame = last[o + i];
          st.a_far = row[0];
          st.a_obj = row[1];
          st.a_probe = row[2];
          h->steps.push_back(st);
          for (int sl = 1; sl < h->nslice; ++sl) h->slice_steps.push_back(row[2 + sl]);
        }
        o += n;
        ++b;
      }
    }
    return PTYB_OK;
  });
}

int ptyb_set_probe_variation(ptyb_handle* h, const double* eigenmodes, int32_t k,
                             const double* weights, int32_t refine_weights,
                             const double* intensity, int32_t refine_intensity) {
  if (!h) return PTYB_INVALID;
  if (k < 0 || (k > 0 && (!eigenmodes || !weights))) {
    h->err = "probe variation: k >= 0 with eigenmodes and weights";
    return PTYB_INVALID;
  }
  if (intensity && k == 0) {
    h->err = "main-mode weights need an eigenmode";
    return PTYB_INVALID;
  }
  return guarded(h, true, [&]() -> int {
    const size_t plane = (size_t)h->N * h->N;
    h->opr_on = k > 0;
    h->opr_k = k;
    h->opr_has_c = intensity != nullptr;
    h->opr_refine_w = refine_weights != 0;
    h->opr_refine_c = refine_intensity != 0;
    if (!h->opr_on) return PTYB_OK;
    h->opr_u = alloc<float2>(h, (size_t)k * plane);
    upload_c64(h, eigenmodes, h->opr_u, (size_t)k * plane, "eigenmodes");
    h->opr_w = alloc<double>(h, (size_t)h->P * k);
    check(h, copy_sync(h, h->opr_w, weights, (size_t)h->P * k * sizeof(double),
                       cudaMemcpyHostToDevice), "weights");
    if (intensity) {
      h->opr_c = alloc<double>(h, h->P);
      check(h, copy_sync(h, h->opr_c, intensity, (size_t)h->P * sizeof(double),
                         cudaMemcpyHostToDevice), "intensity");
    }
    return PTYB_OK;
  });
}

int ptyb_get_probe_variation(ptyb_handle* h, double* eigenmodes, double* weights,
                             double* intensity) {
  if (!h) return PTYB_INVALID;
  return guarded(h, false, [&]() -> int {
    const size_t plane = (size_t)h->N * h->N;
    if (!h->opr_on) return PTYB_OK;
    if (eigenmodes) download_c64(h, h->opr_u, eigenmodes, (size_t)h->opr_k * plane, "eigenmodes");
    if (weights)
      check(h, copy_sync(h, weights, h->opr_w, (size_t)h->P * h->opr_k * sizeof(double),
                         cudaMemcpyDeviceToHost), "weights");
    if (intensity && h->opr_has_c)
      check(h, copy_sync(h, intensity, h->opr_c, (size_t)h->P * sizeof(double),
                         cudaMemcpyDeviceToHost), "intensity");
    return PTYB_OK;
  });
}

}  // extern "C"
