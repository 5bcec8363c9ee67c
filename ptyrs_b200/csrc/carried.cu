// AP, DM and RAAR on the GPU (reference engine/gpu/{ap,dm,raar}.rs; CPU twins
// engine/ptycho.rs:609-754): the carried exit waves mixed and projected by the frame kernel's
// carry mode, the inertia blends of object and probe, and under the position model the
// line-searched probe step and the position step.
#include "engine.cuh"

using namespace ptyb;

namespace ptyb::eng {
namespace {

// AP / DM / RAAR (engine/ptycho.rs:609-754) ---------------------------------------------

// Every frame's carried exit waves (and RAAR's iterate), allocated on first use.
void ensure_carry(ptyb_handle* h, bool iterate) {
  const size_t n = (size_t)h->P * h->K * h->N * h->N;
  if (!h->carry) h->carry = alloc<float2>(h, n);
  if (iterate && !h->carry_it) h->carry_it = alloc<float2>(h, n);
  if (!h->probe_norm) h->probe_norm = alloc<float>(h, (size_t)h->N * h->N);
  if (!h->blend_norm) h->blend_norm = alloc<float>(h, (size_t)h->nyo * h->nxo);
}

// The frame kernel's carry mode over every frame, stack by stack: the carried waves become
// Π(S) + c_refl·(PO − S) with S = c_po·PO + c_psi·carried + c_it·iterate; with `llk`, each
// frame's LLK sums of the field it projects go to h->llk.
void carry_pass(ptyb_handle* h, float c_po, float c_psi, float c_it, float c_refl, bool llk,
                bool iterate, const float2* waves = nullptr) {
  const int stack = std::min(h->P, h->stack);
  const size_t pstride = (size_t)h->K * h->N * h->N;
  for (int s0 = 0; s0 < h->P; s0 += stack) {
    const int n = std::min(stack, h->P - s0);
    FrameArgs a = frame_args(h, h->iota + s0);
    a.carry = h->carry + s0 * pstride;
    a.iter = iterate ? h->carry_it + s0 * pstride : nullptr;
    a.c_po = c_po;
    a.c_psi = c_psi;
    a.c_it = c_it;
    a.c_refl = c_refl;
    a.llk = llk ? h->llk + (size_t)s0 * 4 : nullptr;
    if (waves) {
      // each frame's moved probe in place of P (the position model)
      a.probe = waves + s0 * pstride;
      a.probe_stride = (int)pstride;
    }
    check(h, launch_frame<kCarry>(h, a, n), "carry pass");
    ++h->launches;
  }
}

// psi_to_obj_probe's object blend from the carried waves and the current probe
// (engine/ops.rs:352-381): one tile-owned pass writes the numerator and the norm and takes the
// norm's maximum, then the blend runs per pixel.
void object_blend(ptyb_handle* h, double inertia, const float2* waves = nullptr) {
  GatherArgs g = gather_args(h, h->iota, h->P);
  g.upd = h->carry;
  if (waves) {
    // under the move: num += carried·conj(W), norm += |W|² (engine/features.rs:855-890)
    g.probe = waves;
    g.probe_stride = h->K * h->N * h->N;
  }
  g.pmax = h->scal + kScalObjNorm;
  g.out = h->d_obj;
  g.pre = h->blend_norm;
  check(h, cudaMemsetAsync(g.pmax, 0, sizeof(float), h->stream), "memset");
  timed(h, kKObjBlend, [&] { object_tile_kernel<kGatherBlend><<<ntiles(h), 1024, 0, h->stream>>>(g); }, h->P);
  launched(h, "object blend sums");
  const size_t no = (size_t)h->nyo * h->nxo;
  timed(h, kKAxpy, [&] {
    blend_apply_kernel<<<(unsigned)((no + 255) / 256), 256, 0, h->stream>>>(
        h->object, h->d_obj, h->blend_norm, g.pmax, (float)inertia, no);
  });
  launched(h, "object blend");
}

// The probe blend's chunk sums Σ conj(q·O)·carried and Σ|O|² from the current object; the
// blend itself is probe_blend_finish, so AP's probe sums can read the object before its update.
int probe_blend_sums(ptyb_handle* h, int mode = 2) {
  int nchunk = 0;
  const int chunk = probe_chunk(h, h->P, &nchunk);
  const int plane = h->N * h->N;
  if (nchunk > h->max_den_chunks) {
    h->partial_den = alloc<float>(h, (size_t)nchunk * plane);
    h->max_den_chunks = nchunk;
  }
  ProbeArgs p = {};
  p.object = h->object;
  p.quad = h->quad;
  p.upd = h->carry;
  p.frames = h->iota;
  p.corners = h->corners;
  p.partial = h->partial;
  p.partial_den = h->partial_den;
  p.nslot = h->P;
  p.chunk = chunk;
  p.nxo = h->nxo;
  p.K = h->K;
  p.N = h->N;
  p.mode = mode;
  dim3 grid((plane + 255) / 256, nchunk);
  timed(h, kKProbePartial, [&] { probe_partial_kernel<<<grid, 256, 0, h->stream>>>(p); }, h->P);
  launched(h, "probe partial");
  return nchunk;
}

void probe_blend_finish(ptyb_handle* h, int nchunk, double inertia) {
  const int plane = h->N * h->N, count = h->K * plane;
  float* nmax = h->scal + kScalProbeNorm;
  check(h, cudaMemsetAsync(nmax, 0, sizeof(float), h->stream), "memset");
  timed(h, kKProbeFinal, [&] {
    probe_norm_kernel<<<(plane + 255) / 256, 256, 0, h->stream>>>(h->partial_den, nchunk, plane,
                                                                  h->probe_norm, nmax);
  });
  launched(h, "probe norm");
  timed(h, kKProbeFinal, [&] {
    probe_finalize_kernel<<<(count + 255) / 256, 256, 0, h->stream>>>(
        h->partial, nchunk, count, h->probe, nullptr, nullptr, (float)inertia, 3, h->probe_norm,
        nmax, plane);
  });
  launched(h, "probe blend");
}

// Every frame's moved probe of the current probe and offsets into h->wave_all, and the
// probe's spectrum DFT(q·P) into h->spec.
void move_all_frames(ptyb_handle* h) {
  spectrum_of(h, h->probe, h->spec);
  const int stack = std::min(h->P, h->stack);
  for (int s0 = 0; s0 < h->P; s0 += stack)
    move_frames(h, h->iota + s0, std::min(stack, h->P - s0), h->spec,
                h->wave_all + (size_t)s0 * h->K * h->N * h->N);
}

// Under the position model, the buffers of AP / DM / RAAR: the moved probes, the spectra, a
// stack of planes, the position sums and the probe step's.
void ensure_carry_moves(ptyb_handle* h) {
  const size_t np = (size_t)h->K * h->N * h->N;
  ensure_spec(h);
  if (!h->wave_all) h->wave_all = alloc<float2>(h, (size_t)h->P * np);
  if (h->wave2_slots < h->slots) {
    h->wave2 = alloc<float2>(h, (size_t)h->slots * np);
    h->wave2_slots = h->slots;
  }
  if (!h->ml_pos_sums) h->ml_pos_sums = alloc<double>(h, (size_t)h->P * 4);
  if (!h->pcg_g) {
    h->pcg_g = alloc<float2>(h, np);
    h->pcg_step = alloc<float2>(h, np);
    h->pcg_spec = alloc<float2>(h, np);
    h->pcg_comp = alloc<float2>(h, np);
    h->pcg_norms = alloc<double>(h, (size_t)h->P * h->K);
    h->pcg_modes = alloc<double>(h, (size_t)h->K * 2);
  }
}

// The position sums of the carried waves against the model of the current object and moved
// probes (engine/features.rs:992-1025) into h->ml_pos_sums; h->spec must be the probe's.
void carried_position_sums(ptyb_handle* h) {
  const int stack = std::min(h->P, h->stack);
  const size_t pstride = (size_t)h->K * h->N * h->N;
  for (int s0 = 0; s0 < h->P; s0 += stack) {
    const int n = std::min(stack, h->P - s0);
    MoveArgs md = move_args(h, h->iota + s0, nullptr);
    md.spec = h->spec;
    md.c = h->carry + s0 * pstride;
    md.minus = h->wave_all + s0 * pstride;
    md.sums = h->ml_pos_sums;
    check(h, launch_move<kDerivSums>(h, md, n), "position sums");
    ++h->launches;
  }
}

// The probe's update under the move (engine/features.rs:673-712), from the current object and
// the moved probes in h->wave_all: g = A^H(carried − A·P) through the move's adjoint, frame by
// frame; per mode the step s = g / (Σ|O|² + reg) and α = <g, s> / (‖A·s‖² + reg·‖s‖²) where
// <g, s> > 0; P += α·s.
void probe_pcg_step(ptyb_handle* h, double inertia) {
  const int stack = std::min(h->P, h->stack);
  const int plane = h->N * h->N, K = h->K;
  const size_t pstride = (size_t)K * plane;
  check(h, cudaMemsetAsync(h->pcg_spec, 0, pstride * sizeof(float2), h->stream), "memset");
  check(h, cudaMemsetAsync(h->pcg_comp, 0, pstride * sizeof(float2), h->stream), "memset");
  for (int s0 = 0; s0 < h->P; s0 += stack) {
    const int n = std::min(stack, h->P - s0);
    MoveArgs mb = move_args(h, h->iota + s0, h->wave2);
    mb.c = h->carry + s0 * pstride;
    mb.minus = h->wave_all + s0 * pstride;
    check(h, launch_move<kBackSpectrum>(h, mb, n), "probe residual spectra");
    ++h->launches;
    timed(h, kKProbeFinal, [&] {
      probe_finalize_kernel<<<((int)pstride + 255) / 256, 256, 0, h->stream>>>(
          h->wave2, n, (int)pstride, nullptr, h->pcg_spec, h->pcg_comp, 1.f, 2);
    }, n);
    launched(h, "probe residual sum");
  }
  MoveArgs mi = move_args(h, h->iota, h->pcg_g);
  mi.spec = h->pcg_spec;
  check(h, launch_move<kPlainInverse>(h, mi, 1), "probe residual");
  ++h->launches;
  // Σ|O|² per probe pixel and its maximum
  const int nchunk = probe_blend_sums(h, 3);
  float* nmax = h->scal + kScalProbeNorm;
  check(h, cudaMemsetAsync(nmax, 0, sizeof(float), h->stream), "memset");
  timed(h, kKProbeFinal, [&] {
    probe_norm_kernel<<<(plane + 255) / 256, 256, 0, h->stream>>>(h->partial_den, nchunk, plane,
                                                                  h->probe_norm, nmax);
  });
  launched(h, "probe norm");
  timed(h, kKProbeFinal, [&] {
    probe_pcg_step_kernel<<<K, 1024, 0, h->stream>>>(h->pcg_g, h->probe_norm, nmax,
                                                     (float)inertia, plane, h->pcg_step,
                                                     h->pcg_modes);
  });
  launched(h, "probe step");
  // ‖A·s‖²: the step moved for every frame, weighted by |O|²
  spectrum_of(h, h->pcg_step, h->spec_d);
  for (int s0 = 0; s0 < h->P; s0 += stack) {
    const int n = std::min(stack, h->P - s0);
    move_frames(h, h->iota + s0, n, h->spec_d, h->wave2);
    timed(h, kKMisc, [&] {
      weighted_norm_kernel<<<dim3(n, K), 256, 0, h->stream>>>(h->wave2, h->object, h->iota + s0,
                                                              h->corners, h->nxo, h->N, K,
                                                              h->pcg_norms + (size_t)s0 * K);
    }, n);
    launched(h, "step norms");
  }
  std::vector<double> modes((size_t)K * 2), norms((size_t)h->P * K);
  check(h, cudaMemcpyAsync(modes.data(), h->pcg_modes, modes.size() * sizeof(double),
                           cudaMemcpyDeviceToHost, h->stream),
        "step sums");
  check(h, cudaMemcpyAsync(norms.data(), h->pcg_norms, norms.size() * sizeof(double),
                           cudaMemcpyDeviceToHost, h->stream),
        "step sums");
  check(h, cudaStreamSynchronize(h->stream), "step sums");
  ModeCoefs alpha = {};
  for (int m = 0; m < K; ++m) {
    double curv = modes[2 * m + 1];
    for (int f = 0; f < h->P; ++f) curv += norms[(size_t)f * K + m];
    const double slope = modes[2 * m];
    alpha.c[m] = slope > 0.0 ? (float)(slope / curv) : 0.f;
  }
  timed(h, kKAxpy, [&] {
    probe_modes_axpy_kernel<<<((int)pstride + 255) / 256, 256, 0, h->stream>>>(
        h->probe, h->pcg_step, alpha, plane, (int)pstride);
  });
  launched(h, "probe step");
}

// DM's and RAAR's update (engine/ptycho.rs:732-754): `loops` times an object-only then a
// probe-only update, the probe's from the new object; under the position model each from the
// current probe's moves (recomputed after a probe step), the probe's by the step of
// probe_pcg_step, and the position sums come first, from the waves the cycle starts with.
void update_obj_probe(ptyb_handle* h, bool uo, double oi, bool up, double pi, int loops) {
  if (h->have_offsets) {
    bool fresh = true;  // h->wave_all holds the current probe's moves
    for (int l = 0; l < loops; ++l) {
      if (uo) {
        if (!fresh) move_all_frames(h);
        fresh = true;
        object_blend(h, oi, h->wave_all);
      }
      if (up) {
        if (!fresh) move_all_frames(h);
        probe_pcg_step(h, pi);
        fresh = false;
      }
    }
    return;
  }
  for (int l = 0; l < loops; ++l) {
    if (uo) object_blend(h, oi);
    if (up) probe_blend_finish(h, probe_blend_sums(h), pi);
  }
}

// AP, DM and RAAR run on a single-slice object.
int carried_refusal(ptyb_handle* h, int32_t ncycle, const char* what) {
  if (ncycle < 0) {
    h->err = "ncycle must be >= 0";
    return PTYB_INVALID;
  }
  if (h->nslice > 1) {
    h->err = std::string(what) + " runs on a single-slice object";
    return PTYB_INVALID;
  }
  return PTYB_OK;
}

// DM (RAAR when `raar`) cycles (engine/ptycho.rs:653-730): the LLK of the estimate the cycle
// starts from when due, the mix and projection of the carried waves, the updates, and after a
// recorded cycle the balance of Σ|O| and Σ|P|.
int carried_cycles(ptyb_handle* h, bool raar, double mix, bool uo, double oi, bool up, double pi,
                   int loops, int calc_llk, bool ramp, int32_t ncycle) {
  return guarded(h, true, [&]() -> int {
    ensure_slots(h, std::min(h->P, h->stack));
    ensure_carry(h, raar);
    const bool moves = h->have_offsets, refine = moves && h->refine_offsets;
    if (moves) ensure_carry_moves(h);
    const float2* waves = moves ? h->wave_all : nullptr;
    begin_call(h);
    for (int ic = 0; ic < ncycle; ++ic) {
      const bool due = llk_due(calc_llk, ic, ncycle);
      if (moves) move_all_frames(h);
      ptyb_llk l = {};
      if (due) l = llk_pass(h, waves);
      if (ic == 0) {
        carry_pass(h, 1.f, 0.f, 0.f, 0.f, false, raar, waves);
      } else if (raar) {
        // psi ← (1 − b/2)·psi + (b/2)·(2·PO − it), the next iterate, then Π
        const double hb = 0.5 * mix;
        carry_pass(h, (float)(2.0 * hb), (float)(1.0 - hb), (float)(-hb), 0.f, false, true,
                   waves);
      } else {
        // refl = (2 − a)·PO − (1 − a)·psi; psi ← Π(refl) + (1 − a)·(PO − refl)
        carry_pass(h, (float)(2.0 - mix), (float)(-(1.0 - mix)), 0.f, (float)(1.0 - mix), false,
                   false, waves);
      }
      if (refine) carried_position_sums(h);
      update_obj_probe(h, uo, oi, up, pi, loops);
      if (refine) {
        timed(h, kKSolve, [&] {
          ml_position_step_kernel<<<1, 1024, 0, h->stream>>>(h->ml_pos_sums, h->P, h->offsets);
        });
        launched(h, "position step");
      }
      if (due) {
        record(h, raar ? kAlgRaar : kAlgDm, l);
        split_scale(h, 1.0, nullptr);
      }
      ++h->cycle;
    }
    if (ramp) zero_phase_ramp(h);
    end_call(h, raar ? "raar" : "dm");
    return PTYB_OK;
  });
}

}  // namespace
}  // namespace ptyb::eng

using namespace ptyb::eng;

extern "C" {

int ptyb_ap(ptyb_handle* h, const ptyb_ap_params* p, int32_t ncycle) {
  if (!h || !p) return PTYB_INVALID;
  if (const int e = carried_refusal(h, ncycle, "AP")) return e;
  return guarded(h, true, [&]() -> int {
    ensure_slots(h, std::min(h->P, h->stack));
    ensure_carry(h, false);
    const bool uo = p->update_object != 0, up = p->update_probe != 0;
    const bool moves = h->have_offsets, refine = moves && h->refine_offsets;
    if (moves) ensure_carry_moves(h);
    begin_call(h);
    for (int ic = 0; ic < ncycle; ++ic) {
      // the LLK of the estimate comes from the field the projection reads
      const bool due = llk_due(p->calc_llk, ic, ncycle);
      if (moves) move_all_frames(h);
      carry_pass(h, 1.f, 0.f, 0.f, 0.f, due, false, moves ? h->wave_all : nullptr);
      ptyb_llk l = {};
      if (due) l = llk_of_frames(h);
      if (moves) {
        // under the move (engine/ptycho.rs:627-636): the position sums against the arrays the
        // projection read, the probe's step from the old object, the object's blend under the
        // old probe's moves, then the position step
        if (refine) carried_position_sums(h);
        if (up) probe_pcg_step(h, p->probe_inertia);
        if (uo) object_blend(h, p->obj_inertia, h->wave_all);
        if (refine) {
          timed(h, kKSolve, [&] {
            ml_position_step_kernel<<<1, 1024, 0, h->stream>>>(h->ml_pos_sums, h->P, h->offsets);
          });
          launched(h, "position step");
        }
      } else {
        // both updates from the old arrays: the probe's sums read the object before its blend
        const int nchunk = up ? probe_blend_sums(h) : 0;
        if (uo) object_blend(h, p->obj_inertia);
        if (up) probe_blend_finish(h, nchunk, p->probe_inertia);
      }
      if (due) record(h, kAlgAp, l);
      ++h->cycle;
    }
    if (p->zero_phase_ramp) zero_phase_ramp(h);
    end_call(h, "ap");
    return PTYB_OK;
  });
}

int ptyb_dm(ptyb_handle* h, const ptyb_dm_params* p, int32_t ncycle) {
  if (!h || !p) return PTYB_INVALID;
  if (const int e = carried_refusal(h, ncycle, "DM")) return e;
  if (p->loop_obj_probe < 0) {
    h->err = "loop_obj_probe must be >= 0";
    return PTYB_INVALID;
  }
  return carried_cycles(h, false, p->alpha, p->update_object != 0, p->obj_inertia,
                        p->update_probe != 0, p->probe_inertia, p->loop_obj_probe, p->calc_llk,
                        p->zero_phase_ramp != 0, ncycle);
}

int ptyb_raar(ptyb_handle* h, const ptyb_raar_params* p, int32_t ncycle) {
  if (!h || !p) return PTYB_INVALID;
  if (const int e = carried_refusal(h, ncycle, "RAAR")) return e;
  if (p->loop_obj_probe < 0) {
    h->err = "loop_obj_probe must be >= 0";
    return PTYB_INVALID;
  }
  return carried_cycles(h, true, p->beta, p->update_object != 0, p->obj_inertia,
                        p->update_probe != 0, p->probe_inertia, p->loop_obj_probe, p->calc_llk,
                        p->zero_phase_ramp != 0, ncycle);
}

}  // extern "C"
