// Poisson ML conjugate gradient on the GPU (reference engine/gpu/ml.rs:38-83; CPU twin
// engine/ptycho.rs:497-842) and the hand-written adjoint `ptyb_gradients` (object, probe and
// position gradients, through every slice of a multislice object).
#include "engine.cuh"

using namespace ptyb;

namespace ptyb::eng {

// Every slice's 2·∂L/∂O_s* and the probe's 2·∂L/∂P* of the Poisson LLK sum (or with cost
// kCostBh BH's amplitude cost) through a multislice object over `n` frames (every frame when
// null) (the adjoint of engine/multislice.rs:87-173, 266-286, 399-438): per stack, the exit
// wave's gradient back-propagated through the slices on chip, then per slice
// Σ conj(q_s·in_s)·g_s gathered in frame order, the probe's Σ conj(O_0)·g_0.
void slice_gradients(ptyb_handle* h, bool uo, bool up, const int* frames_in, int nframes,
                     int cost) {
  if (!frames_in) {
    frames_in = h->iota;
    nframes = h->P;
  }
  const int S = h->nslice, stack = std::min(nframes, h->stack);
  ensure_slots(h, stack);
  ensure_ml(h);
  const size_t plane = (size_t)h->N * h->N, fplanes = (size_t)h->K * plane;
  const size_t no = (size_t)h->nyo * h->nxo;
  if (!h->g_slices) {
    h->g_slices = alloc<float2>(h, (size_t)S * no);
    h->g_slices_c = alloc<float2>(h, (size_t)S * no);
  }
  check(h, cudaMemsetAsync(h->g_slices, 0, (size_t)S * no * sizeof(float2), h->stream), "memset");
  check(h, cudaMemsetAsync(h->g_slices_c, 0, (size_t)S * no * sizeof(float2), h->stream), "memset");
  check(h, cudaMemsetAsync(h->g_probe, 0, fplanes * sizeof(float2), h->stream), "memset");
  check(h, cudaMemsetAsync(h->g_probe_c, 0, fplanes * sizeof(float2), h->stream), "memset");
  for (int s0 = 0; s0 < nframes; s0 += stack) {
    const int n = std::min(stack, nframes - s0);
    const int* frames = frames_in + s0;
    const size_t slice_stride = (size_t)n * fplanes;
    SliceArgs sa = {};
    sa.f = frame_args(h, frames);
    sa.f.nslot = n;
    sa.f.cost = cost;
    sa.tf = h->tf;
    sa.incident = h->incident;
    sa.chi = h->chi_slices;
    sa.nslice = S;
    sa.obj_plane = no;
    check(h, launch_slice<kSliceGrad>(h, sa, n), "multislice gradient");
    ++h->launches;
    for (int s = 0; uo && s < S; ++s) {
      GatherArgs g = gather_args(h, frames, n);
      g.upd = h->chi_slices + s * slice_stride;
      g.out = h->g_slices + s * no;
      g.comp = h->g_slices_c + s * no;
      g.quad = s + 1 == S ? h->quad : h->ones;
      if (s > 0) {
        g.probe = h->incident + (s - 1) * slice_stride;
        g.probe_stride = (int)fplanes;
      }
      timed(h, kKObjMl, [&] { object_tile_kernel<kGatherMl><<<ntiles(h), 1024, 0, h->stream>>>(g); }, n);
      launched(h, "slice gradient");
    }
    if (up) {
      int nchunk = 0;
      const int chunk = probe_chunk(h, n, &nchunk);
      ProbeArgs pa = {};
      pa.object = h->object;
      pa.quad = h->ones;
      pa.upd = h->chi_slices;
      pa.frames = frames;
      pa.corners = h->corners;
      pa.omax = h->omax;
      pa.partial = h->partial;
      pa.nslot = n;
      pa.chunk = chunk;
      pa.nxo = h->nxo;
      pa.K = h->K;
      pa.N = h->N;
      pa.mode = 1;
      dim3 grid((h->N * h->N + 255) / 256, nchunk);
      timed(h, kKProbePartial, [&] { probe_partial_kernel<<<grid, 256, 0, h->stream>>>(pa); }, n);
      launched(h, "probe gradient");
      const int count = (int)fplanes;
      timed(h, kKProbeFinal, [&] {
        probe_finalize_kernel<<<(count + 255) / 256, 256, 0, h->stream>>>(
            h->partial, nchunk, count, nullptr, h->g_probe, h->g_probe_c, 1.f, 2);
      });
      launched(h, "probe gradient sum");
    }
  }
}

// Shared memory of the multislice line search for frames of side N with K modes.
size_t slice_gamma_bytes(int N, int K) {
  switch (N) {
    case 64: return slice_gamma_smem_bytes<64, gamma_cluster(64)>(K);
    case 96: return slice_gamma_smem_bytes<96, gamma_cluster(96)>(K);
    case 128: return slice_gamma_smem_bytes<128, gamma_cluster(128)>(K);
    case 192: return slice_gamma_smem_bytes<192, gamma_cluster(192)>(K);
    case 256: return slice_gamma_smem_bytes<256, gamma_cluster(256)>(K);
  }
  return ~size_t(0);
}

namespace {

// The Poisson gradient numerators of object and probe over every frame, by stacks in frame
// order (engine/ptycho.rs:497-561).
// The Poisson gradients of the object and the probe (engine/ptycho.rs:497-569) from one
// detector field per frame, which is kept for the line search; with `refine`, the position
// sums of AP, DM and ML from the magnitude projection of the same field (engine/ptycho.rs:
// 470-480, engine/features.rs:992-1025). Under the position model the probe gradient goes
// back through the move's adjoint in the spectrum, frame by frame (features.rs:897-957).
void ml_gradients(ptyb_handle* h, bool uo, bool up, bool refine, bool pos_grad = false) {
  const size_t no = (size_t)h->nyo * h->nxo, np = (size_t)h->K * h->N * h->N;
  check(h, cudaMemsetAsync(h->g_obj, 0, no * sizeof(float2), h->stream), "memset");
  check(h, cudaMemsetAsync(h->g_obj_c, 0, no * sizeof(float2), h->stream), "memset");
  check(h, cudaMemsetAsync(h->g_probe, 0, np * sizeof(float2), h->stream), "memset");
  check(h, cudaMemsetAsync(h->g_probe_c, 0, np * sizeof(float2), h->stream), "memset");
  if (h->have_offsets)
    check(h, cudaMemsetAsync(h->g_probe_spec, 0, np * sizeof(float2), h->stream), "memset");
  const int stack = std::min(h->P, h->stack);
  const int pstride = h->K * h->N * h->N;
  for (int s0 = 0; s0 < h->P; s0 += stack) {
    const int n = std::min(stack, h->P - s0);
    const int* frames = h->iota + s0;
    FrameArgs a = frame_args(h, frames);
    // the gradient field g of these frames, kept for the line search
    float2* gfield = h->g_all + (size_t)s0 * pstride;
    a.out = gfield;
    const float2* waves = h->have_offsets ? h->wave_all + (size_t)s0 * pstride : nullptr;
    if (waves) {
      // each frame's moved probe conj(q)·T_d(q·P) in place of P (engine/ptycho.rs:373-450)
      a.probe = waves;
      a.probe_stride = pstride;
    }
    a.psi_out = h->psi_all + (size_t)s0 * pstride;
    check(h, launch_frame<kMlGrad>(h, a, n), "ml gradient pass");
    ++h->launches;
    if (refine) {
      // the magnitude projection's change of the exit wave from the kept Ψ
      FrameArgs ap = a;
      ap.out = h->field;
      check(h, launch_frame<kProjectKept>(h, ap, n), "magnitude projection");
      ++h->launches;
    }
    if (uo) {
      GatherArgs g = gather_args(h, frames, n);
      g.upd = gfield;
      g.out = h->g_obj;
      g.comp = h->g_obj_c;
      if (waves) {
        g.probe = waves;
        g.probe_stride = pstride;
      }
      timed(h, kKObjMl, [&] { object_tile_kernel<kGatherMl><<<ntiles(h), 1024, 0, h->stream>>>(g); }, n);
      launched(h, "object gradient");
    }
    if (up && h->have_offsets) {
      // DFT(conj(O_win)·g)·exp(+2πi f·d) per frame, summed in frame order
      MoveArgs mb = move_args(h, frames, h->wave2);
      mb.c = gfield;
      check(h, launch_move<kBackSpectrum>(h, mb, n), "probe gradient spectra");
      ++h->launches;
      timed(h, kKProbeFinal, [&] {
        probe_finalize_kernel<<<(pstride + 255) / 256, 256, 0, h->stream>>>(
            h->wave2, n, pstride, nullptr, h->g_probe_spec, h->g_probe_c, 1.f, 2);
      }, n);
      launched(h, "probe gradient sum");
    } else if (up) {
      int nchunk = 0;
      const int chunk = probe_chunk(h, n, &nchunk);
      ProbeArgs pa = {};
      pa.object = h->object;
      pa.quad = h->quad;
      pa.upd = gfield;
      pa.frames = frames;
      pa.corners = h->corners;
      pa.omax = h->omax;
      pa.partial = h->partial;
      pa.nslot = n;
      pa.chunk = chunk;
      pa.nxo = h->nxo;
      pa.K = h->K;
      pa.N = h->N;
      pa.mode = 1;
      dim3 grid((h->N * h->N + 255) / 256, nchunk);
      timed(h, kKProbePartial, [&] { probe_partial_kernel<<<grid, 256, 0, h->stream>>>(pa); }, pa.nslot);
      launched(h, "probe gradient");
      const int count = h->K * h->N * h->N;
      timed(h, kKProbeFinal, [&] {
        probe_finalize_kernel<<<(count + 255) / 256, 256, 0, h->stream>>>(
            h->partial, nchunk, count, nullptr, h->g_probe, h->g_probe_c, 1.f, 2);
      });
      launched(h, "probe gradient sum");
    }
    if (refine || pos_grad) {
      // the moved wave's derivatives from the probe spectra, dotted on chip with the
      // projection's change of the exit wave (refine) or with the gradient field g, whose
      // sums are ∂L/∂d (engine/features.rs:1055-1100)
      MoveArgs md = move_args(h, frames, nullptr);
      md.spec = h->spec;
      md.c = refine ? h->field : gfield;
      md.sums = h->ml_pos_sums;
      check(h, launch_move<kDerivSums>(h, md, n), "position sums");
      ++h->launches;
    }
  }
  if (up && h->have_offsets) {
    // num = conj(q)·IDFT(Σ_f spectra)
    MoveArgs mi = move_args(h, h->iota, h->g_probe);
    mi.spec = h->g_probe_spec;
    check(h, launch_move<kPlainInverse>(h, mi, 1), "probe gradient");
    ++h->launches;
  }
}

// num and den of the Poisson line search along (dir_obj, dir_probe), frames summed in order.
void ml_gamma(ptyb_handle* h, double* num, double* den) {
  const int stack = std::min(h->P, h->stack);
  if (h->have_offsets) spectrum_of(h, h->dir_probe, h->spec_d);
  GammaArgs a = {};
  a.object = h->object;
  a.d_obj = h->dir_obj;
  a.probe = h->probe;
  a.d_probe = h->dir_probe;
  a.quad = h->quad;
  a.tw = h->tw;
  a.iobs = h->iobs;
  a.corners = h->corners;
  a.nyo = h->nyo;
  a.nxo = h->nxo;
  a.nprobe = h->nprobe;
  a.nobj = h->nobj;
  for (int s0 = 0; s0 < h->P; s0 += stack) {
    const int n = std::min(stack, h->P - s0);
    a.frames = h->iota + s0;
    a.out = h->gamma_sums + (size_t)s0 * 2;
    a.psi = h->psi_all + (size_t)s0 * h->K * h->N * h->N;
    a.g = h->g_all + (size_t)s0 * h->K * h->N * h->N;
    if (h->have_offsets) {
      // the probe and its direction, each moved by the frame's offset (engine/ptycho.rs:527-534)
      move_frames(h, a.frames, n, h->spec_d, h->wave2);
      a.probe = h->wave_all + (size_t)s0 * h->K * h->N * h->N;
      a.d_probe = h->wave2;
      a.probe_stride = h->K * h->N * h->N;
    }
    check(h, launch_gamma(h, a, n), "ml line search");
    ++h->launches;
  }
  std::vector<double> v((size_t)h->P * 2);
  check(h, cudaMemcpyAsync(v.data(), h->gamma_sums, v.size() * sizeof(double),
                           cudaMemcpyDeviceToHost, h->stream),
        "gamma");
  check(h, cudaStreamSynchronize(h->stream), "gamma");
  *num = *den = 0.0;
  for (int f = 0; f < h->P; ++f) {
    *num += v[(size_t)f * 2];
    *den += v[(size_t)f * 2 + 1];
  }
}

// num and den of the Poisson line search along (dir_slices, dir_probe) through the slices
// (multislice.cuh `slice_gamma_kernel`), frames summed in order.
void slice_gamma(ptyb_handle* h, double* num, double* den) {
  const int stack = std::min(h->P, h->stack);
  SliceGammaArgs g = {};
  g.d_obj = h->dir_slices;
  g.d_probe = h->dir_probe;
  for (int s0 = 0; s0 < h->P; s0 += stack) {
    const int n = std::min(stack, h->P - s0);
    g.sa.f = frame_args(h, h->iota + s0);
    g.sa.f.nslot = n;
    g.sa.tf = h->tf;
    g.sa.nslice = h->nslice;
    g.sa.obj_plane = (size_t)h->nyo * h->nxo;
    g.out = h->gamma_sums + (size_t)s0 * 2;
    cudaError_t e = cudaSuccess;
    timed(h, kKGamma, [&] { e = launch_slice_gamma_side(h->N, g, n, h->K, h->stream); }, n);
    check(h, e, "multislice line search");
    ++h->launches;
  }
  std::vector<double> v((size_t)h->P * 2);
  check(h, copy_sync(h, v.data(), h->gamma_sums, v.size() * sizeof(double),
                     cudaMemcpyDeviceToHost),
        "gamma");
  *num = *den = 0.0;
  for (int f = 0; f < h->P; ++f) {
    *num += v[(size_t)f * 2];
    *den += v[(size_t)f * 2 + 1];
  }
}

// ML conjugate gradient through the slices (this build's definition; the reference runs ML
// on one slice): the opening rescale of the probe to the data's photons, per cycle the
// gradients through the slices (slice_gradients), the Polak–Ribière β over every slice and the
// probe, the line search on the second-order expansion (slice_gamma) and the step.
int ml_slices(ptyb_handle* h, const ptyb_ml_params* p, int32_t ncycle) {
  return guarded(h, true, [&]() -> int {
    const int S = h->nslice;
    ensure_slots(h, std::min(h->P, h->stack));
    ensure_ml(h);
    const size_t no = (size_t)S * h->nyo * h->nxo, np = (size_t)h->K * h->N * h->N;
    if (!h->last_slices) {
      h->last_slices = alloc<float2>(h, no);
      h->dir_slices = alloc<float2>(h, no);
    }
    const bool uo = p->update_object != 0, up = p->update_probe != 0;
    begin_call(h);
    // the probe rescaled so the model's photons are the data's
    const ptyb_llk l0 = llk_pass(h);
    const double fp = std::sqrt(h->obs_total / l0.nb_photons_calc);
    timed(h, kKAxpy, [&] {
      scale_kernel<<<blocks_for(np), 256, 0, h->stream>>>(h->probe, (float)fp, np);
    });
    launched(h, "scale");
    check(h, cudaMemsetAsync(h->dir_slices, 0, no * sizeof(float2), h->stream), "memset");
    check(h, cudaMemsetAsync(h->dir_probe, 0, np * sizeof(float2), h->stream), "memset");
    bool have_last = false;
    for (int ic = 0; ic < ncycle; ++ic) {
      const bool due = llk_due(p->calc_llk, ic, ncycle);
      ptyb_llk l = {};
      if (due) l = llk_pass(h);
      slice_gradients(h, uo, up);
      double beta = 0.0;
      if (have_last) {
        double a[2], b[2];
        array_sums(h, h->g_slices, h->last_slices, no, 0, a);
        array_sums(h, h->g_probe, h->last_probe, np, 0, b);
        beta = (a[0] + b[0]) / (a[1] + b[1]);
        if (!(std::isfinite(beta) && beta >= 0.0)) beta = 0.0;
      }
      timed(h, kKAxpy, [&] {
        cg_direction_kernel<<<blocks_for(no), 256, 0, h->stream>>>(h->dir_slices, h->g_slices,
                                                                   (float)beta, no);
      });
      launched(h, "direction");
      timed(h, kKAxpy, [&] {
        cg_direction_kernel<<<blocks_for(np), 256, 0, h->stream>>>(h->dir_probe, h->g_probe,
                                                                   (float)beta, np);
      });
      launched(h, "direction");
      double num = 0.0, den = 0.0;
      slice_gamma(h, &num, &den);
      const double gamma = num / den;
      if (std::isfinite(gamma)) {
        timed(h, kKAxpy, [&] {
          axpy_kernel<<<blocks_for(no), 256, 0, h->stream>>>(h->object, h->dir_slices,
                                                             (float)gamma, no);
        });
        launched(h, "step");
        timed(h, kKAxpy, [&] {
          axpy_kernel<<<blocks_for(np), 256, 0, h->stream>>>(h->probe, h->dir_probe,
                                                             (float)gamma, np);
        });
        launched(h, "step");
      } else {
        timed(h, kKAxpy, [&] {
          cg_direction_kernel<<<blocks_for(no), 256, 0, h->stream>>>(h->dir_slices,
                                                                     h->g_slices, 0.f, no);
        });
        launched(h, "direction");
        timed(h, kKAxpy, [&] {
          cg_direction_kernel<<<blocks_for(np), 256, 0, h->stream>>>(h->dir_probe, h->g_probe,
                                                                     0.f, np);
        });
        launched(h, "direction");
      }
      std::swap(h->g_slices, h->last_slices);
      std::swap(h->g_probe, h->last_probe);
      have_last = true;
      if (due) record(h, kAlgMl, l);
      ++h->cycle;
    }
    end_call(h, "ml");
    return PTYB_OK;
  });
}

// The Poisson sum and its gradients of the handle's state (ptyb_gradients): object and probe
// gradients handed to `sink(g_obj, g_probe, object elements, probe elements)` on the device,
// the position gradient to host d_pos.
template <typename Sink>
int gradients_to(ptyb_handle* h, double* loss, bool want_obj, bool want_probe, double* d_pos,
                 Sink&& sink) {
  if (!h) return PTYB_INVALID;
  if (h->nslice > 1 && (d_pos || h->have_offsets)) {
    h->err = "gradients through slices run without the position model";
    return PTYB_INVALID;
  }
  if (h->nslice > 1)
    return guarded(h, true, [&]() -> int {
      slice_gradients(h, want_obj, want_probe);
      const ptyb_llk l = llk_pass(h);
      if (loss) *loss = l.poisson * h->nb_obs;
      const size_t np = (size_t)h->K * h->N * h->N;
      const size_t no = (size_t)h->nslice * h->nyo * h->nxo;
      sink(h->g_slices, h->g_probe, no, np);
      return PTYB_OK;
    });
  if (d_pos && !h->have_offsets) {
    h->err = "position gradients need position offsets (ptyb_set_positions)";
    return PTYB_INVALID;
  }
  return guarded(h, true, [&]() -> int {
    ensure_slots(h, std::min(h->P, h->stack));
    ensure_ml(h);
    const size_t np = (size_t)h->K * h->N * h->N, no = (size_t)h->nyo * h->nxo;
    if (h->have_offsets) {
      ensure_spec(h);
      if (!h->wave_all) h->wave_all = alloc<float2>(h, (size_t)h->P * np);
      if (h->wave2_slots < h->slots) {
        h->wave2 = alloc<float2>(h, (size_t)h->slots * np);
        h->wave2_slots = h->slots;
      }
      if (!h->ml_pos_sums) h->ml_pos_sums = alloc<double>(h, (size_t)h->P * 4);
      spectrum_of(h, h->probe, h->spec);
      const int stack = std::min(h->P, h->stack);
      for (int s0 = 0; s0 < h->P; s0 += stack)
        move_frames(h, h->iota + s0, std::min(stack, h->P - s0), h->spec,
                    h->wave_all + (size_t)s0 * np);
    }
    ml_gradients(h, want_obj, want_probe, false, d_pos != nullptr);
    const ptyb_llk l = llk_pass(h, h->have_offsets ? h->wave_all : nullptr);
    if (loss) *loss = l.poisson * h->nb_obs;
    sink(h->g_obj, h->g_probe, no, np);
    if (d_pos) {
      std::vector<double> v((size_t)h->P * 4);
      check(h, copy_sync(h, v.data(), h->ml_pos_sums, v.size() * sizeof(double),
                          cudaMemcpyDeviceToHost),
            "gradient");
      for (int f = 0; f < h->P; ++f) {
        d_pos[2 * f] = v[(size_t)f * 4];
        d_pos[2 * f + 1] = v[(size_t)f * 4 + 1];
      }
    }
    return PTYB_OK;
  });
}

}  // namespace
}  // namespace ptyb::eng

using namespace ptyb::eng;

extern "C" {

int ptyb_ml(ptyb_handle* h, const ptyb_ml_params* p, int32_t ncycle) {
  if (!h || !p) return PTYB_INVALID;
  if (ncycle < 0) {
    h->err = "ncycle must be >= 0";
    return PTYB_INVALID;
  }
  if (h->nslice > 1) {
    if (h->have_offsets || p->zero_phase_ramp) {
      h->err = "ML through slices runs without the position model and phase-ramp removal";
      return PTYB_INVALID;
    }
    if (slice_gamma_bytes(h->N, h->K) > 227 * 1024) {
      h->err = "ML through slices: the frame's modes do not fit one cluster's shared memory";
      return PTYB_INVALID;
    }
    return ml_slices(h, p, ncycle);
  }
  return guarded(h, true, [&]() -> int {
    ensure_slots(h, std::min(h->P, h->stack));
    ensure_ml(h);
    const bool refine = h->have_offsets && h->refine_offsets;
    if (h->have_offsets && h->wave2_slots < h->slots) {
      h->wave2 = alloc<float2>(h, (size_t)h->slots * h->K * h->N * h->N);
      h->wave2_slots = h->slots;
    }
    if (refine && !h->ml_pos_sums) h->ml_pos_sums = alloc<double>(h, (size_t)h->P * 4);
    if (h->have_offsets) {
      ensure_spec(h);
      if (!h->wave_all) h->wave_all = alloc<float2>(h, (size_t)h->P * h->K * h->N * h->N);
    }
    const bool uo = p->update_object != 0, up = p->update_probe != 0;
    const size_t no = (size_t)h->nyo * h->nxo, np = (size_t)h->K * h->N * h->N;
    begin_call(h);
    auto move_all = [&] {
      // every frame's moved probe of the current probe, from its spectra
      spectrum_of(h, h->probe, h->spec);
      const int stack = std::min(h->P, h->stack);
      for (int s0 = 0; s0 < h->P; s0 += stack)
        move_frames(h, h->iota + s0, std::min(stack, h->P - s0), h->spec,
                    h->wave_all + (size_t)s0 * h->K * h->N * h->N);
    };
    if (h->have_offsets) move_all();
    // the opening rescale's LLK reads the moved probes, which it scales with the probe
    scale_obj_probe(h, h->have_offsets ? h->wave_all : nullptr);
    check(h, cudaMemsetAsync(h->dir_obj, 0, no * sizeof(float2), h->stream), "memset");
    check(h, cudaMemsetAsync(h->dir_probe, 0, np * sizeof(float2), h->stream), "memset");
    bool have_last = false;
    for (int ic = 0; ic < ncycle; ++ic) {
      const bool due = llk_due(p->calc_llk, ic, ncycle);
      if (h->have_offsets) {
        if (ic == 0)
          spectrum_of(h, h->probe, h->spec);  // the moved probes were scaled above
        else
          move_all();
      }
      ptyb_llk l = {};
      if (due) l = llk_pass(h, h->have_offsets ? h->wave_all : nullptr);
      ml_gradients(h, uo, up, refine);
      double beta = 0.0;
      if (have_last) {
        double a[2], b[2];
        array_sums(h, h->g_obj, h->last_obj, no, 0, a);
        array_sums(h, h->g_probe, h->last_probe, np, 0, b);
        beta = (a[0] + b[0]) / (a[1] + b[1]);
        if (!(std::isfinite(beta) && beta >= 0.0)) beta = 0.0;
      }
      timed(h, kKAxpy, [&] {
        cg_direction_kernel<<<blocks_for(no), 256, 0, h->stream>>>(h->dir_obj, h->g_obj, (float)beta, no);
      });
      launched(h, "direction");
      timed(h, kKAxpy, [&] {
        cg_direction_kernel<<<blocks_for(np), 256, 0, h->stream>>>(h->dir_probe, h->g_probe, (float)beta, np);
      });
      launched(h, "direction");
      double num = 0.0, den = 0.0;
      ml_gamma(h, &num, &den);
      const double gamma = num / den;
      if (std::isfinite(gamma)) {
        timed(h, kKAxpy, [&] {
          axpy_kernel<<<blocks_for(no), 256, 0, h->stream>>>(h->object, h->dir_obj, (float)gamma, no);
        });
        launched(h, "step");
        timed(h, kKAxpy, [&] {
          axpy_kernel<<<blocks_for(np), 256, 0, h->stream>>>(h->probe, h->dir_probe, (float)gamma, np);
        });
        launched(h, "step");
      } else {
        // No update; the direction restarts from the gradient.
        timed(h, kKAxpy, [&] {
          cg_direction_kernel<<<blocks_for(no), 256, 0, h->stream>>>(h->dir_obj, h->g_obj, 0.f, no);
        });
        launched(h, "direction");
        timed(h, kKAxpy, [&] {
          cg_direction_kernel<<<blocks_for(np), 256, 0, h->stream>>>(h->dir_probe, h->g_probe, 0.f, np);
        });
        launched(h, "direction");
      }
      std::swap(h->g_obj, h->last_obj);
      std::swap(h->g_probe, h->last_probe);
      have_last = true;
      if (refine) {
        timed(h, kKSolve, [&] {
          ml_position_step_kernel<<<1, 1024, 0, h->stream>>>(h->ml_pos_sums, h->P, h->offsets);
        });
        launched(h, "position step");
      }
      if (due) record(h, kAlgMl, l);
      ++h->cycle;
    }
    if (p->zero_phase_ramp) zero_phase_ramp(h);
    end_call(h, "ml");
    return PTYB_OK;
  });
}

int ptyb_gradients(ptyb_handle* h, double* loss, double* d_obj, double* d_probe, double* d_pos) {
  return gradients_to(h, loss, d_obj != nullptr, d_probe != nullptr, d_pos,
                      [&](const float2* g_obj, const float2* g_probe, size_t no, size_t np) {
                        if (d_obj) download_c64(h, g_obj, d_obj, no, "gradient");
                        if (d_probe) download_c64(h, g_probe, d_probe, np, "gradient");
                      });
}

int ptyb_gradients_device(ptyb_handle* h, double* loss, void* d_obj, void* d_probe,
                          double* d_pos) {
  if (!h) return PTYB_INVALID;
  if ((d_obj && !on_device(h, d_obj)) || (d_probe && !on_device(h, d_probe))) {
    h->err = "gradient outputs must be device memory of the handle's device";
    return PTYB_INVALID;
  }
  return gradients_to(h, loss, d_obj != nullptr, d_probe != nullptr, d_pos,
                      [&](const float2* g_obj, const float2* g_probe, size_t no, size_t np) {
                        if (d_obj)
                          check(h, copy_sync(h, d_obj, g_obj, no * sizeof(float2),
                                             cudaMemcpyDeviceToDevice),
                                "gradient");
                        if (d_probe)
                          check(h, copy_sync(h, d_probe, g_probe, np * sizeof(float2),
                                             cudaMemcpyDeviceToDevice),
                                "gradient");
                      });
}

}  // extern "C"
