// pty-chi's multislice exit wave and its adjoint on the device (physwkim/ptyrs
// engine/multislice.rs:87-173 forward, 266-286 back-propagation; gaps are angular spectrum,
// engine/propagate.rs:505-531), for LSQML with the Poisson or Gaussian cost.
//
// One cluster per frame holds the frame's K planes, as the frame kernel does. Forward: the
// probe times slice 0's window, then per gap an FFT pair with the transfer function between
// them and the next slice's window (the last also the exit phase q), each incident wave stored
// for the gathers; then the far-field FFT, the xi solver's first pass and the detector field.
// Backward: the field, the second xi pass, the residual, the inverse FFT and χ of the last
// slice, then per gap back through conj(q·O) and the conjugate transfer function.
#pragma once
#include "frame.cuh"

namespace ptyb {

struct SliceArgs {
  FrameArgs f;           // object = slice 0, probe, quad, counts, field, χ out (`out`) …
  const float2* tf;      // [nslice-1][N][N] transfer functions, unshifted DFT order
  float2* incident;      // [nslice-1][slot][K][N][N]: the waves entering slices 1.. (natural)
  float2* chi;           // [nslice][slot][K][N][N]: χ of every slice (natural)
  int nslice;
  size_t obj_plane;      // nyo·nxo: slice s's object at object + s·obj_plane
};

// kSliceGrad: forward (incident waves stored), the Poisson gradient 2(1 − I/Ĩ) of the exit
// wave (masked 0; with cost kCostBh BH's amplitude gradient 2(1 − √I/(√Ĩ + 1e-8))) and its
// back-propagation through the slices into `chi` (no subtraction): every slice's 2·∂L/∂ψ_s*,
// the adjoint of the multislice model.
enum SliceMode : int { kSliceForward = 0, kSliceBackward = 1, kSliceLlk = 2, kSliceGrad = 3 };

// Window of slice s times `v` for every plane's rows of this CTA (shifted layout); the last
// slice also takes q. `conj_mode` multiplies by conj(q·O) instead.
template <int N, int C>
PTYB_D void apply_window(float2* S, const SliceArgs& a, int s, int2 corner, int r, int K,
                         bool conj_mode) {
  using F = FrameShape<N, C>;
  constexpr int H = F::H, T = F::T, L = F::L;
  const bool last = s + 1 == a.nslice;
  const float2* obj = a.f.object + (size_t)s * a.obj_plane;
#pragma unroll 2
  for (int idx = threadIdx.x; idx < H * N; idx += T) {
    const int yl = idx / N, jx = idx % N;
    const int ny = (r * H + yl + N / 2) % N, nx = (jx + N / 2) % N;
    float2 w = obj[(size_t)(corner.x + ny) * a.f.nxo + corner.y + nx];
    if (last) w = cmul(w, a.f.quad[ny * N + nx]);
    if (conj_mode) w = cconj(w);
    for (int m = 0; m < K; ++m) {
      const int line = m * H + yl;
      float2& v = S[line * L + (jx ^ swz(line))];
      v = cmul(v, w);
    }
  }
  __syncthreads();
}

// The planes through gap s in place: FFT, × tf (or its conjugate) / N², inverse FFT.
template <int N, int C>
PTYB_D void through_gap(float2* S, const float2* tf, int K, bool adjoint, const LineTwiddles<N>& ltw,
                        cg::cluster_group& cluster, int r) {
  using F = FrameShape<N, C>;
  constexpr int H = F::H, T = F::T, L = F::L;
  constexpr float inv_n2 = 1.0f / ((float)N * (float)N);
  all_lines<N, C, -1>(S, K * H, ltw);
  transpose<N, C>(S, K, cluster);
  all_lines<N, C, -1>(S, K * H, ltw);
#pragma unroll 2
  for (int idx = threadIdx.x; idx < H * N; idx += T) {
    const int c = idx % H, ky = idx / H;
    float2 t = tf[ky * N + r * H + c];
    if (adjoint) t = cconj(t);
    t = cscale(t, inv_n2);
    for (int m = 0; m < K; ++m) {
      float2& v = S[(m * H + c) * L + (ky ^ swz(m * H + c))];
      v = cmul(v, t);
    }
  }
  __syncthreads();
  all_lines<N, C, +1>(S, K * H, ltw);
  transpose<N, C>(S, K, cluster);
  all_lines<N, C, +1>(S, K * H, ltw);
}

// This CTA's rows of every plane to `dst` ([K][N][N] natural layout), or loaded from it.
template <int N, int C>
PTYB_D void rows_io(float2* S, float2* dst, int r, int K, bool store) {
  using F = FrameShape<N, C>;
  constexpr int H = F::H, T = F::T, L = F::L;
#pragma unroll 2
  for (int idx = threadIdx.x; idx < H * N; idx += T) {
    const int yl = idx / N, jx = idx % N;
    const int ny = (r * H + yl + N / 2) % N, nx = (jx + N / 2) % N;
    for (int m = 0; m < K; ++m) {
      const int line = m * H + yl;
      float2& v = S[line * L + (jx ^ swz(line))];
      float2* g = dst + ((size_t)m * N + ny) * N + nx;
      if (store)
        *g = v;
      else
        v = *g;
    }
  }
  __syncthreads();
}

template <int N, int C, int MODE>
__global__ void __launch_bounds__(FrameShape<N, C>::T, frame_min_blocks<N, C>())
    slice_kernel(SliceArgs sa) {
  using F = FrameShape<N, C>;
  constexpr int H = F::H, T = F::T, L = F::L;
  const FrameArgs& a = sa.f;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int K = a.nprobe;
  float2* S = reinterpret_cast<float2*>(smem_raw);
  float2* twb = S + (size_t)K * H * L;
  double* red = reinterpret_cast<double*>(twb + N);
  cg::cluster_group cluster = cg::this_cluster();
  const int r = C > 1 ? (int)cluster.block_rank() : 0;
  const int slot = blockIdx.x / C;
  const int f = a.frames[slot];
  const int2 corner = a.corners[f];
  const int tid = threadIdx.x;
  LineTwiddles<N> ltw;
  ltw.load(a.tw, tid % F::G);
  const size_t frame_planes = (size_t)K * N * N;
  const size_t slice_stride = (size_t)a.nslot * frame_planes;  // one slice's [slot][K][N][N]
  constexpr float inv_n2 = 1.0f / ((float)N * (float)N);

  if (MODE != kSliceBackward) {
    // Slice 0's exit wave: probe (natural) times the window, in the shifted layout.
#pragma unroll 2
    for (int idx = tid; idx < H * N; idx += T) {
      const int yl = idx / N, jx = idx % N;
      const int ny = (r * H + yl + N / 2) % N, nx = (jx + N / 2) % N;
      for (int m = 0; m < K; ++m) {
        const int line = m * H + yl;
        S[line * L + (jx ^ swz(line))] =
            a.probe[(size_t)slot * a.probe_stride + ((size_t)m * N + ny) * N + nx];
      }
    }
    __syncthreads();
    apply_window<N, C>(S, sa, 0, corner, r, K, false);
    for (int s = 0; s + 1 < sa.nslice; ++s) {
      through_gap<N, C>(S, sa.tf + (size_t)s * N * N, K, false, ltw, cluster, r);
      if (MODE == kSliceForward || MODE == kSliceGrad)
        rows_io<N, C>(S, sa.incident + s * slice_stride + slot * frame_planes, r, K, true);
      apply_window<N, C>(S, sa, s + 1, corner, r, K, false);
    }
    all_lines<N, C, -1>(S, K * H, ltw);
    transpose<N, C>(S, K, cluster);
    all_lines<N, C, -1>(S, K * H, ltw);
  } else {
    const float2* src = a.field + ((size_t)slot * C + r) * K * H * N;
#pragma unroll 8
    for (int idx = tid; idx < K * H * N; idx += T) {
      const int line = idx / N, e = idx % N;
      S[line * L + (e ^ swz(line))] = src[idx];
    }
    __syncthreads();
  }

  // Detector plane (column strips): xi pass, LLK, projection, as the frame kernel.
  constexpr int kPix = H * N / T;
  const float* iobs = a.iobs + (size_t)f * N * N;
  float yo_r[kPix], ic_r[kPix];
#pragma unroll
  for (int i = 0; i < kPix; ++i) {
    const int idx = tid + i * T;
    const int c = idx % H, ky = idx / H;
    yo_r[i] = iobs[ky * N + r * H + c];
    float ic = 0.f;
    for (int m = 0; m < K; ++m) ic += cnorm2(S[(m * H + c) * L + (ky ^ swz(m * H + c))]);
    ic_r[i] = ic * inv_n2;
  }
  if (MODE == kSliceLlk) {
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < kPix; ++i) {
      const float yo = yo_r[i], ic = ic_r[i];
      if (yo < 0.f) continue;
      acc[0] += yo > 0.f ? (double)ic - yo + (double)yo * log((double)yo / ic) : (double)ic;
      const double dg = (double)yo - ic;
      acc[1] += dg * dg / ((double)yo + 1.0);
      const double de = sqrt((double)yo) - sqrt((double)ic);
      acc[2] += 4.0 * de * de;
      acc[3] += ic;
    }
    block_sum<T>(acc, 4, red);
    csync<C>(cluster);
    if (r == 0 && tid == 0) {
      for (int k = 0; k < 4; ++k) {
        double s = 0.0;
        for (int q = 0; q < C; ++q) s += (C > 1 ? cluster.map_shared_rank(red, q) : red)[k];
        a.llk[(size_t)slot * 4 + k] = s;
      }
    }
    csync<C>(cluster);
    return;
  }
  float afar = 0.5f;
  if (MODE != kSliceGrad && a.cost == kCostPoisson) {
    const double prev = MODE == kSliceForward
                            ? batch_mean(a.a_prev, a.frames, a.a_prev_by_frame, a.nslot, red + 7)
                            : batch_mean(a.a_mid, a.frames, 0, a.nslot, red + 7);
    double num = 0.0, den = 0.0;
#pragma unroll
    for (int i = 0; i < kPix; ++i) {
      const float yo = yo_r[i];
      if (yo < 0.f) continue;
      const double yp = (double)ic_r[i], yt = yo;
      const double xi = 1.0 - yt / (yp + 1e-5);
      num += xi * (yp - yt / (1.0 - prev * xi));
      den += xi * xi * yp;
    }
    cluster_sum2<N, C>(num, den, red, cluster);
    const double ratio = den > 0.0 ? num / den : 0.0;
    afar = (float)fmin(fmax(0.5 * prev + 0.5 * ratio, 0.0), 1.0);
    if (r == 0 && tid == 0) a.a_out[slot] = afar;
  } else if (MODE == kSliceBackward && r == 0 && tid == 0) {
    a.a_out[slot] = afar;
  }
  if (MODE == kSliceForward) {
    float2* dst = a.field + ((size_t)slot * C + r) * K * H * N;
#pragma unroll 8
    for (int idx = tid; idx < K * H * N; idx += T) {
      const int line = idx / N, e = idx % N;
      dst[idx] = S[line * L + (e ^ swz(line))];
    }
    return;
  }
#pragma unroll
  for (int i = 0; i < kPix; ++i) {
    const int idx = tid + i * T;
    const int c = idx % H, ky = idx / H;
    const float yo = yo_r[i], ic = ic_r[i];
    float fac;
    if (MODE == kSliceGrad) {
      // GradPoissonFourier (engine/ops.rs:161-195), or BH's (engine/bh.rs:168-275)
      fac = yo < 0.f                ? 0.f
            : a.cost == kCostBh     ? 2.f * (1.f - sqrtf(yo) / (sqrtf(ic) + 1e-8f))
                                    : 2.f * (1.f - yo / fmaxf(ic, 1e-12f));
      fac *= inv_n2;
    } else {
      float cres = 0.f;
      if (yo >= 0.f)
        cres = a.cost == kCostPoisson ? 1.f - yo / (ic + 1e-6f)
                                      : 2.f * (1.f - sqrtf(fmaxf(yo, 0.f)) / (sqrtf(ic) + 1e-9f));
      fac = (1.f - afar * cres) * inv_n2;
    }
    for (int m = 0; m < K; ++m) {
      float2& v = S[(m * H + c) * L + (ky ^ swz(m * H + c))];
      v = cscale(v, fac);
    }
  }
  __syncthreads();
  all_lines<N, C, +1>(S, K * H, ltw);
  transpose<N, C>(S, K, cluster);
  all_lines<N, C, +1>(S, K * H, ltw);
  // χ of the last slice: ψ' − q·O_last·in_last (the gradient: ψ' itself).
  const int last = sa.nslice - 1;
  const float2* in_last = last == 0 ? nullptr : sa.incident + (last - 1) * slice_stride + slot * frame_planes;
  const float2* obj_last = a.object + (size_t)last * sa.obj_plane;
#pragma unroll 2
  for (int idx = tid; idx < (MODE == kSliceGrad ? 0 : H * N); idx += T) {
    const int yl = idx / N, jx = idx % N;
    const int ny = (r * H + yl + N / 2) % N, nx = (jx + N / 2) % N;
    const float2 oq =
        cmul(obj_last[(size_t)(corner.x + ny) * a.nxo + corner.y + nx], a.quad[ny * N + nx]);
    for (int m = 0; m < K; ++m) {
      const int line = m * H + yl;
      const size_t pi = ((size_t)m * N + ny) * N + nx;
      const float2 in = in_last ? in_last[pi] : a.probe[(size_t)slot * a.probe_stride + pi];
      float2& v = S[line * L + (jx ^ swz(line))];
      v = csub(v, cmul(in, oq));
    }
  }
  __syncthreads();
  rows_io<N, C>(S, sa.chi + last * slice_stride + slot * frame_planes, r, K, true);
  for (int s = last - 1; s >= 0; --s) {
    apply_window<N, C>(S, sa, s + 1, corner, r, K, true);
    through_gap<N, C>(S, sa.tf + (size_t)s * N * N, K, true, ltw, cluster, r);
    rows_io<N, C>(S, sa.chi + s * slice_stride + slot * frame_planes, r, K, true);
  }
}

// Per slot, slice s ≥ 1's Eq. 23b sums (engine/lsqml.rs:327-347): with dop = q_s·dO_s·in_s,
// num = Σ Re(conj(dop)·χ_s), den = Σ |dop|² over modes and pixels; sums [slot][2] in double.
static __global__ void __launch_bounds__(512) slice_dots_kernel(const float2* d_obj,
                                                        const float2* incident,
                                                        const float2* quad, const float2* chi,
                                                        const int* frames, const int2* corners,
                                                        int nxo, int K, int N, double* sums) {
  __shared__ double sh[16];
  const int slot = blockIdx.x;
  const int2 c = corners[frames[slot]];
  const size_t plane = (size_t)N * N;
  float s0 = 0.f, s1 = 0.f;
  // mode, pixel, row and column carried along the 512-element strides (N² > 512 at every side)
  const int nn = N * N;
  int m = 0, pix = threadIdx.x, yy = pix / N, xx = pix - yy * N;
  for (int idx = threadIdx.x; idx < K * nn; idx += 512) {
    float2 u = cmul(incident[((size_t)slot * K + m) * plane + pix],
                    d_obj[(size_t)(c.x + yy) * nxo + c.y + xx]);
    if (quad) u = cmul(u, quad[pix]);
    const float2 x = chi[((size_t)slot * K + m) * plane + pix];
    s0 += u.x * x.x + u.y * x.y;
    s1 += cnorm2(u);
    pix += 512;
    xx += 512 % N;
    yy += 512 / N;
    if (xx >= N) {
      xx -= N;
      ++yy;
    }
    if (pix >= nn) {
      pix -= nn;
      yy -= N;
      ++m;
    }
  }
  auto bsum = [&](float v) {
    double d = warp_sum((double)v);
    if (threadIdx.x % 32 == 0) sh[threadIdx.x / 32] = d;
    __syncthreads();
    double t = 0.0;
    for (int w = 0; w < 16; ++w) t += sh[w];
    __syncthreads();
    return t;
  };
  const double num = bsum(s0), den = bsum(s1);
  if (threadIdx.x == 0) {
    sums[(size_t)slot * 2] = num;
    sums[(size_t)slot * 2 + 1] = den;
  }
}

// One block: a_obj_s = max(0.5·num/den·0.9/scale, 0) per frame, their trimmed mean into
// *step (engine/lsqml.rs:327-347, 392-398).
static __global__ void __launch_bounds__(1024) slice_solve_kernel(const double* sums, int nslot,
                                                           double scale, double* log,
                                                           int log_stride, float* step) {
  __shared__ double a[1024], sorted[1024];
  const int t = threadIdx.x;
  if (t < nslot) {
    const double num = sums[t * 2], den = sums[t * 2 + 1];
    a[t] = fmax(0.5 * num / den * 0.9 / scale, 0.0);
    log[(size_t)t * log_stride] = a[t];
  }
  __syncthreads();
  if (t < nslot) {
    int rank = 0;
    const double v = a[t];
    for (int j = 0; j < nslot; ++j) rank += (a[j] < v) || (a[j] == v && j < t);
    sorted[rank] = v;
  }
  __syncthreads();
  if (t == 0) {
    const int k = (int)ceil(nslot * 0.1 / 2.0 - 0.5);
    double s = 0.0;
    for (int i = k; i < nslot - k; ++i) s += sorted[i];
    *step = (float)(s / (nslot - 2 * k));
  }
}

// ML through the slices (this build's definition; the reference runs ML on one slice): the
// Poisson line search along the direction (dO_s, dP) on the second-order expansion of the
// exit waves, one frame per cluster. The wave entering slice s and its first and second Taylor
// coefficients along the direction, w, w′, w″ (w_0 = P, w′_0 = dP, w″_0 = 0), go through the
// slices together: w″ ← O_s·w″ + dO_s·w′, w′ ← O_s·w′ + dO_s·w, w ← O_s·w, then the gap (the
// last slice with the exit phase q, then the far-field transform). With po, a, b the three
// detector fields, per unmasked pixel calc = Σ_m |po|², r = Σ_m Re(p̄o·a),
// s = Σ_m |a|² + 2·Re(p̄o·b), d = 1 − I/max(calc, 1e-32): num = −Σ 2·r·d,
// den = Σ 2·s·d + I·(2r/calc)² (PyNX CG_Poisson_Gamma, engine/ops.rs:206-253). Shared memory
// holds the three sets of K planes.
// With `bh` the kernel takes BH's quadratic form Q(w) = H(w, w) of the amplitude cost along
// the displacement instead (engine/bh.rs:500-575): per unmasked pixel with A = √Σ_m |po|² +
// 1e-8, d = √I and c = Σ_m Re(p̄o·a): 4·(1 − d/A)·Σ_m Re(p̄o·b) + 2·(1 − d/A)·Σ_m |a|² +
// 2·d·c²/A³ (U J″(w, w) = 2·b), into out[slot][0].
struct SliceGammaArgs {
  SliceArgs sa;
  const float2* d_obj;    // [nslice][nyo][nxo]
  const float2* d_probe;  // [K][N][N]
  double* out;            // [slot][2]: num, den
  int bh;
};

template <int N, int C>
__host__ __device__ constexpr size_t slice_gamma_smem_bytes(int K) {
  return 3 * frame_smem_bytes<N, C>(K) - 2 * (N * sizeof(float2) + 160 * sizeof(double));
}

template <int N, int C>
__global__ void __launch_bounds__(FrameShape<N, C>::T, 1) slice_gamma_kernel(SliceGammaArgs g) {
  using F = FrameShape<N, C>;
  constexpr int H = F::H, T = F::T, L = F::L;
  const SliceArgs& sa = g.sa;
  const FrameArgs& a = sa.f;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int K = a.nprobe;
  float2* S = reinterpret_cast<float2*>(smem_raw);  // lines: w (K·H), w′ (K·H), w″ (K·H)
  double* red = reinterpret_cast<double*>(S + 3 * (size_t)K * H * L + N);
  cg::cluster_group cluster = cg::this_cluster();
  const int r = C > 1 ? (int)cluster.block_rank() : 0;
  const int slot = blockIdx.x / C;
  const int f = a.frames[slot];
  const int2 corner = a.corners[f];
  const int tid = threadIdx.x;
  LineTwiddles<N> ltw;
  ltw.load(a.tw, tid % F::G);
  auto at = [&](int set, int m, int yl, int jx) -> float2& {
    const int line = (set * K + m) * H + yl;
    return S[line * L + (jx ^ swz(line))];
  };
#pragma unroll 2
  for (int idx = tid; idx < H * N; idx += T) {
    const int yl = idx / N, jx = idx % N;
    const int ny = (r * H + yl + N / 2) % N, nx = (jx + N / 2) % N;
    for (int m = 0; m < K; ++m) {
      const size_t pi = ((size_t)m * N + ny) * N + nx;
      at(0, m, yl, jx) = a.probe[pi];
      at(1, m, yl, jx) = g.d_probe[pi];
      at(2, m, yl, jx) = make_float2(0.f, 0.f);
    }
  }
  __syncthreads();
  for (int s = 0; s < sa.nslice; ++s) {
    const bool last = s + 1 == sa.nslice;
    const float2* obj = a.object + (size_t)s * sa.obj_plane;
    const float2* dob = g.d_obj + (size_t)s * sa.obj_plane;
#pragma unroll 2
    for (int idx = tid; idx < H * N; idx += T) {
      const int yl = idx / N, jx = idx % N;
      const int ny = (r * H + yl + N / 2) % N, nx = (jx + N / 2) % N;
      const size_t oi = (size_t)(corner.x + ny) * a.nxo + corner.y + nx;
      float2 o = obj[oi], d = dob[oi];
      if (last) {
        const float2 q = a.quad[ny * N + nx];
        o = cmul(o, q);
        d = cmul(d, q);
      }
      for (int m = 0; m < K; ++m) {
        float2 &w = at(0, m, yl, jx), &w1 = at(1, m, yl, jx), &w2 = at(2, m, yl, jx);
        w2 = cadd(cmul(o, w2), cmul(d, w1));
        w1 = cadd(cmul(o, w1), cmul(d, w));
        w = cmul(o, w);
      }
    }
    __syncthreads();
    if (!last) through_gap<N, C>(S, sa.tf + (size_t)s * N * N, 3 * K, false, ltw, cluster, r);
  }
  all_lines<N, C, -1>(S, 3 * K * H, ltw);
  transpose<N, C>(S, 3 * K, cluster);
  all_lines<N, C, -1>(S, 3 * K * H, ltw);
  // Columns kx = r·H + c (lines set·K·H + m·H + c), elements ky.
  constexpr float inv_n2 = 1.0f / ((float)N * (float)N);
  const float* iobs = a.iobs + (size_t)f * N * N;
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  for (int idx = tid; idx < H * N; idx += T) {
    const int c = idx % H, ky = idx / H;
    const float yo = iobs[ky * N + r * H + c];
    if (yo < 0.f) continue;
    double calc = 0.0, rr = 0.0, ss = 0.0, pb = 0.0, aa = 0.0;
    for (int m = 0; m < K; ++m) {
      const int l0 = m * H + c, l1 = (K + m) * H + c, l2 = (2 * K + m) * H + c;
      const float2 po = S[l0 * L + (ky ^ swz(l0))], av = S[l1 * L + (ky ^ swz(l1))],
                   bv = S[l2 * L + (ky ^ swz(l2))];
      calc += (double)cnorm2(po) * inv_n2;
      rr += ((double)po.x * av.x + (double)po.y * av.y) * inv_n2;
      pb += ((double)po.x * bv.x + (double)po.y * bv.y) * inv_n2;
      aa += (double)cnorm2(av) * inv_n2;
    }
    if (g.bh) {
      const double amp = sqrt(calc) + 1e-8, d = sqrt((double)yo), w = 1.0 - d / amp;
      v[0] += 4.0 * w * pb + 2.0 * w * aa + 2.0 * d * rr * rr / (amp * amp * amp);
      continue;
    }
    ss = aa + 2.0 * pb;
    calc = fmax(calc, 1e-32);
    const double d = 1.0 - (double)yo / calc;
    v[0] -= 2.0 * rr * d;
    const double t = 2.0 * rr / calc;
    v[1] += 2.0 * ss * d + (double)yo * t * t;
  }
  block_sum<T>(v, 2, red);
  csync<C>(cluster);
  if (r == 0 && tid == 0) {
    double num = 0.0, den = 0.0;
    for (int q = 0; q < C; ++q) {
      const double* rq = C > 1 ? cluster.map_shared_rank(red, q) : red;
      num += rq[0];
      den += rq[1];
    }
    g.out[slot * 2] = num;
    g.out[slot * 2 + 1] = den;
  }
  csync<C>(cluster);
}

}  // namespace ptyb
