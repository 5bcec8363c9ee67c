// LSQML's batch reductions: the Poisson far-field step, the per-frame 2×2 step-size systems
// (solved in double), the trimmed mean and the update (physwkim/ptyrs engine/lsqml.rs:102-179,
// 286-350, 392-398, 581-643).
#pragma once
#include "common.cuh"

namespace ptyb {

// Block sum in double of one value per thread (T = 256), result in every thread.
template <int T>
PTYB_D double block_sum1(double v, double* sh) {
  v = warp_sum(v);
  if (threadIdx.x % 32 == 0) sh[threadIdx.x / 32] = v;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < T / 32; ++w) s += sh[w];
  __syncthreads();
  return s;
}

// Per slot, the six sums of the step-size system over its modes and pixels (natural layout):
// u = P·dO·q (dop), v = dP·O·q (dpo), c = χ: Σ|u|²+λ0, Σ|v|²+λ0, Σ Re u·v̄, Σ Im u·v̄,
// Σ Re ū·c, Σ Re v̄·c (engine/lsqml.rs:302-323). Each thread sums its pixels in float, the
// block adds the threads' sums in double; λ0 joins once per pixel and mode.
constexpr int kDotParts = 4;  // blocks per frame; their sums are added in block order

static __global__ void __launch_bounds__(512) lsqml_dots_kernel(
    const float2* object, const float2* d_obj, const float2* probe, const float2* d_probe,
    const float2* quad, const float2* chi, const int* frames, const int2* corners, int nxo,
    int K, int N, double lambda0, double* sums, int probe_stride) {
  __shared__ double sh[16];
  const int slot = blockIdx.x / kDotParts, part = blockIdx.x % kDotParts;
  const int2 c = corners[frames[slot]];
  const size_t plane = (size_t)N * N;
  const int span = (K * N * N + kDotParts - 1) / kDotParts;
  const int i0 = part * span, i1 = min(K * N * N, i0 + span);
  float s[6] = {0, 0, 0, 0, 0, 0};
  // mode, pixel, row and column of idx carried along the 512-element strides (no division per
  // element; N² > 512 at every side)
  const int nn = N * N;
  int m = (i0 + (int)threadIdx.x) / nn, pix = (i0 + (int)threadIdx.x) - m * nn;
  int yy = pix / N, xx = pix - yy * N;
#pragma unroll 4
  for (int idx = i0 + threadIdx.x; idx < i1; idx += 512) {
    const size_t o = (size_t)(c.x + yy) * nxo + c.y + xx;
    const float2 q = quad[pix];
    const float2 u = cmul(cmul(probe[(size_t)slot * probe_stride + m * plane + pix], d_obj[o]), q);
    const float2 v = cmul(cmul(d_probe[m * plane + pix], object[o]), q);
    const float2 x = chi[((size_t)slot * K + m) * plane + pix];
    s[0] += cnorm2(u);
    s[1] += cnorm2(v);
    s[2] += u.x * v.x + u.y * v.y;
    s[3] += u.y * v.x - u.x * v.y;
    s[4] += u.x * x.x + u.y * x.y;
    s[5] += v.x * x.x + v.y * x.y;
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
  const double reg = part == 0 ? lambda0 * (double)K * (double)plane : 0.0;
  for (int k = 0; k < 6; ++k) {
    const double t = block_sum1<512>((double)s[k], sh);
    if (threadIdx.x == 0) sums[((size_t)slot * kDotParts + part) * 6 + k] = t + (k < 2 ? reg : 0.0);
  }
}

// One block: the per-frame 2×2 solves in double, trimmed mean of a_obj, mean of a_probe;
// scal[0] = object step, scal[1] = probe step. Records a_far / a_obj / a_probe per slot in
// `log` ([slot][3]) and the frames' a_far in `a_far_all`.
static __global__ void __launch_bounds__(1024) lsqml_solve_kernel(const double* sums, int nslot,
                                                           double scale, const float* a_far,
                                                           const int* frames, float* a_far_all,
                                                           double* log, float* scal,
                                                           int log_stride) {
  __shared__ double aobj[1024], aprb[1024], sorted[1024];
  __shared__ double frame_sums[1024][2];
  __shared__ double means[2];
  const int t = threadIdx.x;
  double s[6] = {0, 0, 0, 0, 0, 0};
  if (t < nslot) {
    for (int p = 0; p < kDotParts; ++p)
      for (int k = 0; k < 6; ++k) s[k] += sums[((size_t)t * kDotParts + p) * 6 + k];
    frame_sums[t][0] = s[0];
    frame_sums[t][1] = s[1];
  }
  __syncthreads();
  if (t == 0) {
    double m0 = 0.0, m1 = 0.0;
    for (int i = 0; i < nslot; ++i) {
      m0 += frame_sums[i][0];
      m1 += frame_sums[i][1];
    }
    means[0] = 0.1 * (m0 / nslot);
    means[1] = 0.1 * (m1 / nslot);
  }
  __syncthreads();
  if (t < nslot) {
    const double a11 = s[0] + means[0], a22 = s[1] + means[1];
    const double det = a11 * a22 - (s[2] * s[2] + s[3] * s[3]);
    const double x0 = (a22 * s[4] - s[2] * s[5]) / det;
    const double x1 = (a11 * s[5] - s[2] * s[4]) / det;
    aobj[t] = 0.9 * fmax(x0, 0.0) / scale;
    aprb[t] = 0.9 * fmax(x1, 0.0);
    a_far_all[frames[t]] = a_far[t];
    log[t * log_stride + 0] = a_far[t];
    log[t * log_stride + 1] = aobj[t];
    log[t * log_stride + 2] = aprb[t];
  }
  __syncthreads();
  if (t < nslot) {
    int rank = 0;
    const double v = aobj[t];
    for (int j = 0; j < nslot; ++j) rank += (aobj[j] < v) || (aobj[j] == v && j < t);
    sorted[rank] = v;
  }
  __syncthreads();
  if (t == 0) {
    const int k = (int)ceil(nslot * 0.1 / 2.0 - 0.5);
    double s = 0.0;
    for (int i = k; i < nslot - k; ++i) s += sorted[i];
    double p = 0.0;
    for (int i = 0; i < nslot; ++i) p += aprb[i];
    scal[0] = (float)(s / (nslot - 2 * k));
    scal[1] = (float)(p / nslot);
  }
}

// x += scal[which]·d over n values.
static __global__ void axpy_scal_kernel(float2* x, const float2* d, const float* scal, int which,
                                 size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  x[i] = cadd(x[i], cscale(d[i], scal[which]));
}

// Max of a non-negative float array into *out (which starts at 0).
static __global__ void max_kernel(const float* v, size_t n, float* out) {
  float m = 0.f;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    m = fmaxf(m, v[i]);
  m = warp_max(m);
  if (threadIdx.x % 32 == 0) atomic_max_nonneg(out, m);
}

}  // namespace ptyb
