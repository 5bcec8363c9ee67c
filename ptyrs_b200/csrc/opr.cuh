// pty-chi's orthogonal probe relaxation (OPR) of probe mode 0 inside LSQML (physwkim/ptyrs
// engine/opr.rs): every frame's own probe c_f·P_0 + Σ_i w_fi·U_i, and the step of the eigenmodes
// U_i, the weights w and the main mode's weights c from each batch's frame probe directions, in
// fixed-order sums (double) so every run gives the same bits.
#pragma once
#include "common.cuh"

namespace ptyb {

// out[slot][m] = c_f·P_0 + Σ_i w_fi·U_i for m = 0, P_m otherwise (engine/opr.rs:88-120).
static __global__ void opr_planes_kernel(const float2* probe, const float2* u, const double* w,
                                  const double* c, const int* frames, int K, int k, int plane,
                                  float2* out) {
  const int slot = blockIdx.y;
  const int f = frames[slot];
  for (int pix = blockIdx.x * blockDim.x + threadIdx.x; pix < plane;
       pix += gridDim.x * blockDim.x) {
    float2 v = probe[pix];
    if (c) v = cscale(v, (float)c[f]);
    for (int i = 0; i < k; ++i) v = cadd(v, cscale(u[(size_t)i * plane + pix], (float)w[(size_t)f * k + i]));
    out[(size_t)slot * K * plane + pix] = v;
    for (int m = 1; m < K; ++m)
      out[((size_t)slot * K + m) * plane + pix] = probe[(size_t)m * plane + pix];
  }
}

// vv[slot] = |O_window|² per pixel.
static __global__ void window_power_kernel(const float2* object, const int* frames, const int2* corners,
                                    int nxo, int N, float* vv) {
  const int slot = blockIdx.y;
  const int2 c = corners[frames[slot]];
  for (int pix = blockIdx.x * blockDim.x + threadIdx.x; pix < N * N;
       pix += gridDim.x * blockDim.x) {
    const int y = pix / N, x = pix % N;
    vv[(size_t)slot * N * N + pix] = cnorm2(object[(size_t)(c.x + y) * nxo + c.y + x]);
  }
}

// Per slot (one block each): s0 = Σ |a|²·vv, s1 + i·s2 = Σ conj(a)·x, over the plane;
// `a` a shared plane, `x` the slot's plane at x + slot·xstride.
static __global__ void __launch_bounds__(256) opr_frame_sums_kernel(const float2* a, const float2* x,
                                                             size_t xstride, const float* vv,
                                                             int plane, double* out) {
  __shared__ double red[3][8];
  const int slot = blockIdx.x;
  const float2* xs = x + (size_t)slot * xstride;
  const float* vs = vv ? vv + (size_t)slot * plane : nullptr;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int pix = threadIdx.x; pix < plane; pix += 256) {
    const float2 av = a[pix], xv = xs[pix];
    if (vs) s0 += (double)cnorm2(av) * vs[pix];
    s1 += (double)av.x * xv.x + (double)av.y * xv.y;
    s2 += (double)av.x * xv.y - (double)av.y * xv.x;
  }
  s0 = warp_sum(s0);
  s1 = warp_sum(s1);
  s2 = warp_sum(s2);
  if (threadIdx.x % 32 == 0) {
    red[0][threadIdx.x / 32] = s0;
    red[1][threadIdx.x / 32] = s1;
    red[2][threadIdx.x / 32] = s2;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += red[threadIdx.x][w];
    out[(size_t)slot * 3 + threadIdx.x] = t;
  }
}

// Σ |x|² over n elements, one block, fixed order.
static __global__ void __launch_bounds__(1024) opr_norm2_kernel(const float2* x, int n, double* out) {
  __shared__ double red[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += 1024) s += (double)cnorm2(x[i]);
  s = warp_sum(s);
  if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 32; ++w) t += red[w];
    *out = t;
  }
}

// The main mode's weights (engine/opr.rs:162-168): c_f += 0.1·Re<P_0, d_b> / Σ|P_0|²·vv_b.
static __global__ void opr_intensity_kernel(const double* sums, const int* frames, int count,
                                     double* c) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < count) c[frames[b]] += 0.1 * sums[b * 3 + 1] / sums[b * 3];
}

// The per-pixel sums over a batch's frames run in blocks of 32 pixels × 8 frame groups: group g
// takes frames [g·chunk, (g+1)·chunk) in order, and the 8 partials are added in group order (a
// fixed order, so every run gives the same bits).
constexpr int kOprGroups = 8;

// r_b = d_b − mean_b d_b.
static __global__ void __launch_bounds__(256) opr_residue_kernel(const float2* d, size_t dstride,
                                                          int count, int plane, float2* r) {
  __shared__ double part[2][kOprGroups][32];
  const int tx = threadIdx.x % 32, ty = threadIdx.x / 32;
  const int pix = blockIdx.x * 32 + tx;
  const int chunk = (count + kOprGroups - 1) / kOprGroups;
  const int b0 = ty * chunk, b1 = min(count, b0 + chunk);
  double mr = 0.0, mi = 0.0;
  if (pix < plane) {
#pragma unroll 4
    for (int b = b0; b < b1; ++b) {
      const float2 v = d[(size_t)b * dstride + pix];
      mr += v.x;
      mi += v.y;
    }
  }
  part[0][ty][tx] = mr;
  part[1][ty][tx] = mi;
  __syncthreads();
  mr = 0.0;
  mi = 0.0;
  for (int g = 0; g < kOprGroups; ++g) {
    mr += part[0][g][tx];
    mi += part[1][g][tx];
  }
  mr /= count;
  mi /= count;
  if (pix >= plane) return;
#pragma unroll 4
  for (int b = b0; b < b1; ++b) {
    const float2 v = d[(size_t)b * dstride + pix];
    r[(size_t)b * plane + pix] = make_float2((float)(v.x - mr), (float)(v.y - mi));
  }
}

// p_b = (Re<r_b, U>/n² + w_b) / Σ_b w_b², one block (engine/opr.rs:186-192).
// Σ_b x_b in frame order by one block of 256 threads: each chunk of 256 terms loaded by all
// threads at once, then added by thread 0 in order (the same bits as a serial loop).
template <class F>
__device__ double ordered_frame_sum(int count, F term) {
  __shared__ double chunk[256];
  double s = 0.0;
  for (int b0 = 0; b0 < count; b0 += 256) {
    const int n = min(256, count - b0);
    if ((int)threadIdx.x < n) chunk[threadIdx.x] = term(b0 + (int)threadIdx.x);
    __syncthreads();
    if (threadIdx.x == 0)
      for (int j = 0; j < n; ++j) s += chunk[j];
    __syncthreads();
  }
  return s;
}

static __global__ void __launch_bounds__(256) opr_coef_kernel(const double* sums, const double* w,
                                                       const int* frames, int k, int i,
                                                       int count, double n, double* p) {
  __shared__ double w2;
  const double s = ordered_frame_sum(count, [&](int b) {
    const double wb = w[(size_t)frames[b] * k + i];
    return wb * wb;
  });
  if (threadIdx.x == 0) w2 = s;
  __syncthreads();
  for (int b = threadIdx.x; b < count; b += blockDim.x)
    p[b] = (sums[b * 3 + 1] / (n * n) + w[(size_t)frames[b] * k + i]) / w2;
}

// e = Σ_b r_b·p_b / count, in the frame groups above.
static __global__ void __launch_bounds__(256) opr_e_kernel(const float2* r, const double* p, int count,
                                                    int plane, float2* e) {
  __shared__ double part[2][kOprGroups][32];
  const int tx = threadIdx.x % 32, ty = threadIdx.x / 32;
  const int pix = blockIdx.x * 32 + tx;
  const int chunk = (count + kOprGroups - 1) / kOprGroups;
  const int b0 = ty * chunk, b1 = min(count, b0 + chunk);
  double er = 0.0, ei = 0.0;
  if (pix < plane) {
#pragma unroll 4
    for (int b = b0; b < b1; ++b) {
      const float2 v = r[(size_t)b * plane + pix];
      er += v.x * p[b];
      ei += v.y * p[b];
    }
  }
  part[0][ty][tx] = er;
  part[1][ty][tx] = ei;
  __syncthreads();
  if (ty != 0 || pix >= plane) return;
  double sr = 0.0, si = 0.0;
  for (int g = 0; g < kOprGroups; ++g) {
    sr += part[0][g][tx];
    si += part[1][g][tx];
  }
  e[pix] = make_float2((float)(sr / count), (float)(si / count));
}

// u += (a_u·√n / mnorm(e))·e, mnorm(e) = √(Σ|e|²/n).
static __global__ void opr_u_step_kernel(float2* u, const float2* e, const double* ne, double a_u,
                                  int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double s = a_u * sqrt((double)n) / sqrt(*ne / n);
  u[i] = make_float2((float)(u[i].x + s * e[i].x), (float)(u[i].y + s * e[i].y));
}

// u *= √n / mnorm(u).
static __global__ void opr_u_scale_kernel(float2* u, const double* nu, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float s = (float)(sqrt((double)n) / sqrt(*nu / n));
  u[i] = cscale(u[i], s);
}

// w_fi = w_bi + Re<U, d_b> / (Σ|U|²·vv_b + 0.1·mean_b Σ|U|²·vv_b), one block
// (engine/opr.rs:200-212).
static __global__ void __launch_bounds__(256) opr_weights_kernel(const double* sums, const int* frames,
                                                          int count, int k, int i, double* w) {
  __shared__ double reg;
  const double s = ordered_frame_sum(count, [&](int b) { return sums[b * 3]; });
  if (threadIdx.x == 0) reg = 0.1 * s / count;
  __syncthreads();
  for (int b = threadIdx.x; b < count; b += blockDim.x) {
    double& wb = w[(size_t)frames[b] * k + i];
    wb = wb + sums[b * 3 + 1] / (sums[b * 3] + reg);
  }
}

// r_b −= (Σ r_b·conj(U) / Σ|U|²)·U (engine/opr.rs:213-219), thread per pixel, frame b =
// blockIdx.y.
static __global__ void opr_gs_kernel(float2* r, const float2* u, const double* sums, const double* uu,
                              int count, int plane) {
  const int pix = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (pix >= plane || b >= count) return;
  const float2 uv = u[pix];
  const double cr = sums[b * 3 + 1] / *uu, ci = sums[b * 3 + 2] / *uu;
  float2& v = r[(size_t)b * plane + pix];
  v = make_float2((float)(v.x - (cr * uv.x - ci * uv.y)), (float)(v.y - (cr * uv.y + ci * uv.x)));
}

}  // namespace ptyb
