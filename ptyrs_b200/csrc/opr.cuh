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

// Sums of up to four doubles over a block of 256 threads in a fixed order (the lanes' tree,
// then the eight warps in order); every thread gets the totals.
template <int M>
PTYB_D void block_sums256(double (&v)[M]) {
  __shared__ double red[M][8];
#pragma unroll
  for (int j = 0; j < M; ++j) v[j] = warp_sum(v[j]);
  __syncthreads();
  if (threadIdx.x % 32 == 0)
#pragma unroll
    for (int j = 0; j < M; ++j) red[j][threadIdx.x / 32] = v[j];
  __syncthreads();
#pragma unroll
  for (int j = 0; j < M; ++j) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += red[j][w];
    v[j] = t;
  }
}

// Whether this block is the grid's last to finish: each block's thread 0 has written its
// results, fences them and counts the block; the block that counts last sees every result and
// resets the counter for the next launch. Nothing waits, so no block depends on another's
// progress.
PTYB_D bool last_block(unsigned* counter) {
  __shared__ bool last;
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x * gridDim.y - 1;
    if (last) *counter = 0;
  }
  __syncthreads();
  if (last) __threadfence();
  return last;
}

// The per-frame sums run in kOprParts blocks per slot b (blockIdx.x = b, blockIdx.y = part),
// each over one contiguous span of the plane; the parts' partials are added in part order by
// the grid's last block, which also takes the batch-wide step.
constexpr int kOprParts = 4;

// The pixels of a block's span, in strides of 256, with their row and column carried along.
struct OprSpan {
  int pix, end, y, x;
  PTYB_D OprSpan(int plane, int N) {
    const int span = (plane + kOprParts - 1) / kOprParts;
    pix = (int)blockIdx.y * span + (int)threadIdx.x;
    end = min(plane, ((int)blockIdx.y + 1) * span);
    y = pix / N;
    x = pix % N;
  }
  PTYB_D void next(int N) {
    pix += 256;
    y += 256 / N;
    x += 256 % N;
    if (x >= N) {
      x -= N;
      ++y;
    }
  }
};

// A slot's total of sum m over its parts, in part order.
PTYB_D double opr_total(const double* part, int M, int b, int m) {
  double t = 0.0;
  for (int q = 0; q < kOprParts; ++q) t += __ldcg(part + ((size_t)b * kOprParts + q) * M + m);
  return t;
}

// The main mode's weights (engine/opr.rs:162-168): per slot b,
// c_f += 0.1·Re<P_0, d_b> / Σ|P_0|²·|O_b|², with |O_b|² taken from the frame's object window.
static __global__ void __launch_bounds__(256) opr_intensity_kernel(
    const float2* p0, const float2* d, size_t dstride, const float2* object, const int* frames,
    const int2* corners, int nxo, int N, unsigned* counter, double* part, double* c) {
  const int b = blockIdx.x, count = gridDim.x;
  const int2 cr = corners[frames[b]];
  const float2* db = d + (size_t)b * dstride;
  const float2* ob = object + (size_t)cr.x * nxo + cr.y;
  double s[2] = {0.0, 0.0};
#pragma unroll 4
  for (OprSpan it(N * N, N); it.pix < it.end; it.next(N)) {
    const float2 pv = p0[it.pix], dv = db[it.pix];
    s[0] += (double)cnorm2(pv) * cnorm2(ob[(size_t)it.y * nxo + it.x]);
    s[1] += (double)pv.x * dv.x + (double)pv.y * dv.y;
  }
  block_sums256(s);
  if (threadIdx.x == 0) {
    part[((size_t)b * kOprParts + blockIdx.y) * 2] = s[0];
    part[((size_t)b * kOprParts + blockIdx.y) * 2 + 1] = s[1];
  }
  if (!last_block(counter)) return;
  for (int j = threadIdx.x; j < count; j += 256)
    c[frames[j]] += 0.1 * opr_total(part, 2, j, 1) / opr_total(part, 2, j, 0);
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

// Per slot b for eigenmode U: with `prev` (the eigenmode before it) first the Gram–Schmidt
// step of the residues against that one, r_b −= (Σ r_b·conj(U') / Σ|U'|²)·U'
// (engine/opr.rs:213-219; `proj` [slot][2] the sums, `uu` Σ|U'|²), then Re Σ conj(U)·r_b; the
// last block turns these dots into the coefficients p_b = (Re<r_b, U>/n² + w_b) / Σ_b w_b²
// (engine/opr.rs:186-192), the sum over the batch in frame order.
static __global__ void __launch_bounds__(256) opr_dots_kernel(
    const float2* u, float2* r, int N, const float2* prev, const double* proj,
    const double* uu, const double* w, const int* frames, int k, int i, unsigned* counter,
    double* part, double* p) {
  const int b = blockIdx.x, count = gridDim.x, plane = N * N;
  float2* rb = r + (size_t)b * plane;
  double cr = 0.0, ci = 0.0;
  if (prev) {
    cr = proj[b * 2] / *uu;
    ci = proj[b * 2 + 1] / *uu;
  }
  double s[1] = {0.0};
#pragma unroll 4
  for (OprSpan it(plane, N); it.pix < it.end; it.next(N)) {
    float2 v = rb[it.pix];
    if (prev) {
      const float2 q = prev[it.pix];
      v = make_float2((float)(v.x - (cr * q.x - ci * q.y)), (float)(v.y - (cr * q.y + ci * q.x)));
      rb[it.pix] = v;
    }
    const float2 uv = u[it.pix];
    s[0] += (double)uv.x * v.x + (double)uv.y * v.y;
  }
  block_sums256(s);
  if (threadIdx.x == 0) part[(size_t)b * kOprParts + blockIdx.y] = s[0];
  if (!last_block(counter)) return;
  __shared__ double w2;
  const double t = ordered_frame_sum(count, [&](int j) {
    const double wj = w[(size_t)frames[j] * k + i];
    return wj * wj;
  });
  if (threadIdx.x == 0) w2 = t;
  __syncthreads();
  const double n2 = (double)plane * plane;
  for (int j = threadIdx.x; j < count; j += blockDim.x)
    p[j] = (opr_total(part, 1, j, 0) / n2 + w[(size_t)frames[j] * k + i]) / w2;
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

// Σ |x|² over n elements by one block of 1024 threads in a fixed order; every thread gets it.
PTYB_D double norm2_1024(const float2* x, int n) {
  __shared__ double red[32];
  __shared__ double total;
  double s = 0.0;
  for (int j = threadIdx.x; j < n; j += 1024) s += (double)cnorm2(x[j]);
  s = warp_sum(s);
  __syncthreads();
  if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 32; ++w) t += red[w];
    total = t;
  }
  __syncthreads();
  return total;
}

// The eigenmode's step, one block (engine/opr.rs:193-199): U += (a_u·√n / mnorm(e))·e, then
// U *= √n / mnorm(U), mnorm(x) = √(Σ|x|²/n); Σ|U|² of the result into *uu for the
// Gram–Schmidt step.
static __global__ void __launch_bounds__(1024) opr_u_kernel(float2* u, const float2* e,
                                                            double a_u, int n, double* uu) {
  const double ne = norm2_1024(e, n);
  const double s = a_u * sqrt((double)n) / sqrt(ne / n);
  for (int j = threadIdx.x; j < n; j += 1024)
    u[j] = make_float2((float)(u[j].x + s * e[j].x), (float)(u[j].y + s * e[j].y));
  __syncthreads();
  const double nu = norm2_1024(u, n);
  const float su = (float)(sqrt((double)n) / sqrt(nu / n));
  for (int j = threadIdx.x; j < n; j += 1024) u[j] = cscale(u[j], su);
  __syncthreads();
  const double t = norm2_1024(u, n);
  if (threadIdx.x == 0) *uu = t;
}

// Per slot b, after the eigenmode's step: with `d` the weights' sums s0 = Σ|U|²·|O_b|² and
// s1 = Re Σ conj(U)·d_b (|O_b|² from the frame's object window) and the last block's weight
// step w_fi += s1_b / (s0_b + 0.1·mean_b s0_b) (engine/opr.rs:200-212, the mean over the batch
// in frame order); with `r` the Gram–Schmidt sums Σ conj(U)·r_b into proj[b] for the next
// eigenmode's residues.
static __global__ void __launch_bounds__(256) opr_weight_proj_kernel(
    const float2* u, const float2* d, size_t dstride, const float2* r, const float2* object,
    const int* frames, const int2* corners, int nxo, int N, int k, int i, unsigned* counter,
    double* part, double* proj, double* w) {
  const int b = blockIdx.x, count = gridDim.x, plane = N * N;
  const int2 cr = corners[frames[b]];
  const float2* db = d ? d + (size_t)b * dstride : nullptr;
  const float2* rb = r ? r + (size_t)b * plane : nullptr;
  const float2* ob = object + (size_t)cr.x * nxo + cr.y;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 4
  for (OprSpan it(plane, N); it.pix < it.end; it.next(N)) {
    const float2 uv = u[it.pix];
    if (db) {
      const float2 dv = db[it.pix];
      s[0] += (double)cnorm2(uv) * cnorm2(ob[(size_t)it.y * nxo + it.x]);
      s[1] += (double)uv.x * dv.x + (double)uv.y * dv.y;
    }
    if (rb) {
      const float2 rv = rb[it.pix];
      s[2] += (double)uv.x * rv.x + (double)uv.y * rv.y;
      s[3] += (double)uv.x * rv.y - (double)uv.y * rv.x;
    }
  }
  block_sums256(s);
  if (threadIdx.x == 0)
#pragma unroll
    for (int m = 0; m < 4; ++m) part[((size_t)b * kOprParts + blockIdx.y) * 4 + m] = s[m];
  if (!last_block(counter)) return;
  if (r)
    for (int j = threadIdx.x; j < count; j += blockDim.x) {
      proj[j * 2] = opr_total(part, 4, j, 2);
      proj[j * 2 + 1] = opr_total(part, 4, j, 3);
    }
  if (!d) return;
  __shared__ double reg;
  const double t = ordered_frame_sum(count, [&](int j) { return opr_total(part, 4, j, 0); });
  if (threadIdx.x == 0) reg = 0.1 * t / count;
  __syncthreads();
  for (int j = threadIdx.x; j < count; j += blockDim.x) {
    double& wj = w[(size_t)frames[j] * k + i];
    wj = wj + opr_total(part, 4, j, 1) / (opr_total(part, 4, j, 0) + reg);
  }
}

}  // namespace ptyb
