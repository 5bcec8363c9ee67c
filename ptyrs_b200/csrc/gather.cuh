// Deterministic scatter-adds of the per-view updates onto the object and the probe.
//
// Object: one CTA owns a 16×16 object tile and lists the launch's views that overlap it in
// ascending slot order (the reference's view order); four thread groups per pixel take every
// fourth view of that list, each with Kahan-compensated float sums, and the groups' sums are
// added in group order. No atomics touch the object and the result does not depend on
// scheduling (the reference's tile-owned gather, ptyrs-kernels/src/lib.rs:388-437; operator
// engine/ops.rs:282-310). Probe: the slots are cut
// into chunks, each CTA sums one chunk in slot order for 256 probe pixels, and a second pass
// adds the chunk sums in chunk order (engine/ops.rs:315-345).
#pragma once
#include "common.cuh"

namespace ptyb {

constexpr int kTile = 16;      // object tile side
constexpr int kGroups = 4;     // view groups per pixel
constexpr int kMaxModes = 4;

enum GatherMode : int {
  kGatherRpie = 0,   // O += step·Σ_m num_m / ((1−α)·D_m + α·pmax)
  kGatherLsqml = 1,  // d_obj = Σ conj(q·P)·χ / √(pre² + floor²)
  kGatherMl = 2,     // grad += Σ conj(q·P)·g (compensated across launches)
  kGatherOverlap = 3,  // pmax = max over pixels of Σ_m D_m
  kGatherIllum = 4,    // pre = (pre + I)/2 with I = Σ|P|² over every view
  kGatherBlend = 5,    // the object blend's sums: out = num, pre = norm, pmax = max norm
};

struct GatherArgs {
  float2* object;          // [nyo][nxo] object mode 0 (rPIE updates it)
  const float2* probe;     // [nprobe][N][N]
  const float2* quad;      // [N][N]
  const float2* upd;       // [slot][K][N][N] natural: Δ, χ or g
  const int* frames;       // [nslot]
  const int2* corners;     // [nframe]
  float* pmax;             // rPIE overlap max (device scalar)
  float* pre;              // LSQML preconditioner [nyo][nxo]
  const float* pre_max;    // LSQML: max of pre (device scalar)
  float2* out;             // LSQML d_obj / ML gradient sum [nyo][nxo]
  float2* comp;            // ML gradient compensation [nyo][nxo]
  float alpha, step, pre_scale;
  int nslot, nyo, nxo, nprobe, N;
  int probe_stride;        // elements between slots' probes (0: the shared probe)
};

// The launch's slots in [s0, s1) (at most 1024) whose window overlaps the tile
// [ty0, ty0+16) × [tx0, tx0+16), in ascending order with their corners: an ordered
// compaction by all 1024 threads (warp ballots, then a prefix over the warps).
PTYB_D int tile_list(const GatherArgs& a, int s0, int s1, int ty0, int tx0, int* list,
                     int2* corner) {
  __shared__ int wbase[32];
  __shared__ int total;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int s = s0 + t;
  bool hit = false;
  int2 c = make_int2(0, 0);
  if (s < s1) {
    c = a.corners[a.frames[s]];
    hit = c.x < ty0 + kTile && c.x + a.N > ty0 && c.y < tx0 + kTile && c.y + a.N > tx0;
  }
  const unsigned m = __ballot_sync(0xffffffffu, hit);
  if (lane == 0) wbase[w] = __popc(m);
  __syncthreads();
  if (w == 0) {
    const int v = wbase[lane];
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += u;
    }
    wbase[lane] = incl - v;
    if (lane == 31) total = incl;
  }
  __syncthreads();
  if (hit) {
    const int pos = wbase[w] + __popc(m & ((1u << lane) - 1u));
    list[pos] = s;
    corner[pos] = c;
  }
  __syncthreads();
  const int n = total;
  __syncthreads();
  return n;
}

template <int MODE>
__global__ void __launch_bounds__(1024, MODE == kGatherRpie || MODE == kGatherBlend ? 1 : 2) object_tile_kernel(GatherArgs a) {
  constexpr int kChunk = 1024;
  constexpr int kPix = kTile * kTile;  // 256 pixels, kGroups threads each
  // The view list (during the walk), then the groups' partial sums (after it).
  constexpr int kListBytes = kChunk * (sizeof(int) + sizeof(int2));
  constexpr int kNumBytes = (kGroups - 1) * kMaxModes * kPix * sizeof(float2);
  constexpr int kDenBytes = (kGroups - 1) * kMaxModes * kPix * sizeof(float);
  constexpr int kPartBytes = kNumBytes + kDenBytes + (kGroups - 1) * kPix * sizeof(int);
  __shared__ __align__(16) unsigned char sm[kListBytes > kPartBytes ? kListBytes : kPartBytes];
  __shared__ float red[32];
  int* list = reinterpret_cast<int*>(sm);
  int2* lcorner = reinterpret_cast<int2*>(sm + kChunk * sizeof(int));
  float2(*part_num)[kMaxModes][kPix] = reinterpret_cast<float2(*)[kMaxModes][kPix]>(sm);
  float(*part_den)[kMaxModes][kPix] = reinterpret_cast<float(*)[kMaxModes][kPix]>(sm + kNumBytes);
  int(*part_cov)[kPix] = reinterpret_cast<int(*)[kPix]>(sm + kNumBytes + kDenBytes);
  const int tiles_x = (a.nxo + kTile - 1) / kTile;
  const int tx0 = (blockIdx.x % tiles_x) * kTile, ty0 = (blockIdx.x / tiles_x) * kTile;
  const int px = threadIdx.x % kPix, grp = threadIdx.x / kPix;
  const int x = tx0 + px % kTile, y = ty0 + px / kTile;
  const bool inside = x < a.nxo && y < a.nyo;
  const int K = a.nprobe;
  const int N = a.N;
  const size_t plane = (size_t)N * N;
  KahanC num[kMaxModes];
  Kahan den[kMaxModes];
#pragma unroll
  for (int m = 0; m < kMaxModes; ++m) {
    num[m].init();
    den[m].init();
  }
  bool covered = false, any = false;
  for (int s0 = 0; s0 < a.nslot; s0 += kChunk) {
    const int s1 = min(a.nslot, s0 + kChunk);
    const int n = tile_list(a, s0, s1, ty0, tx0, list, lcorner);
    any |= n > 0;
#pragma unroll 2
    for (int i = grp; i < n; i += kGroups) {
      const int s = list[i];
      const int2 c = lcorner[i];
      const int yy = y - c.x, xx = x - c.y;
      if (!inside || yy < 0 || yy >= N || xx < 0 || xx >= N) continue;
      covered = true;
      const int pix = yy * N + xx;
      const float2 q = a.quad[pix];
      float2 u[kMaxModes];
#pragma unroll
      for (int m = 0; m < kMaxModes; ++m)
        if (m < K && (MODE == kGatherRpie || MODE == kGatherLsqml || MODE == kGatherMl ||
                      MODE == kGatherBlend))
          u[m] = a.upd[((size_t)s * K + m) * plane + pix];
#pragma unroll
      for (int m = 0; m < kMaxModes; ++m) {
        if (m >= K) break;
        const float2 p = a.probe[(size_t)s * a.probe_stride + m * plane + pix];
        if (MODE == kGatherOverlap || MODE == kGatherIllum || MODE == kGatherRpie ||
            MODE == kGatherBlend)
          den[m].add(cnorm2(p));
        if (MODE == kGatherRpie || MODE == kGatherLsqml || MODE == kGatherMl ||
            MODE == kGatherBlend) {
          const float2 t = cmulc(cmul(p, q), u[m]);  // conj(P·q)·u
          if (MODE == kGatherRpie)
            num[m].add(t);
          else
            num[0].add(t);
        }
      }
    }
  }
  // Groups 1..3 hand their compensated sums to group 0, which adds them in group order.
  __syncthreads();  // the list's space becomes the partial sums'
  if (grp > 0) {
#pragma unroll
    for (int m = 0; m < kMaxModes; ++m) {
      part_num[grp - 1][m][px] = make_float2(num[m].re.s - num[m].re.c, num[m].im.s - num[m].im.c);
      part_den[grp - 1][m][px] = den[m].s - den[m].c;
    }
    part_cov[grp - 1][px] = covered;
  }
  __syncthreads();
  if (grp == 0) {
#pragma unroll
    for (int g = 0; g < kGroups - 1; ++g) {
#pragma unroll
      for (int m = 0; m < kMaxModes; ++m) {
        num[m].add(part_num[g][m][px]);
        den[m].add(part_den[g][m][px]);
      }
      covered |= part_cov[g][px] != 0;
    }
  }
  const size_t o = (size_t)y * a.nxo + x;
  if (MODE == kGatherOverlap || MODE == kGatherBlend) {
    float d = 0.f;
#pragma unroll
    for (int m = 0; m < kMaxModes; ++m)
      if (m < K) d += den[m].s;
    if (MODE == kGatherBlend && inside && grp == 0) {
      // psi_to_obj_probe's object sums (engine/ops.rs:352-369), every pixel, covered or not
      a.out[o] = num[0].value();
      a.pre[o] = d;
    }
    d = warp_max(inside && grp == 0 ? d : 0.f);
    if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = d;
    __syncthreads();
    if (threadIdx.x == 0) {
      float mx = 0.f;
      for (int w = 0; w < 32; ++w) mx = fmaxf(mx, red[w]);
      atomic_max_nonneg(a.pmax, mx);
    }
    return;
  }
  if (!inside || grp != 0) return;
  if (MODE == kGatherRpie) {
    if (!covered) return;
    const float pmax = *a.pmax;
    float2 d = make_float2(0.f, 0.f);
#pragma unroll
    for (int m = 0; m < kMaxModes; ++m) {
      if (m >= K) break;
      const float w = (1.f - a.alpha) * den[m].s + a.alpha * pmax;
      d = cadd(d, cscale(num[m].value(), 1.f / w));
    }
    a.object[o] = cadd(a.object[o], cscale(d, a.step));
  } else if (MODE == kGatherLsqml) {
    const float p = a.pre[o];
    const float fl = 0.1f * (*a.pre_max);
    a.out[o] = cscale(num[0].value(), rsqrtf(p * p + fl * fl));
  } else if (MODE == kGatherMl) {
    if (!any) return;
    // out += num with the running compensation in comp.
    const float2 v = num[0].value();
    float2 g = a.out[o], cc = a.comp[o];
    const float yr = v.x - cc.x, yi = v.y - cc.y;
    const float tr = g.x + yr, ti = g.y + yi;
    cc = make_float2((tr - g.x) - yr, (ti - g.y) - yi);
    a.out[o] = make_float2(tr, ti);
    a.comp[o] = cc;
  } else if (MODE == kGatherIllum) {
    float d = 0.f;
#pragma unroll
    for (int m = 0; m < kMaxModes; ++m)
      if (m < K) d += den[m].s;
    // pty-chi's schedule: (pre + I)/2, the first from pre = I·pre_scale.
    a.pre[o] = a.pre_scale >= 0.f ? 0.5f * (d * a.pre_scale + d) : 0.5f * (a.pre[o] + d);
  }
}

struct ProbeArgs {
  const float2* object;   // [nyo][nxo] object mode 0
  const float2* quad;     // [N][N]
  const float2* upd;      // [slot][K][N][N]
  const int* frames;
  const int2* corners;
  const float* omax;      // rPIE [slot]
  float2* partial;        // [nchunk][K][N][N]
  float* partial_den;     // mode 2: [nchunk][N][N] Σ_slots |O|² over the window
  float alpha;
  // mode 0 rPIE weight, 1 plain conj(q·O), 2 also Σ|O|², 3 Σ|O|² alone
  int nslot, chunk, nxo, K, N, mode;
};

constexpr int kMaxProbeChunk = 256;

// Chunk `blockIdx.y` of slots (at most kMaxProbeChunk), 256 probe pixels per CTA:
// Σ_slots w·upd in slot order.
static __global__ void __launch_bounds__(256) probe_partial_kernel(ProbeArgs a) {
  __shared__ int2 cs[kMaxProbeChunk];
  __shared__ float om[kMaxProbeChunk];
  const int N = a.N;
  const size_t plane = (size_t)N * N;
  const int s0 = blockIdx.y * a.chunk, s1 = min(a.nslot, s0 + a.chunk);
  for (int i = threadIdx.x; i < s1 - s0; i += 256) {
    cs[i] = a.corners[a.frames[s0 + i]];
    om[i] = a.mode == 0 ? a.omax[s0 + i] : 0.f;
  }
  __syncthreads();
  const int pix = blockIdx.x * 256 + threadIdx.x;
  if (pix >= N * N) return;
  const int yy = pix / N, xx = pix % N;
  const float2 q = a.quad[pix];
  KahanC acc[kMaxModes];
  Kahan den;
  den.init();
#pragma unroll
  for (int m = 0; m < kMaxModes; ++m) acc[m].init();
#pragma unroll 4
  for (int s = s0; s < s1; ++s) {
    const int2 c = cs[s - s0];
    const float2 o = a.object[(size_t)(c.x + yy) * a.nxo + c.y + xx];
    if (a.mode >= 2) den.add(cnorm2(o));
    if (a.mode == 3) continue;
    float2 w = cconj(cmul(o, q));
    if (a.mode == 0) w = cscale(w, 1.f / ((1.f - a.alpha) * cnorm2(o) + a.alpha * om[s - s0]));
#pragma unroll
    for (int m = 0; m < kMaxModes; ++m) {
      if (m >= a.K) break;
      acc[m].add(cmul(w, a.upd[((size_t)s * a.K + m) * plane + pix]));
    }
  }
  if (a.mode != 3) {
#pragma unroll
    for (int m = 0; m < kMaxModes; ++m)
      if (m < a.K) a.partial[((size_t)blockIdx.y * a.K + m) * plane + pix] = acc[m].value();
  }
  if (a.mode >= 2) a.partial_den[(size_t)blockIdx.y * plane + pix] = den.s - den.c;
}

// The object blend of AP / DM / RAAR (engine/ops.rs:371-381) from the sums kGatherBlend wrote:
// O = (num + reg·O) / max(norm + reg, 1e-12) with reg = inertia·max norm.
static __global__ void blend_apply_kernel(float2* object, const float2* num, const float* norm,
                                   const float* norm_max, float inertia, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float reg = inertia * (*norm_max);
  object[i] = cscale(cadd(num[i], cscale(object[i], reg)), 1.f / fmaxf(norm[i] + reg, 1e-12f));
}

// The probe step of AP / DM / RAAR under the move (engine/features.rs:673-712), one block per
// probe mode m: with D = max(norm + reg, 1e-12) and reg = inertia·max norm, step = g / D,
// sums[m] = (Σ|g|²/D, reg·Σ|step|²) in double, added in a fixed order.
static __global__ void __launch_bounds__(1024) probe_pcg_step_kernel(const float2* g, const float* norm,
                                                              const float* norm_max,
                                                              float inertia, int plane,
                                                              float2* step, double* sums) {
  __shared__ double red[2][32];
  const int m = blockIdx.x;
  const float reg = inertia * (*norm_max);
  double slope = 0.0, curv = 0.0;
  for (int i = threadIdx.x; i < plane; i += 1024) {
    const float2 v = g[(size_t)m * plane + i];
    const float d = fmaxf(norm[i] + reg, 1e-12f);
    const float2 s = cscale(v, 1.f / d);
    step[(size_t)m * plane + i] = s;
    slope += ((double)v.x * v.x + (double)v.y * v.y) / d;
    curv += (double)reg * ((double)s.x * s.x + (double)s.y * s.y);
  }
  slope = warp_sum(slope);
  curv = warp_sum(curv);
  if (threadIdx.x % 32 == 0) {
    red[0][threadIdx.x / 32] = slope;
    red[1][threadIdx.x / 32] = curv;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < 32; ++w) {
      a += red[0][w];
      b += red[1][w];
    }
    sums[2 * m] = a;
    sums[2 * m + 1] = b;
  }
}

// Per slot and probe mode, Σ_pixels |O_window|²·|W|² in double (‖A·s‖² of one frame's view of
// the moved step W), added in a fixed order; grid (slots, K).
static __global__ void __launch_bounds__(256) weighted_norm_kernel(const float2* waves,
                                                            const float2* object,
                                                            const int* frames,
                                                            const int2* corners, int nxo, int N,
                                                            int K, double* out) {
  __shared__ double red[8];
  const int slot = blockIdx.x, m = blockIdx.y;
  const size_t plane = (size_t)N * N;
  const int2 c = corners[frames[slot]];
  const float2* w = waves + ((size_t)slot * K + m) * plane;
  double acc = 0.0;
  for (int pix = threadIdx.x; pix < N * N; pix += 256) {
    const int y = pix / N, x = pix % N;
    acc += (double)cnorm2(object[(size_t)(c.x + y) * nxo + c.y + x]) * cnorm2(w[pix]);
  }
  acc = warp_sum(acc);
  if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < 8; ++i) s += red[i];
    out[(size_t)slot * K + m] = s;
  }
}

// P_m += alpha_m·step_m over the K probe planes.
struct ModeCoefs {
  float c[kMaxModes];
};
static __global__ void probe_modes_axpy_kernel(float2* probe, const float2* step, ModeCoefs alpha,
                                        int plane, int count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float a = alpha.c[i / plane];
  if (a != 0.f) probe[i] = cadd(probe[i], cscale(step[i], a));
}

// The probe blend's norm Σ_frames |O|² per pixel: the chunks' sums in chunk order into `den`,
// and its maximum into *dmax (zeroed by the caller).
static __global__ void __launch_bounds__(256) probe_norm_kernel(const float* partial_den, int nchunk,
                                                         int plane, float* den, float* dmax) {
  __shared__ float red[8];
  const int i = blockIdx.x * 256 + threadIdx.x;
  float v = 0.f;
  if (i < plane) {
    Kahan acc;
    acc.init();
    for (int ch = 0; ch < nchunk; ++ch) acc.add(partial_den[(size_t)ch * plane + i]);
    v = acc.s - acc.c;
    den[i] = v;
  }
  v = warp_max(v);
  if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    float mx = 0.f;
    for (int w = 0; w < 8; ++w) mx = fmaxf(mx, red[w]);
    atomic_max_nonneg(dmax, mx);
  }
}

// Σ over chunks in order; mode 0: P += coef·Σ; 1: out = coef·Σ; 2: out += Σ compensated;
// 3: the blend P = (Σ + reg·P) / max(norm + reg, 1e-12) with reg = coef·max norm
// (engine/ops.rs:371-381), `norm` one plane shared by the modes.
static __global__ void probe_finalize_kernel(const float2* partial, int nchunk, int count,
                                      float2* probe, float2* out, float2* comp, float coef,
                                      int mode, const float* norm = nullptr,
                                      const float* norm_max = nullptr, int plane = 1) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  KahanC acc;
  acc.init();
  for (int ch = 0; ch < nchunk; ++ch) acc.add(partial[(size_t)ch * count + i]);
  const float2 v = acc.value();
  if (mode == 0) {
    probe[i] = cadd(probe[i], cscale(v, coef));
  } else if (mode == 3) {
    const float reg = coef * (*norm_max);
    probe[i] = cscale(cadd(v, cscale(probe[i], reg)), 1.f / fmaxf(norm[i % plane] + reg, 1e-12f));
  } else if (mode == 1) {
    out[i] = cscale(v, coef);
  } else {
    float2 g = out[i], cc = comp[i];
    const float yr = v.x - cc.x, yi = v.y - cc.y;
    const float tr = g.x + yr, ti = g.y + yi;
    comp[i] = make_float2((tr - g.x) - yr, (ti - g.y) - yi);
    out[i] = make_float2(tr, ti);
  }
}

}  // namespace ptyb
