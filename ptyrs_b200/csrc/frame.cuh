// The per-frame pass of the reconstruction: exit waves → 2-D FFT → detector-plane residual →
// inverse 2-D FFT → exit-wave update, for every probe mode of one diffraction frame, on one
// thread-block cluster whose distributed shared memory holds the frame's K planes.
//
// Cluster of C CTAs, CTA rank r owning H = N/C rows. Shared memory holds K·H lines of N
// float2, each XOR-swizzled (`swz`) so no access pattern conflicts on banks. The row FFTs run
// on rows; a
// cluster-wide transpose through DSMEM turns the rows into H columns per CTA, stored as lines,
// so the column FFTs, the per-pixel projection (which needs every mode at a pixel) and the
// inverse column FFTs run on local lines; a second transpose brings the rows back for the
// inverse row FFTs and the epilogue. Nothing but the object window, the counts and the output
// touches global memory.
//
// Reference operators followed (physwkim/ptyrs): exit wave `obj_probe_to_psi`
// (engine/ops.rs:47-71), unitary FFT (engine/fft.rs:155-234), the rPIE modulus
// (engine/ptycho.rs:928-945), the Poisson gradient (engine/ops.rs:161-195), the LSQML residual
// (engine/lsqml.rs:155-170), the LLK sums (engine/ops.rs:119-154) and PyNX's AP, DM and RAAR
// mixes of carried exit waves around the magnitude projection (engine/ptycho.rs:609-730).
#pragma once
#include <cooperative_groups.h>

#include "common.cuh"
#include "fft.cuh"

namespace cg = cooperative_groups;

namespace ptyb {

enum FrameMode : int {
  kRpie = 0,       // rPIE modulus; out = Δ = ψ' − ψ
  kLsqmlFused = 1, // LSQML residual from a per-frame a_far; out = χ = ψ' − ψ
  kMlGrad = 2,     // Poisson gradient 2(1 − I/Ĩ), masked 0; out = ψ'
  kLlk = 3,        // forward only; per-frame LLK sums
  kStore = 4,      // forward only; detector field and Σ_modes |Ψ|² to global
  kFromStore = 5,  // detector field from global; LSQML residual; out = χ
  kProject = 6,    // magnitude projection √I/max(√Ĩ, 1e-12), masked kept; out = ψ' − ψ
  kProjectKept = 7,// from the detector field a kMlGrad pass kept (psi_out): out = ψ' − ψ as
                   // the inverse of Ψ' − Ψ
  kCarry = 8,      // AP / DM / RAAR: projection of a mix of P·O·q and the carried waves
  kBhGrad = 9,     // BH's amplitude gradient 2(1 − √I/A), A = √Ĩ + 1e-8, masked 0; out = ψ'
                   // (kMlGrad's pass otherwise: the detector field kept in psi_out)
};

// kCostBh: BH's amplitude gradient 2(1 − √I/A), A = √Ĩ + 1e-8 (the multislice gradient pass)
enum Cost : int { kCostPoisson = 0, kCostAmplitude = 1, kCostBh = 2 };

struct FrameArgs {
  const float2* object;  // [nobj][nyo][nxo]
  const float2* probe;   // [nprobe][N][N] natural layout
  const float2* quad;    // [N][N] natural: the plane phase the exit transform starts with
  const float2* tw;      // [N]: e^{-2πi·t/N}
  const float* iobs;     // [nframe][N][N] FFT-shifted layout; < 0 masked
  const int* frames;     // frame of each slot of the launch
  const int2* corners;   // [nframe] window corner (x = oy, y = ox)
  float2* out;           // [slot][K][N][N] natural layout
  float2* field;         // [slot][C][K·H][N] detector field in the CTA's strip layout
  float* icalc;          // [slot][N][N] Σ_modes |Ψ|², detector layout
  float* omax;           // [slot] max |O|² over the window (object mode 0)
  double* llk;           // [slot][4] Poisson, Gaussian, Euclidian, photons
  const float* a_far;    // [slot] LSQML far-field step (kLsqmlFused)
  // LSQML Poisson far-field step, PtychoShelves' xi solver in two passes
  // (engine/lsqml.rs:133-150): kStore runs pass 1 from `a_prev` (by frame when
  // `a_prev_by_frame`), kFromStore pass 2 from `a_mid`; each writes its result to `a_out`.
  const float* a_prev;
  const float* a_mid;
  float* a_out;
  int a_prev_by_frame, nslot;
  int nyo, nxo, nprobe, nobj, cost;
  // Elements between consecutive slots' probes: 0 for the shared probe, K·N·N for the
  // per-frame (moved) probes of the position model.
  int probe_stride;
  // kMlGrad, optional: the detector field Ψ = DFT(P·O·q) of every mode kept for the line
  // search and the magnitude projection, [slot][K][kx][ky] (columns contiguous); kProjectKept
  // reads it back.
  float2* psi_out;
  // kCarry (AP, DM, RAAR; engine/ptycho.rs:609-730): the carried exit waves `carry` and RAAR's
  // iterate `iter` of the launch's frames, [slot][K][N][N] natural layout. The projection's
  // input is S = c_po·PO + c_psi·carry + c_it·iter (iter ← S when `iter` is set); the carried
  // waves become Π(S) + c_refl·(PO − S). Terms whose coefficient is 0 are not read. With `llk`
  // set, the pass also writes the per-frame LLK sums of the field it projects.
  float2* carry;
  float2* iter;
  float c_po, c_psi, c_it, c_refl;
};

template <int N, int C>
struct FrameShape {
  static constexpr int H = N / C;           // rows (then columns) per CTA
  static constexpr int T = H * N / 16;      // threads: 16 transposed values each per mode
  static constexpr int L = N;               // line stride in float2 (lines are swizzled)
  static constexpr int G = LineShape<N>::N2; // threads per line FFT
  static constexpr int E = H * N / T;       // = 16
};

// Resident CTAs per SM the per-frame kernels are compiled for: two at 384 threads or fewer
// (a cap of 128 registers at 256 threads, 113 at the 288 of sides 96 and 192), one above.
template <int N, int C>
__host__ __device__ constexpr int frame_min_blocks() {
  return FrameShape<N, C>::T <= 384 ? 2 : 1;
}

template <int N, int C>
__host__ __device__ constexpr size_t frame_smem_bytes(int K) {
  return (size_t)K * FrameShape<N, C>::H * FrameShape<N, C>::L * sizeof(float2) +
         N * sizeof(float2) + 160 * sizeof(double);
}

// Barrier over the cluster (a plain block barrier when the cluster is one CTA).
template <int C>
PTYB_D void csync(cg::cluster_group& cluster) {
  if (C > 1)
    cluster.sync();
  else
    __syncthreads();
}

// Every local line through a forward (DIR = -1) or inverse (+1) line FFT; the block barrier at
// the end publishes every line to every thread of the CTA.
template <int N, int C, int DIR>
PTYB_D void all_lines(float2* S, int nlines, const LineTwiddles<N>& tw) {
  using F = FrameShape<N, C>;
  const int g = threadIdx.x / F::G, t = threadIdx.x % F::G;
  for (int line = g; line < nlines; line += F::T / F::G)
    line_fft<N, DIR>(S + line * F::L, t, tw, swz(line));
  __syncthreads();
}

// Cluster-wide transpose of the K planes: rows → columns or back (the same map). Value
// (line m·H + c, element j) of CTA r comes from CTA j/H, line m·H + j%H, element r·H + c.
template <int N, int C>
PTYB_D void transpose(float2* S, int K, cg::cluster_group& cluster) {
  using F = FrameShape<N, C>;
  const int r = C > 1 ? (int)cluster.block_rank() : 0;
  csync<C>(cluster);
  for (int m = 0; m < K; ++m) {
    float2 v[F::E];
#pragma unroll
    for (int i = 0; i < F::E; ++i) {
      const int e = threadIdx.x + i * F::T;
      const int c = e % F::H, j = e / F::H;
      const float2* src = C > 1 ? cluster.map_shared_rank(S, j / F::H) : S;
      const int sl = m * F::H + j % F::H;
      v[i] = src[sl * F::L + ((r * F::H + c) ^ swz(sl))];
    }
    csync<C>(cluster);
#pragma unroll
    for (int i = 0; i < F::E; ++i) {
      const int e = threadIdx.x + i * F::T;
      const int c = e % F::H, j = e / F::H;
      const int dl = m * F::H + c;
      S[dl * F::L + (j ^ swz(dl))] = v[i];
    }
  }
  __syncthreads();
}

// Block-wide sums of n ≤ 4 doubles into red[0..n) of thread 0 (others undefined).
template <int T>
PTYB_D void block_sum(double (&v)[4], int n, double* red) {
  for (int k = 0; k < n; ++k) v[k] = warp_sum(v[k]);
  __syncthreads();
  const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
  double* part = red + 8;  // [T/32][4]
  if (lane == 0)
    for (int k = 0; k < n; ++k) part[w * 4 + k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 0; k < n; ++k) {
      double s = 0.0;
      for (int q = 0; q < T / 32; ++q) s += part[q * 4 + k];
      red[k] = s;
    }
  }
  __syncthreads();
}

// Mean of the launch's far-field steps, summed by warp 0 in a fixed order (lane-strided
// partial sums, then a fixed butterfly), so every CTA gets the same value; broadcast through
// `slot` in shared memory (block barrier inside).
PTYB_D double batch_mean(const float* v, const int* frames, int by_frame, int nslot,
                         double* slot) {
  if (threadIdx.x < 32) {
    double s = 0.0;
    for (int i = threadIdx.x; i < nslot; i += 32) s += v[by_frame ? frames[i] : i];
    s = warp_sum(s);
    if (threadIdx.x == 0) *slot = s / nslot;
  }
  __syncthreads();
  return *slot;
}

// Cluster-wide sums of two doubles (every CTA gets the totals, added in rank order).
template <int N, int C>
PTYB_D void cluster_sum2(double& x, double& y, double* red, cg::cluster_group& cluster) {
  using F = FrameShape<N, C>;
  double v[4] = {x, y, 0.0, 0.0};
  block_sum<F::T>(v, 2, red);
  csync<C>(cluster);
  double sx = 0.0, sy = 0.0;
  for (int q = 0; q < C; ++q) {
    const double* rq = C > 1 ? cluster.map_shared_rank(red, q) : red;
    sx += rq[0];
    sy += rq[1];
  }
  csync<C>(cluster);
  x = sx;
  y = sy;
}

// Cluster-wide sums of four doubles, every thread getting them (rank order, as cluster_sum2).
template <int N, int C>
PTYB_D void cluster_sum4(double (&v)[4], double* red, cg::cluster_group& cluster) {
  using F = FrameShape<N, C>;
  block_sum<F::T>(v, 4, red);
  csync<C>(cluster);
  double t[4] = {0.0, 0.0, 0.0, 0.0};
  for (int q = 0; q < C; ++q) {
    const double* rq = C > 1 ? cluster.map_shared_rank(red, q) : red;
#pragma unroll
    for (int k = 0; k < 4; ++k) t[k] += rq[k];
  }
  csync<C>(cluster);
#pragma unroll
  for (int k = 0; k < 4; ++k) v[k] = t[k];
}

// The projection's input S = c_po·po + c_psi·carry + c_it·iter at element `pix` of mode m of
// `slot` (kCarry); the prologue (`store`) also writes it to RAAR's iterate.
template <int N>
PTYB_D float2 carry_mix(const FrameArgs& a, float2 po, int slot, int m, int pix, int K,
                        bool store) {
  const size_t gi = ((size_t)slot * K + m) * N * N + pix;
  float2 v = cscale(po, a.c_po);
  if (a.c_psi != 0.f) v = cadd(v, cscale(a.carry[gi], a.c_psi));
  if (a.c_it != 0.f) v = cadd(v, cscale(a.iter[gi], a.c_it));
  if (store && a.iter) a.iter[gi] = v;
  return v;
}

template <int N, int C, int MODE>
__global__ void __launch_bounds__(FrameShape<N, C>::T,
                                  N == 256 && FrameShape<N, C>::T <= 256 &&
                                          (MODE == kMlGrad || MODE == kBhGrad ||
                                           MODE == kProjectKept ||
                                           MODE == kLlk || MODE == kCarry)
                                      ? 3
                                      : frame_min_blocks<N, C>())
    frame_kernel(FrameArgs a) {
  using F = FrameShape<N, C>;
  constexpr int H = F::H, T = F::T, L = F::L;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int K = a.nprobe * a.nobj;
  float2* S = reinterpret_cast<float2*>(smem_raw);
  float2* tw = S + (size_t)K * H * L;
  double* red = reinterpret_cast<double*>(tw + N);  // 8 results + [T/32 ≤ 32][4] partials
  cg::cluster_group cluster = cg::this_cluster();
  const int r = C > 1 ? (int)cluster.block_rank() : 0;
  const int slot = blockIdx.x / C;
  const int f = a.frames[slot];
  const int2 corner = a.corners[f];
  const int tid = threadIdx.x;
  LineTwiddles<N> ltw;
  ltw.load(a.tw, tid % F::G);
  (void)tw;

  float omax = 0.f;
  if (MODE == kFromStore) {
    const float2* src = a.field + ((size_t)slot * C + r) * K * H * N;
#pragma unroll 8
    for (int idx = tid; idx < K * H * N; idx += T) {
      const int line = idx / N, e = idx % N;
      S[line * L + (e ^ swz(line))] = src[idx];
    }
  } else if (MODE == kProjectKept) {
    // this CTA's columns of the kept Ψ, [slot][m][kx][ky]
    const float2* src = a.psi_out + (size_t)slot * K * N * N;
#pragma unroll 8
    for (int idx = tid; idx < K * H * N; idx += T) {
      const int line = idx / N, e = idx % N, m = line / H, c = line % H;
      S[line * L + (e ^ swz(line))] = src[((size_t)m * N + r * H + c) * N + e];
    }
  } else {
    // Exit waves ψ = P·O·q of shifted rows r·H .. r·H+H-1, every mode; the object window and
    // the phase are read once per pixel.
#pragma unroll 2
    for (int idx = tid; idx < H * N; idx += T) {
      const int yl = idx / N, jx = idx % N;
      const int ny = (r * H + yl + N / 2) % N, nx = (jx + N / 2) % N;
      const float2 q = a.quad[ny * N + nx];
      for (int om = 0; om < a.nobj; ++om) {
        const float2 o = a.object[((size_t)om * a.nyo + corner.x + ny) * a.nxo + corner.y + nx];
        const float2 oq = cmul(o, q);
        if (MODE == kRpie && om == 0) omax = fmaxf(omax, cnorm2(o));
        for (int pm = 0; pm < a.nprobe; ++pm) {
          const int line = (om * a.nprobe + pm) * H + yl;
          // (P·O)·q as P·(O·q): the reference's product up to rounding
          float2 v =
              cmul(a.probe[(size_t)slot * a.probe_stride + ((size_t)pm * N + ny) * N + nx], oq);
          if (MODE == kCarry)
            v = carry_mix<N>(a, v, slot, om * a.nprobe + pm, ny * N + nx, K, true);
          S[line * L + (jx ^ swz(line))] = v;
        }
      }
    }
  }
  __syncthreads();

  if (MODE == kRpie) {
    // max |O|² over the window: block max, then across the cluster in rank order.
    omax = warp_max(omax);
    float* fred = reinterpret_cast<float*>(red + 8);
    if (tid % 32 == 0) fred[tid / 32] = omax;
    __syncthreads();
    if (tid == 0) {
      float mx = 0.f;
      for (int q = 0; q < T / 32; ++q) mx = fmaxf(mx, fred[q]);
      reinterpret_cast<float*>(red)[0] = mx;
    }
  }

  if (MODE != kFromStore && MODE != kProjectKept) {
    all_lines<N, C, -1>(S, K * H, ltw);
    transpose<N, C>(S, K, cluster);  // its first cluster barrier publishes red[0]
    if (MODE == kRpie && r == 0 && tid == 0) {
      float mx = 0.f;
      for (int q = 0; q < C; ++q)
        mx = fmaxf(mx, *reinterpret_cast<float*>(C > 1 ? cluster.map_shared_rank(red, q) : red));
      a.omax[slot] = mx;
    }
    all_lines<N, C, -1>(S, K * H, ltw);
  }

  if ((MODE == kMlGrad || MODE == kBhGrad) && a.psi_out) {
    // Ψ of this CTA's columns to [slot][m][kx][ky]
    float2* dst = a.psi_out + (size_t)slot * K * N * N;
#pragma unroll 8
    for (int idx = tid; idx < K * H * N; idx += T) {
      const int line = idx / N, e = idx % N, m = line / H, c = line % H;
      dst[((size_t)m * N + r * H + c) * N + e] = S[line * L + (e ^ swz(line))];
    }
  }

  // Detector plane: CTA r holds columns r·H .. r·H+H-1 as lines (m·H + c), elements ky.
  // Unnormalised transforms: Ψ_ortho = S/N, and the inverse of the update takes a 1/N more.
  constexpr float inv_n = 1.0f / N;
  constexpr float inv_n2 = 1.0f / ((float)N * (float)N);
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  const float* iobs = a.iobs + (size_t)f * N * N;
  float afar = MODE == kLsqmlFused ? a.a_far[slot] : 0.f;
  // Each thread's 16 pixels (idx = tid + i·T): their counts and model intensity, read once.
  constexpr int kPixPerThread = H * N / T;
  float yo_r[kPixPerThread], ic_r[kPixPerThread];
#pragma unroll
  for (int i = 0; i < kPixPerThread; ++i) {
    const int idx = tid + i * T;
    const int c = idx % H, ky = idx / H;
    yo_r[i] = iobs[ky * N + r * H + c];
    float ic = 0.f;
    for (int m = 0; m < K; ++m) ic += cnorm2(S[(m * H + c) * L + (ky ^ swz(m * H + c))]);
    ic_r[i] = ic * inv_n2;
  }
  if ((MODE == kStore || MODE == kFromStore) && a.cost == kCostPoisson && a.a_out) {
    // One pass of the Poisson xi solver over this frame: with prev the batch mean of the
    // previous pass, a = clip(prev/2 + Σ xi·(Ĩ − I/(1 − prev·xi)) / Σ xi²·Ĩ / 2, 0, 1).
    const double prev = MODE == kStore
                            ? batch_mean(a.a_prev, a.frames, a.a_prev_by_frame, a.nslot, red + 7)
                            : batch_mean(a.a_mid, a.frames, 0, a.nslot, red + 7);
    double num = 0.0, den = 0.0;
#pragma unroll
    for (int i = 0; i < kPixPerThread; ++i) {
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
  }
#pragma unroll
  for (int i = 0; i < kPixPerThread; ++i) {
    if (MODE == kStore && !a.icalc) break;
    const int idx = tid + i * T;
    const int c = idx % H, ky = idx / H;
    const int kx = r * H + c;
    const float ic = ic_r[i];
    const float yo = yo_r[i];
    const bool masked = yo < 0.f;
    if (MODE == kStore) {
      a.icalc[((size_t)slot * N + ky) * N + kx] = ic;
      continue;
    }
    if (MODE == kLlk || (MODE == kCarry && a.llk)) {
      if (!masked) {
        acc[0] += yo > 0.f ? (double)ic - yo + (double)yo * log((double)yo / ic) : (double)ic;
        const double dg = (double)yo - ic;
        acc[1] += dg * dg / ((double)yo + 1.0);
        const double de = sqrt((double)yo) - sqrt((double)ic);
        acc[2] += 4.0 * de * de;
        acc[3] += ic;
      }
      if (MODE == kLlk) continue;
    }
    float fac;
    if (MODE == kRpie) {
      fac = masked ? 1.f : sqrtf(yo + 1e-7f) / (sqrtf(ic) + 1e-7f);
    } else if (MODE == kProjectKept) {
      // ApplyAmplitude (engine/ops.rs:83-107) minus the identity: the kept field Ψ = DFT(ψ)
      // goes to ΔΨ = Ψ' − Ψ, whose inverse is the change ψ' − ψ itself (no model re-read)
      fac = masked ? 0.f : sqrtf(yo) / fmaxf(sqrtf(ic), 1e-12f) - 1.f;
    } else if (MODE == kProject || MODE == kCarry) {
      // ApplyAmplitude (engine/ops.rs:83-107)
      fac = masked ? 1.f : sqrtf(yo) / fmaxf(sqrtf(ic), 1e-12f);
    } else if (MODE == kMlGrad) {
      fac = masked ? 0.f : 2.f * (1.f - yo / fmaxf(ic, 1e-12f));
    } else if (MODE == kBhGrad) {
      // BH's residual (engine/bh.rs:255-265)
      fac = masked ? 0.f : 2.f * (1.f - sqrtf(yo) / (sqrtf(ic) + 1e-8f));
    } else {
      float cres = 0.f;
      if (!masked)
        cres = a.cost == kCostPoisson ? 1.f - yo / (ic + 1e-6f)
                                      : 2.f * (1.f - sqrtf(fmaxf(yo, 0.f)) / (sqrtf(ic) + 1e-9f));
      fac = 1.f - afar * cres;
    }
    fac *= inv_n2;
    for (int m = 0; m < K; ++m) {
      float2& v = S[(m * H + c) * L + (ky ^ swz(m * H + c))];
      v = cscale(v, fac);
    }
  }
  (void)inv_n;

  if (MODE == kLlk || (MODE == kCarry && a.llk)) {
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
    if (MODE == kLlk) return;
  }
  if (MODE == kStore) {
    __syncthreads();
    float2* dst = a.field + ((size_t)slot * C + r) * K * H * N;
#pragma unroll 8
    for (int idx = tid; idx < K * H * N; idx += T) {
      const int line = idx / N, e = idx % N;
      dst[idx] = S[line * L + (e ^ swz(line))];
    }
    return;
  }
  __syncthreads();
  all_lines<N, C, +1>(S, K * H, ltw);
  transpose<N, C>(S, K, cluster);
  all_lines<N, C, +1>(S, K * H, ltw);

  // Epilogue on shifted rows: dst = ψ' − ψ (or ψ'), natural layout; the object window and the
  // phase are read once per pixel.
  auto epilogue = [&](float2* base, bool subtract) {
    float2* dst = base + (size_t)slot * K * N * N;
#pragma unroll 2
    for (int idx = tid; idx < H * N; idx += T) {
      const int yl = idx / N, jx = idx % N;
      const int ny = (r * H + yl + N / 2) % N, nx = (jx + N / 2) % N;
      float2 q = make_float2(0.f, 0.f);
      if (subtract) q = a.quad[ny * N + nx];
      for (int om = 0; om < a.nobj; ++om) {
        float2 oq = make_float2(0.f, 0.f);
        if (subtract)
          oq = cmul(a.object[((size_t)om * a.nyo + corner.x + ny) * a.nxo + corner.y + nx], q);
        for (int pm = 0; pm < a.nprobe; ++pm) {
          const int m = om * a.nprobe + pm;
          const int line = m * H + yl;
          float2 v = S[line * L + (jx ^ swz(line))];
          if (subtract)
            v = csub(v, cmul(a.probe[(size_t)slot * a.probe_stride + ((size_t)pm * N + ny) * N + nx],
                             oq));
          dst[((size_t)m * N + ny) * N + nx] = v;
        }
      }
    }
  };
  if (MODE == kCarry) {
    // carried waves ← Π(S) + c_refl·(PO − S), in place (this thread read these pixels above)
#pragma unroll 2
    for (int idx = tid; idx < H * N; idx += T) {
      const int yl = idx / N, jx = idx % N;
      const int ny = (r * H + yl + N / 2) % N, nx = (jx + N / 2) % N;
      const int pix = ny * N + nx;
      float2 oq = make_float2(0.f, 0.f);
      if (a.c_refl != 0.f)
        oq = cmul(a.object[(size_t)(corner.x + ny) * a.nxo + corner.y + nx], a.quad[pix]);
      for (int m = 0; m < K; ++m) {
        const int line = m * H + yl;
        float2 v = S[line * L + (jx ^ swz(line))];
        const size_t gi = ((size_t)slot * K + m) * N * N + pix;
        if (a.c_refl != 0.f) {
          const float2 po =
              cmul(a.probe[(size_t)slot * a.probe_stride + (size_t)m * N * N + pix], oq);
          v = cadd(v, cscale(csub(po, carry_mix<N>(a, po, slot, m, pix, K, false)), a.c_refl));
        }
        a.carry[gi] = v;
      }
    }
    return;
  }
  epilogue(a.out, MODE != kMlGrad && MODE != kBhGrad && MODE != kProjectKept);
}

}  // namespace ptyb
