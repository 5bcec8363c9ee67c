// The per-frame pass of the reconstruction: exit waves → 2-D FFT → detector-plane residual →
// inverse 2-D FFT → exit-wave update, for every probe mode of one diffraction frame, on one
// thread-block cluster whose distributed shared memory holds the frame's K planes.
//
// Cluster of C CTAs, CTA rank r owning H = N/C rows. Shared memory holds K·H lines of
// L = N+1 float2 (the pad keeps transposed accesses off one bank). The row FFTs run on rows; a
// cluster-wide transpose through DSMEM turns the rows into H columns per CTA, stored as lines,
// so the column FFTs, the per-pixel projection (which needs every mode at a pixel) and the
// inverse column FFTs run on local lines; a second transpose brings the rows back for the
// inverse row FFTs and the epilogue. Nothing but the object window, the counts and the output
// touches global memory.
//
// Reference operators followed (physwkim/ptyrs): exit wave `obj_probe_to_psi`
// (engine/ops.rs:47-71), unitary FFT (engine/fft.rs:155-234), the rPIE modulus
// (engine/ptycho.rs:928-945), the Poisson gradient (engine/ops.rs:161-195), the LSQML residual
// (engine/lsqml.rs:155-170) and the LLK sums (engine/ops.rs:119-154).
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
};

enum Cost : int { kCostPoisson = 0, kCostAmplitude = 1 };

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
  const float* a_far;    // [slot] LSQML far-field step
  int nyo, nxo, nprobe, nobj, cost;
};

template <int N, int C>
struct FrameShape {
  static constexpr int H = N / C;           // rows (then columns) per CTA
  static constexpr int T = H * N / 16;      // threads: 16 transposed values each per mode
  static constexpr int L = N + 1;           // line stride in float2
  static constexpr int G = LineShape<N>::N2; // threads per line FFT
  static constexpr int E = H * N / T;       // = 16
};

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
PTYB_D void all_lines(float2* S, int nlines, const float2* tw) {
  using F = FrameShape<N, C>;
  const int g = threadIdx.x / F::G, t = threadIdx.x % F::G;
  for (int line = g; line < nlines; line += F::T / F::G) line_fft<N, DIR>(S + line * F::L, t, tw);
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
      v[i] = src[(m * F::H + j % F::H) * F::L + r * F::H + c];
    }
    csync<C>(cluster);
#pragma unroll
    for (int i = 0; i < F::E; ++i) {
      const int e = threadIdx.x + i * F::T;
      const int c = e % F::H, j = e / F::H;
      S[(m * F::H + c) * F::L + j] = v[i];
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

template <int N, int C, int MODE>
__global__ void __launch_bounds__(FrameShape<N, C>::T)
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
  for (int i = tid; i < N; i += T) tw[i] = a.tw[i];

  float omax = 0.f;
  if (MODE == kFromStore) {
    const float2* src = a.field + ((size_t)slot * C + r) * K * H * N;
    for (int idx = tid; idx < K * H * N; idx += T) {
      const int line = idx / N, e = idx % N;
      S[line * L + e] = src[idx];
    }
  } else {
    // Exit waves ψ = P·O·q of shifted rows r·H .. r·H+H-1, every mode.
    for (int idx = tid; idx < K * H * N; idx += T) {
      const int m = idx / (H * N), rem = idx % (H * N);
      const int yl = rem / N, jx = rem % N;
      const int ny = (r * H + yl + N / 2) & (N - 1), nx = (jx + N / 2) & (N - 1);
      const int pm = m % a.nprobe, om = m / a.nprobe;
      const float2 p = a.probe[((size_t)pm * N + ny) * N + nx];
      const float2 o = a.object[((size_t)om * a.nyo + corner.x + ny) * a.nxo + corner.y + nx];
      const float2 q = a.quad[ny * N + nx];
      S[(m * H + yl) * L + jx] = cmul(cmul(p, o), q);
      if (MODE == kRpie && om == 0) omax = fmaxf(omax, cnorm2(o));
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

  if (MODE != kFromStore) {
    all_lines<N, C, -1>(S, K * H, tw);
    transpose<N, C>(S, K, cluster);  // its first cluster barrier publishes red[0]
    if (MODE == kRpie && r == 0 && tid == 0) {
      float mx = 0.f;
      for (int q = 0; q < C; ++q)
        mx = fmaxf(mx, *reinterpret_cast<float*>(C > 1 ? cluster.map_shared_rank(red, q) : red));
      a.omax[slot] = mx;
    }
    all_lines<N, C, -1>(S, K * H, tw);
  }

  // Detector plane: CTA r holds columns r·H .. r·H+H-1 as lines (m·H + c), elements ky.
  // Unnormalised transforms: Ψ_ortho = S/N, and the inverse of the update takes a 1/N more.
  constexpr float inv_n = 1.0f / N;
  constexpr float inv_n2 = 1.0f / ((float)N * (float)N);
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  const float* iobs = a.iobs + (size_t)f * N * N;
  const float afar = (MODE == kLsqmlFused || MODE == kFromStore) ? a.a_far[slot] : 0.f;
  for (int idx = tid; idx < H * N; idx += T) {
    const int c = idx % H, ky = idx / H;
    const int kx = r * H + c;
    float ic = 0.f;
    for (int m = 0; m < K; ++m) ic += cnorm2(S[(m * H + c) * L + ky]);
    ic *= inv_n2;
    const float yo = iobs[ky * N + kx];
    const bool masked = yo < 0.f;
    if (MODE == kStore) {
      a.icalc[((size_t)slot * N + ky) * N + kx] = ic;
      continue;
    }
    if (MODE == kLlk) {
      if (!masked) {
        acc[0] += yo > 0.f ? (double)ic - yo + (double)yo * log((double)yo / ic) : (double)ic;
        const double dg = (double)yo - ic;
        acc[1] += dg * dg / ((double)yo + 1.0);
        const double de = sqrt((double)yo) - sqrt((double)ic);
        acc[2] += 4.0 * de * de;
        acc[3] += ic;
      }
      continue;
    }
    float fac;
    if (MODE == kRpie) {
      fac = masked ? 1.f : sqrtf(yo + 1e-7f) / (sqrtf(ic) + 1e-7f);
    } else if (MODE == kMlGrad) {
      fac = masked ? 0.f : 2.f * (1.f - yo / fmaxf(ic, 1e-12f));
    } else {
      float cres = 0.f;
      if (!masked)
        cres = a.cost == kCostPoisson ? 1.f - yo / (ic + 1e-6f)
                                      : 2.f * (1.f - sqrtf(fmaxf(yo, 0.f)) / (sqrtf(ic) + 1e-9f));
      fac = 1.f - afar * cres;
    }
    fac *= inv_n2;
    for (int m = 0; m < K; ++m) {
      float2& v = S[(m * H + c) * L + ky];
      v = cscale(v, fac);
    }
  }
  (void)inv_n;

  if (MODE == kLlk) {
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
  if (MODE == kStore) {
    __syncthreads();
    float2* dst = a.field + ((size_t)slot * C + r) * K * H * N;
    for (int idx = tid; idx < K * H * N; idx += T) {
      const int line = idx / N, e = idx % N;
      dst[idx] = S[line * L + e];
    }
    return;
  }
  __syncthreads();
  all_lines<N, C, +1>(S, K * H, tw);
  transpose<N, C>(S, K, cluster);
  all_lines<N, C, +1>(S, K * H, tw);

  // Epilogue on shifted rows: out = ψ' − ψ (or ψ'), natural layout.
  float2* out = a.out + (size_t)slot * K * N * N;
  for (int idx = tid; idx < K * H * N; idx += T) {
    const int m = idx / (H * N), rem = idx % (H * N);
    const int yl = rem / N, jx = rem % N;
    const int ny = (r * H + yl + N / 2) & (N - 1), nx = (jx + N / 2) & (N - 1);
    float2 v = S[(m * H + yl) * L + jx];
    if (MODE != kMlGrad) {
      const int pm = m % a.nprobe, om = m / a.nprobe;
      const float2 p = a.probe[((size_t)pm * N + ny) * N + nx];
      const float2 o = a.object[((size_t)om * a.nyo + corner.x + ny) * a.nxo + corner.y + nx];
      const float2 q = a.quad[ny * N + nx];
      v = csub(v, cmul(cmul(p, o), q));
    }
    out[((size_t)m * N + ny) * N + nx] = v;
  }
}

}  // namespace ptyb
