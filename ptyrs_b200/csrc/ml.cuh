// Poisson maximum-likelihood conjugate gradient on the device (physwkim/ptyrs
// engine/ptycho.rs:775-842): the line-search numerator and denominator of
// `cg_poisson_gamma` (engine/ops.rs:206-253) per frame, and the array reductions of the
// Polak–Ribière β and of `scale_obj_probe` (engine/ptycho.rs:577-591).
#pragma once
#include "frame.cuh"

namespace ptyb {

// Per frame: with po = F(P·O·q) the gradient pass kept, a = F(P·dO·q + dP·O·q) and
// b = F(dP·dO·q) mode by mode, per-pixel accumulators calc = Σ|po|², r = Σ Re(p̄o·a),
// s = Σ |a|² + 2·Re(p̄o·b); then over unmasked pixels, d = 1 − I/max(calc, 1e-32):
// num = −Σ 2·r·d, den = Σ 2·s·d + I·(2r/calc)². The b-term of den is linear in b, so it is
// taken in the exit plane against the gradient pass's field (no transform of b). Shared
// memory: one plane of H lines (a) and the three accumulators (rows padded to N + 1), so two
// CTAs share an SM.
struct GammaArgs {
  const float2* object;
  const float2* d_obj;
  const float2* probe;
  const float2* d_probe;
  const float2* quad;
  const float2* tw;
  const float* iobs;
  const int* frames;
  const int2* corners;
  double* out;  // [slot][2]: num, den
  int nyo, nxo, nprobe, nobj;
  // Elements between consecutive slots' probe and probe direction: 0 for the shared ones,
  // K·N·N for the per-frame moved ones of the position model.
  int probe_stride;
  // po = DFT(P·O·q) of every slot and mode as the gradient pass kept it, [slot][K][kx][ky],
  // and its exit-plane gradient field g = IDFT(2(1 − I/Ĩ)·po)/N² (masked 0), [slot][K][N][N].
  const float2* psi;
  const float2* g;
};

template <int N, int C>
__host__ __device__ constexpr size_t gamma_smem_bytes() {
  using F = FrameShape<N, C>;
  return (size_t)F::H * F::L * sizeof(float2) + 3 * (size_t)F::H * (N + 1) * sizeof(float) +
         N * sizeof(float2) + 160 * sizeof(double);
}

template <int N, int C>
__global__ void __launch_bounds__(FrameShape<N, C>::T, 2) gamma_kernel(GammaArgs a) {
  using F = FrameShape<N, C>;
  constexpr int H = F::H, T = F::T, L = F::L, AS = N + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* S1 = reinterpret_cast<float2*>(smem_raw);           // a, then b
  float* acc = reinterpret_cast<float*>(S1 + (size_t)H * L);  // [3][H][N + 1]
  double* red = reinterpret_cast<double*>(acc + 3 * H * AS + 2 * N);
  cg::cluster_group cluster = cg::this_cluster();
  const int r = C > 1 ? (int)cluster.block_rank() : 0;
  const int slot = blockIdx.x / C;
  const int f = a.frames[slot];
  const int2 corner = a.corners[f];
  const int tid = threadIdx.x;
  const int K = a.nprobe * a.nobj;
  constexpr float inv_n2 = 1.0f / ((float)N * (float)N);
  LineTwiddles<N> ltw;
  ltw.load(a.tw, tid % F::G);
  for (int i = tid; i < 3 * H * AS; i += T) acc[i] = 0.f;
  // the kept detector columns the column phase reads, fetched into L2 now
  for (int i = tid; i < K * H * (N / 16); i += T) {
    const int row = i / (N / 16), m = row / H, c = row % H;
    asm volatile("prefetch.global.L2 [%0];" ::"l"(a.psi + ((size_t)slot * K + m) * N * N +
                                                  (size_t)(r * H + c) * N + (i % (N / 16)) * 16));
  }

  // The b-term of den, Σ_pix 2·d·2·Re(p̄o·B)/N², by Parseval in the exit plane:
  // 2·Re Σ_x conj(g)·b with g = IDFT(2d·po)/N² the gradient pass's field (0 where masked).
  double gb = 0.0;
  for (int m = 0; m < K; ++m) {
    const int pm = m % a.nprobe, om = m / a.nprobe;
    const float2* po_m = a.psi + ((size_t)slot * K + m) * N * N + (size_t)r * H * N;
    const float2* g_m = a.g + ((size_t)slot * K + m) * N * N;
    // Exit-plane rows of a; b and its product with g on the way.
#pragma unroll 4
    for (int idx = tid; idx < H * N; idx += T) {
      const int yl = idx / N, jx = idx % N;
      const int ny = (r * H + yl + N / 2) % N, nx = (jx + N / 2) % N;
      const size_t pi = (size_t)slot * a.probe_stride + ((size_t)pm * N + ny) * N + nx;
      const size_t oi = ((size_t)om * a.nyo + corner.x + ny) * a.nxo + corner.y + nx;
      const float2 dp = a.d_probe[pi], dob = a.d_obj[oi], q = a.quad[ny * N + nx];
      const float2 v = cadd(cmul(a.probe[pi], dob), cmul(dp, a.object[oi]));
      S1[yl * L + (jx ^ swz(yl))] = cmul(v, q);
      const float2 b = cmul(cmul(dp, dob), q), gv = g_m[(size_t)ny * N + nx];
      gb += (double)gv.x * b.x + (double)gv.y * b.y;
    }
    __syncthreads();
    all_lines<N, C, -1>(S1, H, ltw);
    transpose<N, C>(S1, 1, cluster);
    all_lines<N, C, -1>(S1, H, ltw);
    // Columns kx = r·H + c, elements ky; po read from the gradient pass's columns.
#pragma unroll 4
    for (int idx = tid; idx < H * N; idx += T) {
      const int c = idx / N, ky = idx % N;
      const float2 po = po_m[(size_t)c * N + ky], v = S1[c * L + (ky ^ swz(c))];
      acc[c * AS + ky] += cnorm2(po) * inv_n2;
      acc[(H + c) * AS + ky] += (po.x * v.x + po.y * v.y) * inv_n2;
      acc[(2 * H + c) * AS + ky] += cnorm2(v) * inv_n2;
    }
    __syncthreads();
  }
  const float* iobs = a.iobs + (size_t)f * N * N;
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  for (int idx = tid; idx < H * N; idx += T) {
    const int c = idx % H, ky = idx / H;
    const float yo = iobs[ky * N + r * H + c];
    if (yo < 0.f) continue;
    const double calc = fmax((double)acc[c * AS + ky], 1e-32);
    const double rr = acc[(H + c) * AS + ky], ss = acc[(2 * H + c) * AS + ky];
    const double d = 1.0 - (double)yo / calc;
    v[0] -= 2.0 * rr * d;
    const double t = 2.0 * rr / calc;
    v[1] += 2.0 * ss * d + (double)yo * t * t;
  }
  v[1] += 2.0 * gb;
  block_sum<T>(v, 2, red);
  csync<C>(cluster);
  if (r == 0 && tid == 0) {
    double num = 0.0, den = 0.0;
    for (int q = 0; q < C; ++q) {
      const double* rq = C > 1 ? cluster.map_shared_rank(red, q) : red;
      num += rq[0];
      den += rq[1];
    }
    a.out[slot * 2] = num;
    a.out[slot * 2 + 1] = den;
  }
  csync<C>(cluster);
}

// Per block, in double: mode 0 Σ Re(conj(g)·(g − h)) and Σ |h|² (Polak–Ribière);
// mode 1 Σ |g| (the modulus sum of scale_obj_probe); mode 2 Σ Re(conj(g)·h) (BH's ⟨g, D⟩).
// Partial sums [block][2].
static __global__ void __launch_bounds__(256) array_sums_kernel(const float2* g, const float2* h,
                                                         size_t n, int mode, double* partial) {
  __shared__ double sh[16];
  double s0 = 0.0, s1 = 0.0;
  for (size_t i = (size_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (size_t)gridDim.x * 256) {
    const float2 a = g[i];
    if (mode == 0) {
      const float2 b = h[i];
      s0 += (double)a.x * ((double)a.x - b.x) + (double)a.y * ((double)a.y - b.y);
      s1 += (double)b.x * b.x + (double)b.y * b.y;
    } else if (mode == 2) {
      const float2 b = h[i];
      s0 += (double)a.x * b.x + (double)a.y * b.y;
    } else {
      s0 += sqrt((double)a.x * a.x + (double)a.y * a.y);
    }
  }
  s0 = warp_sum(s0);
  s1 = warp_sum(s1);
  if (threadIdx.x % 32 == 0) {
    sh[threadIdx.x / 32] = s0;
    sh[8 + threadIdx.x / 32] = s1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a0 = 0.0, a1 = 0.0;
    for (int w = 0; w < 8; ++w) {
      a0 += sh[w];
      a1 += sh[8 + w];
    }
    partial[blockIdx.x * 2] = a0;
    partial[blockIdx.x * 2 + 1] = a1;
  }
}

// d = beta·d − g.
static __global__ void cg_direction_kernel(float2* d, const float2* g, float beta, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float2 a = d[i], b = g[i];
  d[i] = make_float2(a.x * beta - b.x, a.y * beta - b.y);
}

// x += gamma·d (gamma in double, applied in float).
static __global__ void axpy_kernel(float2* x, const float2* d, float gamma, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  x[i] = cadd(x[i], cscale(d[i], gamma));
}

// x *= s.
static __global__ void scale_kernel(float2* x, float s, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  x[i] = cscale(x[i], s);
}

// x[k][y][x] *= exp(i·2π·sign·(dy·(y − hy)/sy + dx·(x − hx)/sx)) for every plane k
// (the ramps of `zero_phase_ramp`, engine/ptycho.rs:1153-1170), phase in double.
static __global__ void ramp_kernel(float2* x, int nplanes, int ny, int nx, double dy, double dx,
                            double sy, double sx, double sign) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t n = (size_t)nplanes * ny * nx;
  if (i >= n) return;
  const int yy = (int)((i / nx) % ny), xx = (int)(i % nx);
  const double ph = sign * 2.0 * 3.14159265358979323846 *
                    (dy * (yy - ny / 2) / sy + dx * (xx - nx / 2) / sx);
  double sn, cs;
  sincos(ph, &sn, &cs);
  const float2 v = x[i];
  x[i] = make_float2((float)(v.x * cs - v.y * sn), (float)(v.x * sn + v.y * cs));
}

}  // namespace ptyb
