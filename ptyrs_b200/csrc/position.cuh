// The position model under Patch sampling (physwkim/ptyrs engine/features.rs:337-527,
// engine/lsqml.rs:237-270): each frame's probe moved by its sub-pixel offset on the periodic
// grid, the adjoint move of the probe directions, the Fourier derivative of the object window,
// pty-chi's gradient position sums and its clipped SGD step (in double).
#pragma once
#include "frame.cuh"

namespace ptyb {

enum MoveMode : int {
  kMoveBack = 1,      // planes[slot][m] = conj(q)·T_{−d}(q·planes)  (the adjoint move, in place)
  kDerivWindow = 2,   // planes[slot][a] = ∂_a O_window (periodic Fourier derivative), a = y, x
  kSpectrum = 4,      // planes[m] = DFT(q·P_m), unnormalised, [ky][kx] (one slot)
  kFromSpectrum = 5,  // planes[slot][m] = conj(q)·T_d(q·P_m), probe of frame f moved by d_f,
                      // from the spectrum `spec`
  kDerivSums = 6,     // per frame and axis, the position sums of AP, DM and ML from ∂T_d(q·P)
  kBackSpectrum = 7,  // planes[slot][m] = DFT(conj(O_win)·c_m)·exp(+2πi f·d)/N², [ky][kx]: one
                      // frame's term of the probe back-projection through the move's adjoint
  kPlainInverse = 8,  // planes[m] = conj(q)·IDFT(spec_m), unnormalised (one slot)
  kMoveOwn = 9,       // planes[slot][m] = conj(q)·T_d(q·planes), in place: each frame's own
                      // probe planes (the probe variation's) moved by its offset
  kDerivMove = 10     // planes[slot][m] = conj(q)·∂T_d(q·P_m) from the spectrum `spec`: the
                      // first (deriv 1 y, 2 x) or second (3 yy, 4 yx, 5 xx) derivative over
                      // the offset of kFromSpectrum's moved probe (BH's position terms)
};

struct MoveArgs {
  const float2* probe;    // [K][N][N] shared probe (kSpectrum)
  const float2* quad;     // [N][N]
  const float2* tw;       // [N]
  const float2* object;   // [nyo][nxo] (kDerivWindow, kDerivSums, kBackSpectrum)
  const int* frames;
  const int2* corners;
  const double* offsets;  // [nframe][2] (dy, dx) in object pixels
  float2* planes;         // [slot][K][N][N]
  int nxo, K;
  const float2* spec;     // [K][N][N] a spectrum, [ky][kx] (kFromSpectrum, kDerivSums,
                          // kPlainInverse)
  const float2* c;        // [slot][K][N][N] natural: the change of the exit wave (kDerivSums),
                          // the exit-plane gradient (kBackSpectrum)
  double* sums;           // [nframe][4] num_y, num_x, den_y, den_x (kDerivSums)
  int deriv;              // kDerivMove: 1 ∂y, 2 ∂x, 3 ∂y∂y, 4 ∂y∂x, 5 ∂x∂x
  // Optional, [slot][K][N][N] natural: each frame's moved probes W; kDerivSums and
  // kBackSpectrum then take c − W·O·q, the carried waves' residual against the model
  // (AP / DM / RAAR, engine/features.rs:653-725, 992-1025).
  const float2* minus;
};

// numpy fftfreq of index k of n points (engine/features.rs:337-344).
PTYB_D float fft_freq(int k, int n) { return (float)(k < (n + 1) / 2 ? k : k - n) / (float)n; }

template <int N, int C, int MODE>
__global__ void __launch_bounds__(FrameShape<N, C>::T,
                                  N == 256 && FrameShape<N, C>::T <= 256 &&
                                          (MODE == kFromSpectrum || MODE == kBackSpectrum ||
                                           MODE == kSpectrum || MODE == kPlainInverse)
                                      ? 3
                                      : frame_min_blocks<N, C>())
    move_kernel(MoveArgs a) {
  using F = FrameShape<N, C>;
  constexpr int H = F::H, T = F::T, L = F::L;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int K = MODE == kDerivWindow ? 2 : a.K;
  // planes held in shared memory: the position sums hold the two axes of one mode at a time
  const int KP = MODE == kDerivSums ? max(K, 2) : K;
  float2* S = reinterpret_cast<float2*>(smem_raw);
  double* red = reinterpret_cast<double*>(S + (size_t)KP * H * L + N);
  cg::cluster_group cluster = cg::this_cluster();
  const int r = C > 1 ? (int)cluster.block_rank() : 0;
  const int slot = blockIdx.x / C;
  constexpr bool one = MODE == kSpectrum || MODE == kPlainInverse;  // not per frame
  const int f = one ? 0 : a.frames[slot];
  const int2 corner = one ? make_int2(0, 0) : a.corners[f];
  const int tid = threadIdx.x;
  LineTwiddles<N> ltw;
  ltw.load(a.tw, tid % F::G);
  const size_t plane = (size_t)N * N;
  float2* out = a.planes + (size_t)slot * K * plane;
  constexpr float inv_n2 = 1.0f / ((float)N * (float)N);
  constexpr bool from_spec = MODE == kFromSpectrum || MODE == kDerivSums ||
                              MODE == kPlainInverse || MODE == kDerivMove;
  constexpr bool in_place = MODE == kMoveBack || MODE == kMoveOwn;
  constexpr bool moves = in_place || MODE == kFromSpectrum || MODE == kDerivSums ||
                         MODE == kDerivMove ||
                         MODE == kBackSpectrum;
  constexpr bool bare = MODE == kDerivWindow;

  float dy = 0.f, dx = 0.f;
  if (moves) {
    const float sgn = MODE == kMoveBack || MODE == kBackSpectrum ? -1.f : 1.f;
    dy = sgn * (float)a.offsets[2 * f];
    dx = sgn * (float)a.offsets[2 * f + 1];
  }
  // The translation phase exp(−2πi f·d) = exp(−2πi fy·dy)·exp(−2πi fx·dx), over N²: the row
  // factor for every ky in the free N-entry region after the planes, the column factor of this
  // thread's one column (T is a multiple of H, so a thread keeps c = tid % H).
  float2* ey = S + (size_t)KP * H * L;
  float2 ex = make_float2(1.f, 0.f);
  if (moves) {
    for (int k = tid; k < N; k += T) {
      float sn, cs;
      sincospif(-2.f * fft_freq(k, N) * dy, &sn, &cs);
      ey[k] = make_float2(cs * inv_n2, sn * inv_n2);
    }
    float sn, cs;
    sincospif(-2.f * fft_freq(r * H + tid % H, N) * dx, &sn, &cs);
    ex = make_float2(cs, sn);
  }

  if (!from_spec) {
    // Natural-layout rows r·H .. r·H+H-1 of every plane, then the forward transform.
#pragma unroll 2
    for (int idx = tid; idx < H * N; idx += T) {
      const int yl = idx / N, x = idx % N, y = r * H + yl;
      float2 w;
      if (MODE == kSpectrum || in_place)
        w = a.quad[y * N + x];
      else if (MODE == kBackSpectrum)
        w = cconj(a.object[(size_t)(corner.x + y) * a.nxo + corner.y + x]);
      for (int m = 0; m < K; ++m) {
        float2 v;
        if (MODE == kSpectrum)
          v = cmul(w, a.probe[m * plane + y * N + x]);
        else if (in_place)
          v = cmul(w, out[m * plane + y * N + x]);
        else if (MODE == kBackSpectrum) {
          float2 cv = a.c[(size_t)slot * K * plane + m * plane + y * N + x];
          if (a.minus)
            cv = csub(cv, cmul(cmul(a.minus[(size_t)slot * K * plane + m * plane + y * N + x],
                                    cconj(w)),
                               a.quad[y * N + x]));
          v = cmul(w, cv);
        }
        else
          v = a.object[(size_t)(corner.x + y) * a.nxo + corner.y + x];
        const int line = m * H + yl;
        S[line * L + (x ^ swz(line))] = v;
      }
    }
    __syncthreads();
    all_lines<N, C, -1>(S, K * H, ltw);
    transpose<N, C>(S, K, cluster);
    all_lines<N, C, -1>(S, K * H, ltw);
    if (MODE == kSpectrum || MODE == kBackSpectrum) {
      // Spectrum columns kx = r·H + c (lines m·H + c, elements ky) to [slot][m][ky][kx].
#pragma unroll 2
      for (int idx = tid; idx < H * N; idx += T) {
        const int c = idx % H, ky = idx / H;
        const float2 e = MODE == kBackSpectrum ? cmul(ey[ky], ex) : make_float2(1.f, 0.f);
        for (int m = 0; m < K; ++m)
          out[((size_t)m * N + ky) * N + r * H + c] =
              cmul(S[(m * H + c) * L + (ky ^ swz(m * H + c))], e);
      }
      return;
    }
  } else if (moves) {
    __syncthreads();  // the row factors
  }

  if (MODE == kDerivSums) {
    // Both axes of one mode at a time, the planes holding ∂_y and ∂_x of mode m's moved probe:
    // each mode's spectrum, field plane and window are read once for both axes.
    constexpr float two_pi = 2.f * 3.14159265358979f;
    const float2* cf = a.c + (size_t)slot * K * plane;
    double v4[4] = {0.0, 0.0, 0.0, 0.0};  // num_y, num_x, den_y, den_x
#pragma unroll 1
    for (int m = 0; m < K; ++m) {
#pragma unroll 2
      for (int idx = tid; idx < H * N; idx += T) {
        const int c = idx % H, ky = idx / H, kx = r * H + c;
        const float2 v = cmul(a.spec[((size_t)m * N + ky) * N + kx], cmul(ey[ky], ex));
        // × (−2πi·f_axis): the derivative of the translation phase (engine/features.rs:372-387)
        const float wy = two_pi * fft_freq(ky, N), wx = two_pi * fft_freq(kx, N);
        S[c * L + (ky ^ swz(c))] = make_float2(wy * v.y, -wy * v.x);
        S[(H + c) * L + (ky ^ swz(H + c))] = make_float2(wx * v.y, -wx * v.x);
      }
      __syncthreads();
      // two planes, as a value the compiler does not unroll the transforms' plane loops over
      int two = 2;
      asm volatile("" : "+r"(two));
      all_lines<N, C, +1>(S, two * H, ltw);
      transpose<N, C>(S, two, cluster);
      all_lines<N, C, +1>(S, two * H, ltw);
      // dψ = O·∂W on natural rows; num = Σ Re(conj(c)·dψ), den = Σ |dψ|² over modes and
      // pixels (engine/features.rs:992-1025)
#pragma unroll 2
      for (int idx = tid; idx < H * N; idx += T) {
        const int yl = idx / N, x = idx % N, y = r * H + yl;
        const float2 o = a.object[(size_t)(corner.x + y) * a.nxo + corner.y + x];
        float2 v = cf[m * plane + y * N + x];
        if (a.minus)
          v = csub(v, cmul(cmul(a.minus[(size_t)slot * K * plane + m * plane + y * N + x], o),
                           a.quad[y * N + x]));
#pragma unroll
        for (int ax = 0; ax < 2; ++ax) {
          const int line = ax * H + yl;
          const float2 d = cmul(o, S[line * L + (x ^ swz(line))]);
          v4[ax] += (double)v.x * d.x + (double)v.y * d.y;
          v4[2 + ax] += (double)d.x * d.x + (double)d.y * d.y;
        }
      }
      __syncthreads();  // the next mode's spectrum overwrites the planes read above
    }
    cluster_sum4<N, C>(v4, red, cluster);
    if (r == 0 && tid == 0)
#pragma unroll
      for (int k = 0; k < 4; ++k) a.sums[(size_t)f * 4 + k] = v4[k];
    return;
  }

  {
    // Spectrum: column kx = r·H + c as line (m·H + c), element ky.
#pragma unroll 2
    for (int idx = tid; idx < H * N; idx += T) {
      const int c = idx % H, ky = idx / H, kx = r * H + c;
      const float fy = fft_freq(ky, N), fx = fft_freq(kx, N);
      float2 e = make_float2(1.f, 0.f);
      if (moves) {
        e = cmul(ey[ky], ex);
        if (MODE == kDerivMove) {
          // × (−2πi·f_a) or × (−2πi·f_a)(−2πi·f_b) = −4π²·f_a·f_b
          const float wy = 2.f * 3.14159265358979f * fy, wx = 2.f * 3.14159265358979f * fx;
          if (a.deriv <= 2) {
            const float w = a.deriv == 1 ? wy : wx;
            e = make_float2(w * e.y, -w * e.x);
          } else {
            const float w = a.deriv == 3 ? -wy * wy : a.deriv == 4 ? -wy * wx : -wx * wx;
            e = make_float2(w * e.x, w * e.y);
          }
        }
      }
      for (int m = 0; m < K; ++m) {
        float2& v = S[(m * H + c) * L + (ky ^ swz(m * H + c))];
        if (from_spec) {
          v = cmul(a.spec[((size_t)m * N + ky) * N + kx], e);
        } else if (MODE == kDerivWindow) {
          const float w = 2.f * 3.14159265358979f * (m == 0 ? fy : fx) * inv_n2;
          v = make_float2(-w * v.y, w * v.x);  // × 2πi·f_axis
        } else {
          v = cmul(v, e);
        }
      }
    }
    __syncthreads();
    all_lines<N, C, +1>(S, K * H, ltw);
    transpose<N, C>(S, K, cluster);
    all_lines<N, C, +1>(S, K * H, ltw);

#pragma unroll 2
    for (int idx = tid; idx < H * N; idx += T) {
      const int yl = idx / N, x = idx % N, y = r * H + yl;
      const float2 cq = bare ? make_float2(1.f, 0.f) : cconj(a.quad[y * N + x]);
      for (int m = 0; m < K; ++m) {
        const int line = m * H + yl;
        const float2 v = S[line * L + (x ^ swz(line))];
        out[m * plane + y * N + x] = bare ? v : cmul(cq, v);
      }
    }
  }
}

template <int N, int C>
__host__ __device__ constexpr size_t move_smem_bytes(int K) {
  return frame_smem_bytes<N, C>(K);
}

// planes[slot][m] = w·χ_m per natural pixel: each frame's probe direction before its adjoint
// move, w = conj(q·O_window) (LSQML, engine/lsqml.rs:200-207) or, with `omax`, rPIE's weight
// conj(q·O)/((1 − α)|O|² + α·max|O|²) (engine/ptycho.rs:1007-1026).
static __global__ void probe_terms_kernel(const float2* object, const float2* quad, const float2* chi,
                                   const int* frames, const int2* corners, int nxo, int K, int N,
                                   float2* planes, const float* omax = nullptr,
                                   float alpha = 0.f) {
  const int slot = blockIdx.y;
  const size_t plane = (size_t)N * N;
  const int2 c = corners[frames[slot]];
  for (int pix = blockIdx.x * blockDim.x + threadIdx.x; pix < N * N;
       pix += gridDim.x * blockDim.x) {
    const int y = pix / N, x = pix % N;
    const float2 o = object[(size_t)(c.x + y) * nxo + c.y + x];
    float2 w = cconj(cmul(quad[pix], o));
    if (omax) w = cscale(w, 1.f / ((1.f - alpha) * cnorm2(o) + alpha * omax[slot]));
    for (int m = 0; m < K; ++m) {
      const size_t i = ((size_t)slot * K + m) * plane + pix;
      planes[i] = cmul(w, chi[i]);
    }
  }
}

// Per slot, pty-chi's position sums on mode 0 (engine/features.rs:459-492): with w the
// frame's moved probe times q, per axis num = Σ Re(conj(∂O·w)·χ), den = Σ |∂O·w|²;
// sums[slot] = (num_y, num_x, den_y, den_x) in double.
static __global__ void __launch_bounds__(256) position_sums_kernel(const float2* dwin,
                                                           const float2* wave, int wave_stride,
                                                           const float2* quad,
                                                           const float2* chi, int K, int N,
                                                           double* sums) {
  __shared__ double sh[8];
  const int slot = blockIdx.x;
  const size_t plane = (size_t)N * N;
  double s[4] = {0, 0, 0, 0};
  for (int pix = threadIdx.x; pix < N * N; pix += 256) {
    const float2 w = cmul(wave[(size_t)slot * wave_stride + pix], quad[pix]);
    const float2 c = chi[(size_t)slot * K * plane + pix];
    for (int a = 0; a < 2; ++a) {
      const float2 u = cmul(dwin[((size_t)slot * 2 + a) * plane + pix], w);
      s[a] += (double)u.x * c.x + (double)u.y * c.y;
      s[2 + a] += (double)u.x * u.x + (double)u.y * u.y;
    }
  }
  for (int k = 0; k < 4; ++k) {
    double v = warp_sum(s[k]);
    if (threadIdx.x % 32 == 0) sh[threadIdx.x / 32] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < 8; ++w) t += sh[w];
      sums[(size_t)slot * 4 + k] = t;
    }
    __syncthreads();
  }
}

// pty-chi's gradient position step on the batch (engine/features.rs:496-521), one thread in
// double: delta = num/(den + max(max_batch den, eps)), dx = 0.3·delta at the batch's frames
// (0 elsewhere), each axis clipped to min(10·mean|dx − mean dx|, 0.1) over every frame.
static __global__ void position_step_kernel(const double* sums, int nslot, int nframe, double eps,
                                     const int* frames, double* offsets) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int a = 0; a < 2; ++a) {
    double mx = eps;
    for (int s = 0; s < nslot; ++s) mx = fmax(mx, sums[s * 4 + 2 + a]);
    double total = 0.0;
    for (int s = 0; s < nslot; ++s) total += 0.3 * (sums[s * 4 + a] / (sums[s * 4 + 2 + a] + mx));
    const double mean = total / nframe;
    double dev = (double)(nframe - nslot) * fabs(mean);
    for (int s = 0; s < nslot; ++s)
      dev += fabs(0.3 * (sums[s * 4 + a] / (sums[s * 4 + 2 + a] + mx)) - mean);
    const double limit = fmin(10.0 * (dev / nframe), 0.1);
    for (int s = 0; s < nslot; ++s) {
      const double dx = 0.3 * (sums[s * 4 + a] / (sums[s * 4 + 2 + a] + mx));
      offsets[2 * frames[s] + a] += fmin(fmax(dx, -limit), limit);
    }
  }
}

// Block sum of one double per thread in a fixed order (lane trees, then warps in order).
template <int T>
PTYB_D double fixed_block_sum(double v, double* sh) {
  v = warp_sum(v);
  __syncthreads();
  if (threadIdx.x % 32 == 0) sh[threadIdx.x / 32] = v;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < T / 32; ++w) s += sh[w];
  return s;
}

// The position step of AP, DM and ML on every frame (engine/features.rs:1028-1047), one block:
// per axis, with max the largest den, step = clip(0.3·num / (den + max), ±0.1) (0 where that
// denominator is not positive) and d += step − mean(step) over every frame.
static __global__ void __launch_bounds__(1024) ml_position_step_kernel(const double* sums, int nframe,
                                                               double* offsets) {
  __shared__ double sh[32];
  const int t = threadIdx.x;
  for (int a = 0; a < 2; ++a) {
    double mx = 0.0;
    for (int f = t; f < nframe; f += 1024) mx = fmax(mx, sums[(size_t)f * 4 + 2 + a]);
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    __syncthreads();
    if (t % 32 == 0) sh[t / 32] = mx;
    __syncthreads();
    mx = 0.0;
    for (int w = 0; w < 32; ++w) mx = fmax(mx, sh[w]);
    auto step = [&](int f) {
      const double den = sums[(size_t)f * 4 + 2 + a] + mx;
      return den > 0.0 ? fmin(fmax(0.3 * sums[(size_t)f * 4 + a] / den, -0.1), 0.1) : 0.0;
    };
    double part = 0.0;
    for (int f = t; f < nframe; f += 1024) part += step(f);
    const double mean = fixed_block_sum<1024>(part, sh) / nframe;
    for (int f = t; f < nframe; f += 1024) offsets[2 * f + a] += step(f) - mean;
    __syncthreads();
  }
}

}  // namespace ptyb
