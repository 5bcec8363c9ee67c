// Shared-memory line FFTs of length N = N1·N2 (N1 ∈ {8, 16, 24}, N2 ∈ {4, 8, 16}) for sm_100a.
//
// A line lives in shared memory, N contiguous float2. G = N2 threads of one warp transform it
// in place: each thread runs an N1-point DFT in registers over a stride-N2 decimation of the
// line, applies the twiddles ω_N^{n2·k1}, exchanges through the line itself (swizzled so
// neither the writes nor the reads conflict on banks) and runs N1/N2 N2-point DFTs, writing the
// result in natural order. Forward uses e^{-2πi·nk/N}, inverse e^{+2πi·nk/N}; neither scales.
#pragma once
#include "common.cuh"

namespace ptyb {

// cos(2π·t/16) for t = 0..15.
PTYB_HD constexpr float cos16(int t) {
  switch (t & 15) {
    case 0: return 1.0f;
    case 1: case 15: return 0.92387953251128674f;
    case 2: case 14: return 0.70710678118654752f;
    case 3: case 13: return 0.38268343236508977f;
    case 4: case 12: return 0.0f;
    case 5: case 11: return -0.38268343236508977f;
    case 6: case 10: return -0.70710678118654752f;
    case 7: case 9: return -0.92387953251128674f;
    default: return -1.0f;
  }
}

// x · e^{DIR·2πi·t/R} with DIR = -1 (forward) or +1 (inverse); t and R compile-time after
// unrolling, so the trivial rotations cost no multiply.
template <int R, int DIR>
PTYB_D float2 rotate(float2 x, int t) {
  const int t16 = (t * (16 / R)) & 15;
  if (t16 == 0) return x;
  if (t16 == 8) return make_float2(-x.x, -x.y);
  if (t16 == 4) return DIR < 0 ? make_float2(x.y, -x.x) : make_float2(-x.y, x.x);
  if (t16 == 12) return DIR < 0 ? make_float2(-x.y, x.x) : make_float2(x.y, -x.x);
  const float c = cos16(t16);
  const float s = DIR * cos16(t16 + 12);  // DIR·sin(2πt/16)
  return make_float2(x.x * c - x.y * s, x.x * s + x.y * c);
}

template <int R>
PTYB_HD constexpr int bitrev(int i) {
  int r = 0;
  for (int b = 1; b < R; b <<= 1) {
    r = (r << 1) | (i & 1);
    i >>= 1;
  }
  return r;
}

// Radix-2 stages of span 2·HALF .. R of an in-register DIT DFT.
template <int R, int DIR, int HALF>
PTYB_D void dft_stages(float2 (&x)[R]) {
  if constexpr (HALF < R) {
#pragma unroll
    for (int k = 0; k < R; k += 2 * HALF) {
#pragma unroll
      for (int j = 0; j < HALF; ++j) {
        const float2 b = rotate<2 * HALF, DIR>(x[k + j + HALF], j);
        const float2 a = x[k + j];
        x[k + j] = cadd(a, b);
        x[k + j + HALF] = csub(a, b);
      }
    }
    dft_stages<R, DIR, 2 * HALF>(x);
  }
}

// cos(2π·t/24) for t = 0..23.
PTYB_HD constexpr float cos24(int t) {
  switch (((t % 24) + 24) % 24) {
    case 0: return 1.0f;
    case 1: case 23: return 0.96592582628906829f;
    case 2: case 22: return 0.86602540378443865f;
    case 3: case 21: return 0.70710678118654752f;
    case 4: case 20: return 0.5f;
    case 5: case 19: return 0.25881904510252076f;
    case 6: case 18: return 0.0f;
    case 7: case 17: return -0.25881904510252076f;
    case 8: case 16: return -0.5f;
    case 9: case 15: return -0.70710678118654752f;
    case 10: case 14: return -0.86602540378443865f;
    case 11: case 13: return -0.96592582628906829f;
    default: return -1.0f;
  }
}

// x · e^{DIR·2πi·t/24} (t compile-time after unrolling).
template <int DIR>
PTYB_D float2 rotate24(float2 x, int t) {
  if (t % 24 == 0) return x;
  const float c = cos24(t);
  const float s = DIR * cos24(t - 6);  // DIR·sin(2πt/24)
  return make_float2(x.x * c - x.y * s, x.x * s + x.y * c);
}

template <int R, int DIR>
PTYB_D void dft(float2 (&x)[R]);

// In-register DFT of 24 points as 3 × 8: with n = 3a + b and k = c + 8d,
// X[c + 8d] = Σ_b e^{DIR·2πi·bd/3}·(e^{DIR·2πi·bc/24}·Σ_a x[3a + b]·e^{DIR·2πi·ac/8}):
// three 8-point DFTs, the twiddles, then eight 3-point butterflies.
template <int DIR>
PTYB_D void dft24(float2 (&x)[24]) {
  float2 y[3][8];
#pragma unroll
  for (int b = 0; b < 3; ++b) {
#pragma unroll
    for (int a = 0; a < 8; ++a) y[b][a] = x[3 * a + b];
    dft<8, DIR>(y[b]);
#pragma unroll
    for (int c = 1; c < 8; ++c) y[b][c] = rotate24<DIR>(y[b][c], b * c);
  }
  constexpr float h3 = 0.86602540378443865f;  // sin(2π/3)
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const float2 s = cadd(y[1][c], y[2][c]), d = csub(y[1][c], y[2][c]);
    const float2 t = make_float2(y[0][c].x - 0.5f * s.x, y[0][c].y - 0.5f * s.y);
    const float2 u = make_float2(-DIR * h3 * d.y, DIR * h3 * d.x);  // DIR·i·sin(2π/3)·d
    x[c] = cadd(y[0][c], s);
    x[c + 8] = cadd(t, u);
    x[c + 16] = csub(t, u);
  }
}

// In-register DFT of R = 2, 4, 8, 16 or 24 points: x[k] ← Σ_n x[n]·e^{DIR·2πi·nk/R}.
template <int R, int DIR>
PTYB_D void dft(float2 (&x)[R]) {
  if constexpr (R == 24) {
    dft24<DIR>(x);
  } else {
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int j = bitrev<R>(i);
      if (i < j) {
        float2 t = x[i];
        x[i] = x[j];
        x[j] = t;
      }
    }
    dft_stages<R, DIR, 1>(x);
  }
}

template <int N>
struct LineShape;
template <>
struct LineShape<64> {
  static constexpr int N1 = 8, N2 = 8;
};
template <>
struct LineShape<128> {
  static constexpr int N1 = 16, N2 = 8;
};
template <>
struct LineShape<256> {
  static constexpr int N1 = 16, N2 = 16;
};
template <>
struct LineShape<96> {
  static constexpr int N1 = 24, N2 = 4;
};
template <>
struct LineShape<192> {
  static constexpr int N1 = 24, N2 = 8;
};

// Bank swizzle of a shared-memory line: element e of line `l` sits at l·N + (e ^ swz(l)).
// Consecutive lines differ in bit 3 and any 16 consecutive lines take 16 distinct values, so
// the line FFT's accesses (two to four lines per warp) and the column accesses across lines
// each hit 16 distinct 8-byte bank pairs per half-warp.
PTYB_HD int swz(int l) { return ((l & 1) << 3) | ((l >> 1) & 7); }

// The step-1 twiddles ω_N^{t·k1}, k1 = 1..N1-1, of a thread's fixed line offset t (forward
// sign; the inverse conjugates them), loaded once per thread.
template <int N>
struct LineTwiddles {
  float2 w[LineShape<N>::N1];
  PTYB_D void load(const float2* tw, int t) {
#pragma unroll
    for (int k1 = 1; k1 < LineShape<N>::N1; ++k1) w[k1] = tw[(t * k1) % N];
  }
};

// In-place FFT of one shared-memory line (swizzled by `sw`) by the G = N2 threads
// t = 0..G-1 of a warp (the whole warp calls it together).
template <int N, int DIR>
PTYB_D void line_fft(float2* line, int t, const LineTwiddles<N>& tw, int sw) {
  constexpr int N1 = LineShape<N>::N1, N2 = LineShape<N>::N2;
  constexpr int P = N1 / N2;
  float2 v[N1];
#pragma unroll
  for (int n1 = 0; n1 < N1; ++n1) v[n1] = line[(N2 * n1 + t) ^ sw];
  dft<N1, DIR>(v);
#pragma unroll
  for (int k1 = 1; k1 < N1; ++k1) v[k1] = cmul(v[k1], DIR < 0 ? tw.w[k1] : cconj(tw.w[k1]));
  __syncwarp();
#pragma unroll
  for (int k1 = 0; k1 < N1; ++k1) line[(k1 * N2 + ((t + k1) & (N2 - 1))) ^ sw] = v[k1];
  __syncwarp();
#pragma unroll
  for (int p = 0; p < P; ++p) {
    const int k1 = t + N2 * p;
    float2 u[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) u[n2] = line[(k1 * N2 + ((n2 + k1) & (N2 - 1))) ^ sw];
    dft<N2, DIR>(u);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) v[p * N2 + k2] = u[k2];
  }
  __syncwarp();
#pragma unroll
  for (int p = 0; p < P; ++p) {
    const int k1 = t + N2 * p;
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) line[(k1 + N1 * k2) ^ sw] = v[p * N2 + k2];
  }
  __syncwarp();
}

}  // namespace ptyb
