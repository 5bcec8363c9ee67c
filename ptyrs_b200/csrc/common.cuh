// Shared device helpers: complex float2 arithmetic and compensated sums.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define PTYB_HD __host__ __device__ __forceinline__
#define PTYB_D __device__ __forceinline__

PTYB_HD float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
PTYB_HD float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
PTYB_HD float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
PTYB_HD float2 cmulc(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
PTYB_HD float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
PTYB_HD float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
PTYB_HD float cnorm2(float2 a) { return a.x * a.x + a.y * a.y; }

// Kahan-compensated accumulation of a float: sum and running compensation.
struct Kahan {
  float s, c;
  PTYB_D void init() { s = 0.f; c = 0.f; }
  PTYB_D void add(float v) {
    float y = v - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
  }
};

struct KahanC {
  Kahan re, im;
  PTYB_D void init() { re.init(); im.init(); }
  PTYB_D void add(float2 v) { re.add(v.x); im.add(v.y); }
  PTYB_D float2 value() const { return make_float2(re.s, im.s); }
};

// Bits of a non-negative float order as the float does, so an unsigned atomicMax on them is
// a float max that gives the same result in any order.
PTYB_D void atomic_max_nonneg(float* addr, float v) {
  atomicMax(reinterpret_cast<unsigned int*>(addr), __float_as_uint(fmaxf(v, 0.f)));
}

// Warp and block reductions in double.
PTYB_D double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
PTYB_D float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
