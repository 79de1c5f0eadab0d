// fmath.h — exp, log and pow for the render passes, written so that the same float
// operations run on the device and on the host: IEEE add/mul/div/sqrt, explicit
// fmaf, exact power-of-two scaling. The GPU passes and any host computation that
// uses these functions therefore produce identical bits.
//
// exp: Cody & Waite's argument reduction x = k ln2 + r (ln2 split in a short high
// part and a low correction, applied with fmaf), then e^r for |r| <= ln2/2 by its
// Taylor series to degree 8 (truncation error below 3e-9 relative) in Horner form,
// scaled by 2^k built from the exponent bits.
// log: x = m 2^e with m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s) with
// s = (m - 1) / (m + 1), |s| <= 0.172, by the odd series of atanh to s^13.
// pow(x, y) = exp(y log x) for x > 0 (WGSL leaves x < 0 undefined; NaN here).
#pragma once
#include <math.h>
#include <stdint.h>
#include <string.h>

#ifdef __CUDACC__
#define P4A_HD __host__ __device__ __forceinline__
#else
#define P4A_HD inline
#endif

namespace p4a {

P4A_HD float fm_bits_float(uint32_t b) {
#ifdef __CUDA_ARCH__
  return __uint_as_float(b);
#else
  float f;
  memcpy(&f, &b, 4);
  return f;
#endif
}
P4A_HD uint32_t fm_float_bits(float f) {
#ifdef __CUDA_ARCH__
  return __float_as_uint(f);
#else
  uint32_t b;
  memcpy(&b, &f, 4);
  return b;
#endif
}

// x * 2^k for a normal or zero x and any k, exact unless the result is subnormal
// (then rounded once, as IEEE multiplication rounds).
P4A_HD float fm_scale2(float x, int k) {
  while (k > 127) {
    x = x * 1.7014118346046923e38f;  // 2^127
    k -= 127;
  }
  while (k < -126) {
    x = x * 1.1754943508222875e-38f;  // 2^-126
    k += 126;
  }
  return x * fm_bits_float((uint32_t)(k + 127) << 23);
}

P4A_HD float fm_exp(float x) {
  if (x != x) return x;
  if (x > 88.72283935546875f) return INFINITY;
  if (x < -103.97208404541016f) return 0.0f;
  const float k = rintf(x * 1.44269502162933349609375f);
  float r = fmaf(-k, 0.693145751953125f, x);
  r = fmaf(-k, 1.428606765330187045e-6f, r);
  float p = 2.48015873015873e-5f;              // 1/8!
  p = fmaf(p, r, 1.984126984126984e-4f);       // 1/7!
  p = fmaf(p, r, 1.388888888888889e-3f);       // 1/6!
  p = fmaf(p, r, 8.333333333333333e-3f);       // 1/5!
  p = fmaf(p, r, 4.166666666666667e-2f);       // 1/4!
  p = fmaf(p, r, 1.666666666666667e-1f);       // 1/3!
  p = fmaf(p, r, 0.5f);
  p = fmaf(p, r, 1.0f);
  p = fmaf(p, r, 1.0f);
  return fm_scale2(p, (int)k);
}

P4A_HD float fm_log(float x) {
  if (x != x || x < 0.0f) return NAN;
  if (x == 0.0f) return -INFINITY;
  if (x == INFINITY) return x;
  int e = 0;
  if (x < 1.1754943508222875e-38f) {  // subnormal: scale into the normal range
    x = x * 16777216.0f;
    e = -24;
  }
  const uint32_t b = fm_float_bits(x);
  e += (int)((b >> 23) & 0xffu) - 127;
  float m = fm_bits_float((b & 0x7fffffu) | 0x3f800000u);
  if (m > 1.41421353816986083984375f) {
    m = m * 0.5f;
    e += 1;
  }
  const float s = (m - 1.0f) / (m + 1.0f);
  const float z = s * s;
  float p = 0.15384615384615385f;              // 2/13
  p = fmaf(p, z, 0.18181818181818182f);        // 2/11
  p = fmaf(p, z, 0.22222222222222222f);        // 2/9
  p = fmaf(p, z, 0.2857142857142857f);         // 2/7
  p = fmaf(p, z, 0.4f);                        // 2/5
  p = fmaf(p, z, 0.6666666666666666f);         // 2/3
  p = fmaf(p, z, 2.0f);
  const float fe = (float)e;
  return fmaf(fe, 0.693145751953125f, fmaf(s, p, fe * 1.428606765330187045e-6f));
}

P4A_HD float fm_pow(float x, float y) {
  if (x > 0.0f) return fm_exp(y * fm_log(x));
  if (x == 0.0f) return y > 0.0f ? 0.0f : (y == 0.0f ? 1.0f : INFINITY);
  return NAN;
}

}  // namespace p4a
