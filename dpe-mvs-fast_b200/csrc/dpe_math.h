// dpe_math.h -- elementary functions with the same bits on the host and the device.
//
// The cost kernels need exp (bilateral weights, view-sampling probabilities) and sin / cos of
// small angles (normal perturbation).  Library implementations differ between CUDA and the host
// C library by an ulp here and there, and an ulp in a window weight can flip a tie between two
// hypotheses.  These functions use only +, -, * and exact scaling, evaluated in a fixed order, so
// any build without multiply-add contraction (the exact device build, the CPU oracle) computes
// identical results; a contracting build differs by rounding only.
//
//   dpe_expf:  Cody and Waite's argument reduction (W. J. Cody, W. Waite, "Software Manual for
//              the Elementary Functions", 1980): x = n ln2 + r with |r| <= ln2 / 2, ln2 split into
//              a high part with trailing zero bits (n * ln2_hi is exact for |n| < 2^8) and a low
//              part; e^r by its Taylor polynomial to degree 7 (truncation below 6e-9 relative on
//              the reduced interval); scaled by 2^n in two exact steps so gradual underflow is
//              handled.  About 1 ulp.
//   dpe_sincos_small: Taylor series of sin and cos to degree 9 / 8, for |a| <= 0.1 (the
//              perturbation angles are at most 0.01 pi): truncation below 1e-16 relative.
#pragma once

#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define DPE_HD __host__ __device__ __forceinline__
#else
#define DPE_HD inline
#endif

namespace dpe {

DPE_HD float dpe_bits_to_float(uint32_t u) {
  float f;
  memcpy(&f, &u, 4);
  return f;
}

// Round to nearest integer, ties away from zero, for |v| < 2^22 (valid for the reduced range).
DPE_HD float dpe_round_small(float v) {
  const float h = v < 0.0f ? -0.5f : 0.5f;
  return (float)(int)(v + h);
}

DPE_HD float dpe_expf(float x) {
  if (!(x == x)) return x;                    // NaN
  if (x > 88.7f) return dpe_bits_to_float(0x7f800000u);  // overflow: +inf
  if (x < -104.0f) return 0.0f;                // below the smallest denormal
  const float kLog2e = 1.44269502162933349609375f;
  const float kLn2Hi = 0.693145751953125f;     // 0x3f317200: 15 significant bits
  const float kLn2Lo = 1.428606765330187045e-06f;
  const float n = dpe_round_small(x * kLog2e);
  const float r = (x - n * kLn2Hi) - n * kLn2Lo;
  // e^r = 1 + r + r^2/2! + ... + r^7/7!, Horner
  float p = 1.0f / 5040.0f;
  p = p * r + 1.0f / 720.0f;
  p = p * r + 1.0f / 120.0f;
  p = p * r + 1.0f / 24.0f;
  p = p * r + 1.0f / 6.0f;
  p = p * r + 0.5f;
  p = p * r + 1.0f;
  p = p * r + 1.0f;
  // p * 2^n, in two exact power-of-two steps (each factor a normal float)
  const int ni = (int)n;
  const int n1 = ni / 2, n2 = ni - n1;
  const float s1 = dpe_bits_to_float((uint32_t)(n1 + 127) << 23);
  const float s2 = dpe_bits_to_float((uint32_t)(n2 + 127) << 23);
  return (p * s1) * s2;
}

DPE_HD void dpe_sincos_small(float a, float *s, float *c) {
  const float a2 = a * a;
  float ps = 1.0f / 362880.0f;  // sin: a (1 - a^2/3! + a^4/5! - a^6/7! + a^8/9!)
  ps = ps * a2 - 1.0f / 5040.0f;
  ps = ps * a2 + 1.0f / 120.0f;
  ps = ps * a2 - 1.0f / 6.0f;
  ps = ps * a2 + 1.0f;
  *s = ps * a;
  float pc = 1.0f / 40320.0f;   // cos: 1 - a^2/2! + a^4/4! - a^6/6! + a^8/8!
  pc = pc * a2 - 1.0f / 720.0f;
  pc = pc * a2 + 1.0f / 24.0f;
  pc = pc * a2 - 0.5f;
  *c = pc * a2 + 1.0f;
}

}  // namespace dpe
