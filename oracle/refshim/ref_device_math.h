// ref_device_math.h -- HOST STAND-IN (TEST INFRASTRUCTURE: the reference-pinned oracle under
// oracle/_ref), force-included before the reference's DPE.cu when it is compiled for the CPU.
//
// Device code resolves unqualified math calls with float arguments to float functions (CUDA's
// math library overloads sqrt(float), fabs(float), min(float, float) ...), where host C++ would
// promote them to double.  These overloads restore the device meanings, so the host build of the
// kernels computes in the precision the reference wrote:
//   * sqrt / sqrtf, fabs, floor, round: the IEEE float operations;
//   * rsqrtf(x): 1 / sqrtf(x), correctly rounded steps (the device's approximate reciprocal
//     square root is not restated);
//   * expf and exp(float): dpe_expf (dpe_math.h, Cody-Waite reduction + Taylor polynomial), the
//     function the CPU oracle and the CUDA kernels share, in place of the device's fast-math
//     exponential;
//   * sin / cos of a float with |a| <= 0.1 (the perturbation angles, DPE.cu:401-406): the shared
//     dpe_sincos_small; other float arguments go through the double functions;
//   * min / max: integer ones for ints, fminf / fmaxf for floats.
// Double arguments keep the C library's double functions, as on the device.
#ifndef REFSHIM_REF_DEVICE_MATH_H_
#define REFSHIM_REF_DEVICE_MATH_H_

// every standard header the reference pulls in, first, so the macros below reach only its code
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <chrono>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <random>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../dpe-mvs-fast_b200/csrc/dpe_math.h"
#include "cuda_runtime.h"

inline float sqrt(float x) { return std::sqrt(x); }
inline float fabs(float x) { return std::fabs(x); }
inline float floor(float x) { return std::floor(x); }
inline float round(float x) { return std::round(x); }
inline float rsqrtf(float x) { return 1.0f / std::sqrt(x); }
inline float ref_expf(float x) { return dpe::dpe_expf(x); }
inline float exp(float x) { return dpe::dpe_expf(x); }
inline float sin(float a) {
  if (std::fabs(a) <= 0.1f) { float s, c; dpe::dpe_sincos_small(a, &s, &c); return s; }
  return (float)std::sin((double)a);
}
inline float cos(float a) {
  if (std::fabs(a) <= 0.1f) { float s, c; dpe::dpe_sincos_small(a, &s, &c); return c; }
  return (float)std::cos((double)a);
}
inline float tan(float a) { return (float)std::tan((double)a); }
inline float pow(float x, int n) {
  float r = 1.0f;
  for (int i = 0; i < (n < 0 ? -n : n); ++i) r *= x;
  return n < 0 ? 1.0f / r : r;
}
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
inline float min(float a, float b) { return std::fmin(a, b); }
inline float max(float a, float b) { return std::fmax(a, b); }
inline bool isnan(float x) { return std::isnan(x); }
#define expf(x) ref_expf(x)

#endif
