// oracle_common.h -- shared helpers of the CPU oracle (TEST INFRASTRUCTURE ONLY).
//
// The oracle is the checker for the CUDA path: only tests/, __graft_entry__.smoke() and the
// cpu_baseline leg of bench.py may load it.  It is never part of the product path.
//
// Parity status: the reference has no tests or golden vectors; the oracle restates its algorithm
// (DPE.cu, DPE.cpp) and is pinned bit for bit to the reference's own code compiled for the CPU
// (oracle/_ref, oracle/ref_harness.cpp, tests/test_ref_oracle.py).
#ifndef DPE_ORACLE_COMMON_H_
#define DPE_ORACLE_COMMON_H_

#include "../dpe-mvs-fast_b200/csrc/dpe_math.h"  // exp / sin / cos with the kernels' bits
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include "../include/dpe_b200.h"

namespace oracle {

struct f2 { float x, y; };
struct f3 { float x, y, z; };
struct f4 { float x, y, z, w; };
struct s2 { int16_t x, y; };

// OpenCV's MIN/MAX macros (cvdef.h), which the reference picks up through main.h:4-9.
// Their NaN behaviour differs from std::min/max, so they are spelled out.
template <class A, class B> static inline auto CV_MIN(A a, B b) -> decltype(a + b) { return a > b ? b : a; }
template <class A, class B> static inline auto CV_MAX(A a, B b) -> decltype(a + b) { return a < b ? b : a; }

// float -> int conversion with the semantics of the GPU (cvt.rzi.s32): truncate, NaN -> 0,
// saturate out-of-range values.  C++ leaves these cases undefined; the reference runs on a GPU.
static inline int f2i(double v) {
  if (v != v) return 0;
  if (v >= 2147483647.0) return 2147483647;
  if (v <= -2147483648.0) return (-2147483647 - 1);
  return (int)v;
}

// ---------------------------------------------------------------------------------------------
// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw, "Parallel random numbers:
// as easy as 1, 2, 3", SC'11).  Replaces the reference's XORWOW curandState seeded with
// clock64() (DPE.cu:1024-1037), which is not reproducible.
// ---------------------------------------------------------------------------------------------
static inline void philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  for (int round = 0; round < 10; ++round) {
    if (round > 0) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    c0 = hi1 ^ c1 ^ k0; c1 = lo1; c2 = hi0 ^ c3 ^ k1; c3 = lo0;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// Per-pixel stream: draw n of pixel p is word 0 of philox({n, p, 0x5EED, 0}, seed).
struct PixelRng {
  uint32_t key[2];
  uint32_t pixel;
  uint32_t *counter;
  uint32_t next_u32() {
    const uint32_t ctr[4] = {*counter, pixel, 0x5EEDu, 0u};
    uint32_t out[4];
    philox4x32_10(ctr, key, out);
    ++(*counter);
    return out[0];
  }
  // uniform float in (0, 1], the range of curand_uniform
  float uniform() { return (float)((next_u32() >> 8) + 1u) * (1.0f / 16777216.0f); }
};

}  // namespace oracle
#endif
