// dpe_device.cuh -- device-side building blocks of the sm_100a PatchMatch kernels.
//
// Geometry and cost functions restate the reference's device helpers (DPE.cu:9-957) in FP32
// without fast-math; the per-pixel reference window of the strong NCC is hoisted out of the
// hypothesis loop (weights and reference moments do not depend on the plane).
#pragma once

#include <cfloat>
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "../../include/dpe_b200.h"
#include "dpe_math.h"
#include "kernel_ids.h"

namespace dpe {

constexpr int kMaxImages = DPE_MAX_IMAGES;
constexpr int kMaxSrc = DPE_MAX_IMAGES - 1;
constexpr int kNeighbours = DPE_NEIGHBOUR_NUM;
constexpr int kMaxWin = 6;  // taps per window side for radius 5 / step 2 (DPE.cu:728-737)
// Minimum resident blocks per multiprocessor requested for the strong-window cost kernels
// (__launch_bounds__): bounds their registers, trading spills against occupancy.  Measured on
// the 10-view 1600x1200 schedule: the cooperative strong update runs fastest at 8 blocks of 128
// (64 registers; 2 % faster than 6 blocks at 80), the sweep kernels unconstrained.
#ifndef DPE_COST_MIN_BLOCKS
#define DPE_COST_MIN_BLOCKS 1
#endif
#ifndef DPE_STRONG_MIN_BLOCKS
#define DPE_STRONG_MIN_BLOCKS 8
#endif
// the same bound for the cooperative DepthToWeak sweep (measured: 8 blocks, 64 registers, 4 %
// faster than unbounded; the cooperative LocalRefine, with its larger shared-memory block, runs
// fastest unbounded and uses DPE_COST_MIN_BLOCKS)
#ifndef DPE_SWEEP_MIN_BLOCKS
#define DPE_SWEEP_MIN_BLOCKS 8
#endif
// Unrolling of a window column's taps (the reference window, radius 5 / step 2, has 6 per column)
// in the kernels that sweep one plane family over all sources (DepthToWeak, LocalRefine, the
// random initialisation).  Measured on the 10-view 1600x1200 schedule with the packed tap
// arithmetic: the whole column (6) makes DepthToWeak 6 % and LocalRefine 7 % faster than 3, and 2
// is slower than 3.
#ifndef DPE_SWEEP_UNROLL
#define DPE_SWEEP_UNROLL 6
#endif
constexpr int kSweepUnroll = DPE_SWEEP_UNROLL;
// taps of a window column unrolled in the strong update's cost evaluations (0: rolled loop).
// Measured on the 10-view 1600x1200 schedule with the packed tap arithmetic: unrolling by 2 makes
// the cooperative strong update 5 % faster (the next tap's gathers issue before this tap's blend);
// by 3 or 6 it was 35-40 % slower with the scalar taps (registers, under the 8-block bound).
#ifndef DPE_STRONG_UNROLL
#define DPE_STRONG_UNROLL 2
#endif
constexpr int kStrongUnroll = DPE_STRONG_UNROLL;

// All per-call read-only data (cameras, relative poses, params, buffer pointers).  It lives in a
// small device buffer written once per call; kernels receive its address.
struct PMArgs {
  int W, H, N, lowW, lowH, pad_w;  // pad_w = W + 2 (images carry a 1-texel clamp border)
  dpe_params P;
  dpe_camera cam[kMaxImages];
  // Plane-independent parts of each source's homography H = A - b m^T / w (homography_base):
  // composed in double (window centres are projected in double), and the same rounded to float.
  double dA[kMaxImages][9], db[kMaxImages][3], dm[4];
  float hA[kMaxImages][9], hb[kMaxImages][3], hm[4];
  uint32_t key[2];
  const float *img[kMaxImages];  // padded (W+2)*(H+2) float images
  // Staged source images (dpe_options::staging FP16 / BF16): pair[s][o] holds the padded texels
  // P[o] and P[o+1] as two 16-bit values in one 32-bit word, so a bilinear footprint is two loads.
  const uint32_t *pair[kMaxImages];
  int stage;  // DPE_STAGE_*: storage the cost kernels sample the source images from
  int gn;     // 1: Gauss-Newton plane hypothesis in the strong update (dpe_options::gn_refine)
  const float *dep[kMaxImages];  // W*H depth maps (geom consistency)
  // state
  float4 *plane;
  float4 *plane_snap;
  float4 *fit_plane;
  float *cost;
  float *cost_snap;
  float *complexity;
  uint32_t *views;
  uint32_t *rng_ctr;
  uint4 *vweight;          // 32 4-bit sample counts per pixel
  uint8_t *weak;
  uint8_t *reliable;
  const uint8_t *edge;
  const uint8_t *edge_low;
  const int32_t *label;
  int32_t *nmap;
  int32_t *radius;
  short2 *neigh;
  short2 *lab_bound;
  short2 *edge_neigh;
  short2 *nearest;
  unsigned long long *counters;  // per kernel class: [2k] strong NCC evals, [2k+1] weak (counting runs)
  // Weak-texture pass.  The WEAK pixels of each colour are listed once per call (wlist, wcount,
  // raster order); a listed pixel's position in its list is its slot in the scratch below, which
  // every colour pass reuses.
  const int *wlist[2];
  const int *wcount;  // [2]
  int wtab_stride;    // table entries per slot: kMaxWin^2 for the centre window + 8 deformable windows
  int wtaps;          // taps of one deformable window
  float2 *wtab;       // [slot][tap] bilateral weight w and w * (r - c) of every window tap
  float4 *wwin;       // [slot][9] reference sums (s_w, s_r, s_rr) of each window
  float *wcost;       // [slot][10][N-1] deformable NCC: 8 candidates, the current plane, the fit plane
  float *wgeom;       // [slot][10][N-1] geometric cost of the same hypotheses
  float4 *whyp;       // [slot][5] random refinement hypotheses
  float *wcost_r;     // [slot][5][N-1] deformable NCC of the random hypotheses
  float *wgeom_r;     // [slot][5][N-1] geometric cost of the random hypotheses
  float4 *wstate;     // [slot][2] plane after the candidate and fit-plane steps; (depth, cost, cost0, wn)
};

// Plane-independent parts of the homography of source camera sc with respect to the reference
// camera rc (DPE.cu:457-517).  H = Ks (Rrel - trel n^T / w) Kr^-1 is written as A - b m^T / w with
//   A = Ks Rrel Kr^-1,  b = Ks trel,  m = Kr^-T n = (nx / fx, ny / fy, nz - nx cx / fx - ny cy / fy),
// Rrel = Rs Rr^T, trel = Rs (Cr - Cs) and camera centres C = -R^T t.  A, b and the entries of
// Kr^-1 (m = (1/fx, 1/fy, -cx/fx, -cy/fy) here) are composed once per call on the host in double.
// The reference composes the same products in float per hypothesis; the float rounding of the
// camera products moves the entries of H by a few ulps, which at source coordinates of ~2000 px
// places a window ~1e-4 px off.
inline void homography_base(const dpe_camera &rc, const dpe_camera &sc, double A[9], double b[3], double m[4]) {
  double rC[3], sC[3], Rr[9], Cr[3], tr[3], MK[9];
  for (int k = 0; k < 3; ++k) {
    rC[k] = -((double)rc.R[k] * rc.t[0] + (double)rc.R[3 + k] * rc.t[1] + (double)rc.R[6 + k] * rc.t[2]);
    sC[k] = -((double)sc.R[k] * sc.t[0] + (double)sc.R[3 + k] * sc.t[1] + (double)sc.R[6 + k] * sc.t[2]);
  }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      Rr[3 * i + j] = (double)sc.R[3 * i] * rc.R[3 * j] + (double)sc.R[3 * i + 1] * rc.R[3 * j + 1] +
                      (double)sc.R[3 * i + 2] * rc.R[3 * j + 2];
  for (int k = 0; k < 3; ++k) Cr[k] = rC[k] - sC[k];
  for (int i = 0; i < 3; ++i)
    tr[i] = (double)sc.R[3 * i] * Cr[0] + (double)sc.R[3 * i + 1] * Cr[1] + (double)sc.R[3 * i + 2] * Cr[2];
  m[0] = 1.0 / rc.K[0];
  m[1] = 1.0 / rc.K[4];
  m[2] = -(double)rc.K[2] / rc.K[0];
  m[3] = -(double)rc.K[5] / rc.K[4];
  for (int i = 0; i < 3; ++i) {
    MK[3 * i] = Rr[3 * i] * m[0];
    MK[3 * i + 1] = Rr[3 * i + 1] * m[1];
    MK[3 * i + 2] = Rr[3 * i] * m[2] + Rr[3 * i + 1] * m[3] + Rr[3 * i + 2];
  }
  for (int j = 0; j < 3; ++j) {
    A[j] = (double)sc.K[0] * MK[j] + (double)sc.K[2] * MK[6 + j];
    A[3 + j] = (double)sc.K[4] * MK[3 + j] + (double)sc.K[5] * MK[6 + j];
    A[6 + j] = (double)sc.K[8] * MK[6 + j];
  }
  b[0] = (double)sc.K[0] * tr[0] + (double)sc.K[2] * tr[2];
  b[1] = (double)sc.K[4] * tr[1] + (double)sc.K[5] * tr[2];
  b[2] = (double)sc.K[8] * tr[2];
}
// Fills the homography bases of every source of a call (cameras already in a.cam).
inline void set_homography_bases(PMArgs &a) {
  for (int s = 1; s < a.N; ++s) {
    homography_base(a.cam[0], a.cam[s], a.dA[s], a.db[s], a.dm);
    for (int k = 0; k < 9; ++k) a.hA[s][k] = (float)a.dA[s][k];
    for (int k = 0; k < 3; ++k) a.hb[s][k] = (float)a.db[s][k];
  }
  for (int k = 0; k < 4; ++k) a.hm[k] = (float)a.dm[k];
}

// ------------------------------------------------------------------ checked builds
// With -DDPE_CHECKED every global access of the PatchMatch kernels goes through G(): an index
// outside [0, n) is recorded in g_oob (first hit: tag, index, bound; plus a hit count) and
// redirected to element 0, so a bad index is reported instead of faulting.
#ifdef DPE_CHECKED
__device__ long long g_oob[4];
template <class T> __device__ __forceinline__ T *dpe_chk(T *base, long long idx, long long n, int tag) {
  if (idx < 0 || idx >= n) {
    if (atomicAdd((unsigned long long *)&g_oob[3], 1ull) == 0ull) {
      g_oob[0] = tag; g_oob[1] = idx; g_oob[2] = n;
    }
    idx = 0;
  }
  return base + idx;
}
#define G(arr, idx, n, tag) (*::dpe::dpe_chk(&(arr)[0], (long long)(idx), (long long)(n), (tag)))
#else
#define G(arr, idx, n, tag) ((arr)[idx])
#endif

// ------------------------------------------------------------------ OpenCV MIN/MAX semantics
template <class A, class B> __device__ __forceinline__ auto cvmin(A a, B b) -> decltype(a + b) { return a > b ? b : a; }
template <class A, class B> __device__ __forceinline__ auto cvmax(A a, B b) -> decltype(a + b) { return a < b ? b : a; }

__device__ __forceinline__ int isSet(uint32_t v, int n) { return (v >> n) & 1; }
__device__ __forceinline__ void setBit(uint32_t *v, int n) { *v |= (1u << n); }
__device__ __forceinline__ void unSetBit(uint32_t *v, int n) { *v &= (0xFFFFFFFEu << n); }

// ------------------------------------------------------------------ Philox4x32-10
// Salmon et al., SC'11.  Draw n of pixel p is word 0 of philox({n, p, 0x5EED, 0}, key).
__device__ __forceinline__ uint32_t philox_word0(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                                 uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r > 0) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
    const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
  }
  return c0;
}
__device__ __forceinline__ void philox4(const uint32_t ci[4], const uint32_t ki[2], uint32_t out[4]) {
  uint32_t c0 = ci[0], c1 = ci[1], c2 = ci[2], c3 = ci[3], k0 = ki[0], k1 = ki[1];
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r > 0) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
    const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// Per-pixel random stream; the counter lives in a register and is written back by the owner.
struct Rng {
  uint32_t k0, k1, pixel, ctr;
  __device__ __forceinline__ uint32_t u32() { return philox_word0(ctr++, pixel, 0x5EEDu, 0u, k0, k1); }
  __device__ __forceinline__ float uniform() { return (float)((u32() >> 8) + 1u) * (1.0f / 16777216.0f); }
};
__device__ __forceinline__ Rng make_rng(const PMArgs &a, int center) {
  return Rng{a.key[0], a.key[1], (uint32_t)center, G(a.rng_ctr, center, (long long)a.W * a.H, 106)};
}

// ------------------------------------------------------------------ image access
__device__ __forceinline__ float img_ld(const float *img, long long off, long long n, int tag) {
#ifdef DPE_CHECKED
  return *dpe_chk(img, off, n, tag);
#else
  return __ldg(img + off);
#endif
}
__device__ __forceinline__ float texel(const PMArgs &a, int im, int x, int y) {
  x = min(max(x, 0), a.W - 1);
  y = min(max(y, 0), a.H - 1);
  return img_ld(a.img[im], (long long)(y + 1) * a.pad_w + (x + 1), (long long)a.pad_w * (a.H + 2), 101);
}
// floor(x) as a float and as an int, for -1 <= x < 2^22 (a clamped sample coordinate).  On the
// device, x + 1.5 * 2^23 rounded toward -inf is exactly 1.5 * 2^23 + floor(x): the sum lies in
// [2^23, 2^24), where float spacing is 1.  So the floor is one FADD with a rounding mode on the FMA
// pipe, and the int is an integer subtract, instead of a round and a float-to-int conversion on the
// conversion pipe (16 per clock per SM, the bound of the tap loops).  Same value as floorf.
__device__ __forceinline__ float floor_split(float x, int *ix) {
#ifdef __CUDA_ARCH__
  const float f = __fadd_rd(x, 12582912.0f);
  *ix = __float_as_int(f) - 0x4B400000;
  return f - 12582912.0f;
#else
  const float f = floorf(x);
  *ix = (int)f;
  return f;
#endif
}

// Packed pairs of FP32 operations: on sm_100 one FADD2 / FMUL2 instruction performs two IEEE
// round-to-nearest (or, for the round-down add, round-down) operations, with exactly the results
// of the two scalar operations; the tap loops are bound by instruction issue, and pairing the x and
// y coordinates (and the two bilinear rows) cuts their arithmetic instructions.  One rule keeps the
// results exact: a packed add never takes a packed product as an operand.  Measured on the B200,
// the compiler turns add2(mul2(a, b), mul2(c, d)) into a fused multiply-add pair even without
// contraction (-fmad=false), which rounds once instead of twice; products are therefore summed
// with scalar adds.  Host builds of this source use the scalar forms.
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  return __fadd2_rn(a, b);
#else
  return make_float2(a.x + b.x, a.y + b.y);
#endif
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return add2(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  return __fmul2_rn(a, b);
#else
  return make_float2(a.x * b.x, a.y * b.y);
#endif
}
// floor_split of both coordinates of a pair.
__device__ __forceinline__ float2 floor_split2(float2 v, int *ix, int *iy) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  const float2 f = __fadd2_rd(v, make_float2(12582912.0f, 12582912.0f));
  *ix = __float_as_int(f.x) - 0x4B400000;
  *iy = __float_as_int(f.y) - 0x4B400000;
  return add2(f, make_float2(-12582912.0f, -12582912.0f));
#else
  return make_float2(floor_split(v.x, ix), floor_split(v.y, iy));
#endif
}

// tex2D(x+0.5, y+0.5) with linear filtering and clamp-to-edge addressing, exact FP32 weights.
// The padded border makes the four reads branch-free for x0 in [-1, W-1].
__device__ __forceinline__ float bilinear(const float *__restrict__ img, int pad_w, int W, int H, float x, float y) {
  const float xc = fminf(fmaxf(x, -1.0f), (float)(W - 1));
  const float yc = fminf(fmaxf(y, -1.0f), (float)(H - 1));
  int ix, iy;
  const float fx = floor_split(xc, &ix), fy = floor_split(yc, &iy);
  const float ax = xc - fx, ay = yc - fy;
  const long long o = (long long)(iy + 1) * pad_w + (ix + 1);
  const long long n = (long long)pad_w * (H + 2);
  const float v00 = img_ld(img, o, n, 102), v10 = img_ld(img, o + 1, n, 103);
  const float v01 = img_ld(img, o + pad_w, n, 104), v11 = img_ld(img, o + pad_w + 1, n, 105);
  const float top = (1.0f - ax) * v00 + ax * v10;
  const float bot = (1.0f - ax) * v01 + ax * v11;
  return (1.0f - ay) * top + ay * bot;
}
// ------------------------------------------------------------------ source samplers
// A source image as the cost kernels sample it.  fetch(o) returns the 2x2 texel footprint of
// padded offset o, (P[o], P[o+1], P[o+pw], P[o+pw+1]), in FP32; the interpolation is shared, so
// samplers differ only in storage.  FP32 samples equal bilinear() above exactly.
struct SrcF32 {
  const float *p;
  int pw;
  long long n;
  __device__ __forceinline__ float4 fetch(int o) const {
    return make_float4(img_ld(p, o, n, 102), img_ld(p, o + 1, n, 103), img_ld(p, o + pw, n, 104),
                       img_ld(p, o + pw + 1, n, 105));
  }
};
__device__ __forceinline__ uint32_t pair_ld(const uint32_t *p, long long off, long long n, int tag) {
#ifdef DPE_CHECKED
  return *dpe_chk(p, off, n, tag);
#else
  return __ldg(p + off);
#endif
}
// FP16 pairs: low half P[o], high half P[o+1].
struct SrcF16 {
  const uint32_t *p;
  int pw;
  long long n;
  __device__ __forceinline__ float4 fetch(int o) const {
    const uint32_t t = pair_ld(p, o, n, 108), b = pair_ld(p, o + pw, n, 109);
    return make_float4(__half2float(__ushort_as_half((unsigned short)(t & 0xFFFFu))),
                       __half2float(__ushort_as_half((unsigned short)(t >> 16))),
                       __half2float(__ushort_as_half((unsigned short)(b & 0xFFFFu))),
                       __half2float(__ushort_as_half((unsigned short)(b >> 16))));
  }
};
// BF16 pairs: a bfloat16 is the top half of an FP32 word, so widening is a shift.
struct SrcBF16 {
  const uint32_t *p;
  int pw;
  long long n;
  __device__ __forceinline__ float4 fetch(int o) const {
    const uint32_t t = pair_ld(p, o, n, 110), b = pair_ld(p, o + pw, n, 111);
    return make_float4(__uint_as_float(t << 16), __uint_as_float(t & 0xFFFF0000u), __uint_as_float(b << 16),
                       __uint_as_float(b & 0xFFFF0000u));
  }
};
// kClamp = false: the caller knows -1 <= x <= W-1 and -1 <= y <= H-1, where the clamp is the
// identity.
template <class Src, bool kClamp = true>
__device__ __forceinline__ float bilinear_s(const Src &src, int W, int H, float x, float y) {
  const float2 c = kClamp ? make_float2(fminf(fmaxf(x, -1.0f), (float)(W - 1)), fminf(fmaxf(y, -1.0f), (float)(H - 1)))
                          : make_float2(x, y);
  int ix, iy;
  const float2 f = floor_split2(c, &ix, &iy);
  const float2 a = sub2(c, f);                            // (ax, ay)
  const float2 oa = sub2(make_float2(1.0f, 1.0f), a);     // (1 - ax, 1 - ay)
  const float4 v = src.fetch((iy + 1) * src.pw + (ix + 1));
  // (top, bot) = (1 - ax) (v00, v01) + ax (v10, v11); then (1 - ay) top + ay bot; products are
  // summed with scalar adds (see add2)
  const float2 l = mul2(make_float2(oa.x, oa.x), make_float2(v.x, v.z));
  const float2 rt = mul2(make_float2(a.x, a.x), make_float2(v.y, v.w));
  const float2 r = mul2(make_float2(oa.y, a.y), make_float2(l.x + rt.x, l.y + rt.y));
  return r.x + r.y;
}
__device__ __forceinline__ SrcF32 src_f32(const PMArgs &a, int s) {
  return SrcF32{a.img[s], a.pad_w, (long long)a.pad_w * (a.H + 2)};
}
__device__ __forceinline__ SrcF16 src_f16(const PMArgs &a, int s) {
  return SrcF16{a.pair[s], a.pad_w, (long long)a.pad_w * (a.H + 2)};
}
__device__ __forceinline__ SrcBF16 src_bf16(const PMArgs &a, int s) {
  return SrcBF16{a.pair[s], a.pad_w, (long long)a.pad_w * (a.H + 2)};
}
// The sampler of a staging (DPE_STAGE_*), chosen at compile time: each cost kernel is built once
// per staging, so a kernel carries only its own tap loop.
template <int kStage> struct SrcOf;
template <> struct SrcOf<DPE_STAGE_FP32> {
  static __device__ __forceinline__ SrcF32 make(const PMArgs &a, int s) { return src_f32(a, s); }
};
template <> struct SrcOf<DPE_STAGE_FP16> {
  static __device__ __forceinline__ SrcF16 make(const PMArgs &a, int s) { return src_f16(a, s); }
};
template <> struct SrcOf<DPE_STAGE_BF16> {
  static __device__ __forceinline__ SrcBF16 make(const PMArgs &a, int s) { return src_bf16(a, s); }
};

// ------------------------------------------------------------------ geometry (DPE.cu:313-546)
__device__ __forceinline__ void point3d(const dpe_camera &c, int x, int y, float depth, float X[3]) {
  X[0] = depth * ((float)x - c.K[2]) / c.K[0];
  X[1] = depth * ((float)y - c.K[5]) / c.K[4];
  X[2] = depth;
}
__device__ __forceinline__ float4 view_direction(const dpe_camera &c, int x, int y, float depth) {
  float X[3];
  point3d(c, x, y, depth, X);
  const float norm = sqrtf(X[0] * X[0] + X[1] * X[1] + X[2] * X[2]);
  return make_float4(X[0] / norm, X[1] / norm, X[2] / norm, 0.0f);
}
__device__ __forceinline__ float dist_to_origin(const dpe_camera &c, int x, int y, float depth, float4 n) {
  float X[3];
  point3d(c, x, y, depth, X);
  return -(n.x * X[0] + n.y * X[1] + n.z * X[2]);
}
__device__ __forceinline__ float depth_from_plane(const dpe_camera &c, float4 pl, int x, int y) {
  return -pl.w * c.K[0] /
         (((float)x - c.K[2]) * pl.x + (c.K[0] / c.K[4]) * ((float)y - c.K[5]) * pl.y + c.K[0] * pl.z);
}
__device__ __forceinline__ float4 normal_to_world(const dpe_camera &c, float4 p) {
  return make_float4(c.R[0] * p.x + c.R[3] * p.y + c.R[6] * p.z, c.R[1] * p.x + c.R[4] * p.y + c.R[7] * p.z,
                     c.R[2] * p.x + c.R[5] * p.y + c.R[8] * p.z, p.w);
}
__device__ __forceinline__ float4 normal_to_ref(const dpe_camera &c, float4 p) {
  return make_float4(c.R[0] * p.x + c.R[1] * p.y + c.R[2] * p.z, c.R[3] * p.x + c.R[4] * p.y + c.R[5] * p.z,
                     c.R[6] * p.x + c.R[7] * p.y + c.R[8] * p.z, p.w);
}
__device__ __forceinline__ void normalize3(float4 *v) {
  const float inv = 1.0f / sqrtf(v->x * v->x + v->y * v->y + v->z * v->z);
  v->x *= inv; v->y *= inv; v->z *= inv;
}
__device__ __forceinline__ void normalize3(float3 *v) {
  const float inv = 1.0f / sqrtf(v->x * v->x + v->y * v->y + v->z * v->z);
  v->x *= inv; v->y *= inv; v->z *= inv;
}
__device__ __forceinline__ void normalize2(float2 *v) {
  const float inv = 1.0f / sqrtf(v->x * v->x + v->y * v->y);
  v->x *= inv; v->y *= inv;
}

// Marsaglia sphere point facing the camera (DPE.cu:365-391); rejection capped at 64 tries.
__device__ __forceinline__ float4 random_normal(const dpe_camera &c, int x, int y, Rng &rng, float depth) {
  float q1 = 1.0f, q2 = 1.0f, s = 2.0f;
  for (int tries = 0; s >= 1.0f && tries < 64; ++tries) {
    q1 = 2.0f * rng.uniform() - 1.0f;
    q2 = 2.0f * rng.uniform() - 1.0f;
    s = q1 * q1 + q2 * q2;
  }
  const float sq = sqrtf(fmaxf(1.0f - s, 0.0f));
  float4 n = make_float4(2.0f * q1 * sq, 2.0f * q2 * sq, 1.0f - 2.0f * s, 0.0f);
  const float4 v = view_direction(c, x, y, depth);
  if (n.x * v.x + n.y * v.y + n.z * v.z > 0.0f) { n.x = -n.x; n.y = -n.y; n.z = -n.z; }
  normalize3(&n);
  return n;
}

// Euler-angle perturbation (DPE.cu:393-428)
__device__ __forceinline__ float4 perturbed_normal(const dpe_camera &c, int x, int y, float4 n, Rng &rng, float pert) {
  const float4 v = view_direction(c, x, y, 1.0f);
  const float a1 = (rng.uniform() - 0.5f) * pert;
  const float a2 = (rng.uniform() - 0.5f) * pert;
  const float a3 = (rng.uniform() - 0.5f) * pert;
  float s1, s2, s3, c1, c2, c3;
  dpe_sincos_small(a1, &s1, &c1);  // |a| <= 0.01 pi
  dpe_sincos_small(a2, &s2, &c2);
  dpe_sincos_small(a3, &s3, &c3);
  const float R0 = c2 * c3, R1 = c3 * s1 * s2 - c1 * s3, R2 = s1 * s3 + c1 * c3 * s2;
  const float R3 = c2 * s3, R4 = c1 * c3 + s1 * s2 * s3, R5 = c1 * s2 * s3 - c3 * s1;
  const float R6 = -s2, R7 = c2 * s1, R8 = c1 * c2;
  float4 r = make_float4(R0 * n.x + R1 * n.y + R2 * n.z, R3 * n.x + R4 * n.y + R5 * n.z, R6 * n.x + R7 * n.y + R8 * n.z, n.w);
  if (r.x * v.x + r.y * v.y + r.z * v.z >= 0.0f) r = n;
  normalize3(&r);
  return r;
}

// Homography of a reference-camera plane into source `s` (DPE.cu:457-517) in float, from the
// per-call bases: H = A - (b / w) m^T with m = (nx / fx, ny / fy, nz - nx cx / fx - ny cy / fy).
__device__ __forceinline__ void homography(const PMArgs &a, int s, float4 pl, float H[9]) {
  const float m[3] = {pl.x * a.hm[0], pl.y * a.hm[1], pl.x * a.hm[2] + pl.y * a.hm[3] + pl.z};
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const float bi = a.hb[s][i] / pl.w;
#pragma unroll
    for (int j = 0; j < 3; ++j) H[3 * i + j] = a.hA[s][3 * i + j] - bi * m[j];
  }
}
__device__ __forceinline__ float2 project(const float H[9], int x, int y) {
  const float fx = (float)x, fy = (float)y;
  const float X = H[0] * fx + H[1] * fy + H[2];
  const float Y = H[3] * fx + H[4] * fy + H[5];
  const float Z = H[6] * fx + H[7] * fy + H[8];
  return make_float2(X / Z, Y / Z);
}
// project() at a tap of a deformable window, float coordinates.  The fast device build divides by
// the hardware reciprocal (as the strong window's taps do); the exact build and host builds keep
// the IEEE quotients X / Z and Y / Z.
__device__ __forceinline__ float tap_rcp(float z);
__device__ __forceinline__ float2 project_tap(const float H[9], float fx, float fy) {
  const float2 px = mul2(make_float2(H[0], H[3]), make_float2(fx, fx));
  const float2 py = mul2(make_float2(H[1], H[4]), make_float2(fy, fy));
  const float X = px.x + py.x + H[2];
  const float Y = px.y + py.y + H[5];
  const float Z = H[6] * fx + H[7] * fy + H[8];
#if defined(__CUDA_ARCH__) && !defined(DPE_EXACT)
  const float iz = tap_rcp(Z);
  return mul2(make_float2(X, Y), make_float2(iz, iz));
#else
  return make_float2(X / Z, Y / Z);
#endif
}

__device__ __forceinline__ float bilateral_weight(float dx, float dy, float pix, float center, float ss, float sc) {
  const float spatial = sqrtf(dx * dx + dy * dy);
  const float color = fabsf(pix - center);
  return dpe_expf(-spatial / (2.0f * ss * ss) - color / (2.0f * sc * sc));
}

// ------------------------------------------------------------------ strong NCC
// The weighted moments are accumulated on intensities shifted by the window's reference centre
// value c (r - c, s - c).  Variance and covariance are shift invariant, so the cost is the
// reference's; the shift removes the cancellation of E[x^2] - E[x]^2 at mean ~128-200 that costs
// FP32 about 1e-4 on low-contrast windows (the compensated form).

// Hypothesis-invariant part of the strong window of one pixel: per tap the bilateral weight w and
// w*(r - c), plus the normalised reference moments.  The per-tap arrays live in the thread's
// local memory, which L1 serves well here.  (A block-shared copy measured slower: 36 KB of static
// shared memory per block cuts the resident blocks and the L1 left for the image gathers.)
constexpr int kWinTaps = kMaxWin * kMaxWin;
struct RefWindow {
  float2 t_[kWinTaps];  // per tap (w, w * (r - c)): one 8-byte load per tap
  float center, inv_wsum, mean_r, var_r;
  unsigned long long *cnt;  // this kernel's strong-evaluation counter (counting runs only)
  __device__ __forceinline__ float2 tap(int k) const { return G(t_, k, kWinTaps, 322); }
  __device__ __forceinline__ float w(int k) const { return tap(k).x; }
  __device__ __forceinline__ float wr(int k) const { return tap(k).y; }
};
#define DPE_REF_WINDOW(rw) ::dpe::RefWindow rw
// The same window held once per pixel in shared memory, read by every thread that evaluates a
// hypothesis of that pixel (the cooperative strong update).  The threads of one pixel read the
// same tap together, so a warp's read is one broadcast per pixel.
struct SmemWindow {
  const float2 *t_;
  float center, inv_wsum, mean_r, var_r;
  unsigned long long *cnt;
  __device__ __forceinline__ float2 tap(int k) const { return t_[k]; }
  __device__ __forceinline__ float w(int k) const { return t_[k].x; }
  __device__ __forceinline__ float wr(int k) const { return t_[k].y; }
};

__device__ __forceinline__ void build_ref_window(const PMArgs &a, int px, int py, RefWindow &rw, int kid) {
  rw.cnt = a.counters ? a.counters + 2 * kid : nullptr;
  const int r = a.P.strong_radius, inc = a.P.strong_increment;
  const float center = texel(a, 0, px, py);
  float sw = 0.f, swr = 0.f, swrr = 0.f;
  int k = 0;
  for (int i = -r; i <= r; i += inc) {
    for (int j = -r; j <= r; j += inc) {
      const float rp = texel(a, 0, px + i, py + j);
      const float w = bilateral_weight((float)i, (float)j, rp, center, a.P.sigma_spatial, a.P.sigma_color);
      const float rc = rp - center;
      G(rw.t_, k, kWinTaps, 320) = make_float2(w, w * rc);
      sw += w; swr += w * rc; swrr += w * rc * rc;
      ++k;
    }
  }
  rw.center = center;
  rw.inv_wsum = 1.0f / sw;
  rw.mean_r = swr * rw.inv_wsum;
  rw.var_r = swrr * rw.inv_wsum - rw.mean_r * rw.mean_r;
}

// Reciprocal of a tap's projective depth.  The fast device build uses the hardware reciprocal
// (rcp.approx.ftz, within 1 ulp of 1/z; the perspective divide only places the bilinear sample,
// so the difference is far inside the NCC's 1e-4 bar).  The exact build (DPE_EXACT) and host
// builds of this source keep the IEEE quotient.
__device__ __forceinline__ float tap_rcp(float z) {
#if defined(__CUDA_ARCH__) && !defined(DPE_EXACT)
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(z));
  return r;
#else
  return 1.0f / z;
#endif
}
// Projection of one strong window into source s.  The window centre p0 = (px, py) goes through
// the homography in double, from the double bases: in float, the rounding of the homography's
// entries and of the numerators at source coordinates of ~2000 px places the whole window up to
// ~1e-4 px off, and on low-contrast windows the NCC moves by about as much.  The centre is kept
// as an integer texel (U0, V0) plus a float fraction, and each tap p0 + (dx, dy) as a float
// offset from it:
//   u(p0 + d) - uc = ((H00 - uc H20) dx + (H01 - uc H21) dy) / (Zc + H20 dx + H21 dy),
// whose terms are small, so float arithmetic places the taps to ~1e-6 px.  The plane enters in
// double too; the per-tap arithmetic is float.
struct WinProj {
  int U0, V0;   // integer part of the projected centre
  float2 fuv;   // its fraction (fu, fv), in [0, 1]
  float2 g03;   // the dx coefficients (H00 - uc H20, H10 - vc H20)
  float2 g14;   // the dy coefficients (H01 - uc H21, H11 - vc H21)
  float zc;     // projective depth of the centre
  float h6, h7; // H20, H21
  float2 lo, hi;  // the texture clamp [-1, W-1] x [-1, H-1] relative to (U0, V0)
};
// Fills wp for plane pl at pixel (px, py) of source s; false when the centre does not project
// inside the source (the cost is then 2, DPE.cu:709-712).
__device__ __forceinline__ bool window_projection(const PMArgs &a, int s, float4 pl, int px, int py, WinProj &wp) {
  const double *A = a.dA[s], *b = a.db[s];
  const double m0 = (double)pl.x * a.dm[0], m1 = (double)pl.y * a.dm[1];
  const double m2 = (double)pl.x * a.dm[2] + (double)pl.y * a.dm[3] + (double)pl.z;
  const double iw = 1.0 / (double)pl.w;
  const double x = (double)px, y = (double)py;
  const double q = (m0 * x + m1 * y + m2) * iw;  // m . p0 / w
  const double X = A[0] * x + A[1] * y + A[2] - b[0] * q;
  const double Y = A[3] * x + A[4] * y + A[5] - b[1] * q;
  const double Z = A[6] * x + A[7] * y + A[8] - b[2] * q;
  const double iz = 1.0 / Z;
  const double uc = X * iz, vc = Y * iz;
  const dpe_camera &sc = a.cam[s];
  if (!(uc >= 0.0 && uc < (double)sc.width && vc >= 0.0 && vc < (double)sc.height)) return false;
  const double U = floor(uc), V = floor(vc);
  wp.U0 = (int)U;
  wp.V0 = (int)V;
  wp.fuv = make_float2((float)(uc - U), (float)(vc - V));
  wp.zc = (float)Z;
  const double bw0 = b[0] * iw, bw1 = b[1] * iw, bw2 = b[2] * iw;
  const double h6 = A[6] - bw2 * m0, h7 = A[7] - bw2 * m1;
  wp.g03 = make_float2((float)((A[0] - bw0 * m0) - uc * h6), (float)((A[3] - bw1 * m0) - vc * h6));
  wp.g14 = make_float2((float)((A[1] - bw0 * m1) - uc * h7), (float)((A[4] - bw1 * m1) - vc * h7));
  wp.h6 = (float)h6;
  wp.h7 = (float)h7;
  wp.lo = make_float2((float)(-1 - wp.U0), (float)(-1 - wp.V0));
  wp.hi = make_float2((float)(a.W - 1 - wp.U0), (float)(a.H - 1 - wp.V0));
  return true;
}
// bilinear_s at (U0 + x, V0 + y): the clamp to [-1, W-1] x [-1, H-1] and the split into texel and
// weight are taken on the offsets, which equals them on the absolute coordinates.  The x and y
// halves and the two rows of the blend run as packed pairs (the same operations as bilinear_s).
template <class Src, bool kClamp = true>
__device__ __forceinline__ float bilinear_w(const Src &src, const WinProj &wp, float2 p) {
  const float2 c = kClamp ? make_float2(fminf(fmaxf(p.x, wp.lo.x), wp.hi.x), fminf(fmaxf(p.y, wp.lo.y), wp.hi.y)) : p;
  int ix, iy;
  const float2 f = floor_split2(c, &ix, &iy);
  const float2 a = sub2(c, f);                            // (ax, ay)
  const float2 oa = sub2(make_float2(1.0f, 1.0f), a);     // (1 - ax, 1 - ay)
  const float4 v = src.fetch((wp.V0 + iy + 1) * src.pw + (wp.U0 + ix + 1));
  // (top, bot) = (1 - ax) (v00, v01) + ax (v10, v11); then (1 - ay) top + ay bot
  const float2 l = mul2(make_float2(oa.x, oa.x), make_float2(v.x, v.z));
  const float2 rt = mul2(make_float2(a.x, a.x), make_float2(v.y, v.w));
  const float2 r = mul2(make_float2(oa.y, a.y), make_float2(l.x + rt.x, l.y + rt.y));
  return r.x + r.y;
}
// One tap of the strong window: sample the source at the projected tap and accumulate the
// hypothesis-dependent moments (sums of w*s, w*s^2, w*(r-c)*s over s = sample - c); acc holds
// (sum w*s, sum w*(r-c)*s).  cxy and cz carry the tap column's dx terms.
template <bool kClamp, class Src, class RW>
__device__ __forceinline__ void strong_tap(const WinProj &wp, const Src &src, const RW &rw, float2 cxy, float cz,
                                           float dy, int k, float2 &acc, float &s_ss) {
  const float2 gy = mul2(wp.g14, make_float2(dy, dy));
  const float Z = wp.h7 * dy + cz;
  const float iz = tap_rcp(Z);
  const float2 t = mul2(make_float2(gy.x + cxy.x, gy.y + cxy.y), make_float2(iz, iz));  // (X, Y) / Z
  const float sv = bilinear_w<Src, kClamp>(src, wp, make_float2(wp.fuv.x + t.x, wp.fuv.y + t.y)) - rw.center;
  const float2 m = mul2(rw.tap(k), make_float2(sv, sv));  // (w s, w (r - c) s)
  const float q = m.x * sv;
  acc.x += m.x;
  acc.y += m.y;
  s_ss += q;
}
// ComputeBilateralNCCOld (DPE.cu:696-782) with the reference window precomputed; the window loop
// for one source sampler, columns dx outer and rows dy inner as the reference window's taps.
template <bool kClamp, class Src, int kUnroll, class RW>
__device__ __forceinline__ void strong_window(const PMArgs &a, const WinProj &wp, const Src &src, const RW &rw,
                                              float &s_s, float &s_ss, float &s_rs) {
  const int r = a.P.strong_radius, inc = a.P.strong_increment;
  float2 acc = make_float2(s_s, s_rs);
  // Tap offsets are small whole numbers, so stepping them by float adds gives the same floats as
  // converting each integer, without a conversion per tap.
  if (kUnroll > 0 && r == 5 && inc == 2) {
    for (int ii = 0; ii < 6; ++ii) {
      const float dx = (float)(2 * ii - 5);
      const float2 cxy = mul2(wp.g03, make_float2(dx, dx));
      const float cz = wp.h6 * dx + wp.zc;
#pragma unroll(kUnroll > 0 ? kUnroll : 1)
      for (int jj = 0; jj < 6; ++jj)
        strong_tap<kClamp>(wp, src, rw, cxy, cz, (float)(2 * jj - 5), 6 * ii + jj, acc, s_ss);
    }
  } else {
    int k = 0;
    const float finc = (float)inc, d0 = (float)(-r);
    float dx = d0;
    for (int i = -r; i <= r; i += inc, dx += finc) {
      const float2 cxy = mul2(wp.g03, make_float2(dx, dx));
      const float cz = wp.h6 * dx + wp.zc;
      float dy = d0;
      for (int j = -r; j <= r; j += inc, dy += finc)
        strong_tap<kClamp>(wp, src, rw, cxy, cz, dy, k++, acc, s_ss);
    }
  }
  s_s = acc.x;
  s_rs = acc.y;
}
template <class Src, int kUnroll, class RW>
__device__ __forceinline__ float ncc_strong_src(const PMArgs &a, const WinProj &wp, const Src &src, const RW &rw) {
  float s_s = 0.f, s_ss = 0.f, s_rs = 0.f;
  // (a clamp-free copy of the loop for windows that project inside the source measured slower:
  // the second copy costs registers under the strong update's occupancy bound)
  strong_window<true, Src, kUnroll>(a, wp, src, rw, s_s, s_ss, s_rs);
  const float m_s = s_s * rw.inv_wsum;
  const float var_s = s_ss * rw.inv_wsum - m_s * m_s;
  if (rw.var_r < 1e-5f || var_s < 1e-5f) return 2.0f;
  const float cov = s_rs * rw.inv_wsum - rw.mean_r * m_s;
  return fmaxf(0.0f, fminf(2.0f, 1.0f - cov / sqrtf(rw.var_r * var_s)));
}
template <int kStage = DPE_STAGE_FP32, int kUnroll = 0, class RW>
__device__ __forceinline__ float ncc_strong(const PMArgs &a, int px, int py, int s, float4 pl, const RW &rw) {
  WinProj wp;
  if (!window_projection(a, s, pl, px, py, wp)) return 2.0f;
  if (rw.cnt) atomicAdd(rw.cnt, 1ull);
  return ncc_strong_src<decltype(SrcOf<kStage>::make(a, s)), kUnroll, RW>(a, wp, SrcOf<kStage>::make(a, s), rw);
}

// ------------------------------------------------------------------ strong NCC adjoint
// Cost and gradient of the strong NCC with respect to the plane (nx, ny, nz, w), and optionally
// with respect to the source image's pixels (accumulated into gimg, W*H, with atomics, each
// query's contribution times gscale: the upstream weight of its cost).  Two passes
// over the window, the second recomputing the projections instead of storing the patch:
//   pass 1: the moments and the cost, exactly as ncc_strong;
//   pass 2: per tap, dC/ds (s = bilinear sample) from the moments, through the bilinear slope to
//           the projected point, through the projection to the homography entries.
// dC/dH then goes through H = A - (b / w) m^T (homography_base) to the plane.  Where the cost is the
// constant 2 (centre outside the source, flat window) or clamped to [0, 2], the gradient is zero.
template <class RW>
__device__ __forceinline__ float ncc_strong_adjoint(const PMArgs &a, int px, int py, int s, float4 pl,
                                                    const RW &rw, float g[4], float *gimg, float gscale = 1.0f) {
  g[0] = g[1] = g[2] = g[3] = 0.0f;
  WinProj wp;
  if (!window_projection(a, s, pl, px, py, wp)) return 2.0f;
  const int r = a.P.strong_radius, inc = a.P.strong_increment;
  // pass 1: ncc_strong's own window loop
  float s_s = 0.f, s_ss = 0.f, s_rs = 0.f;
  strong_window<true, SrcF32, 0>(a, wp, src_f32(a, s), rw, s_s, s_ss, s_rs);
  const float m_s = s_s * rw.inv_wsum;
  const float var_s = s_ss * rw.inv_wsum - m_s * m_s;
  if (rw.var_r < 1e-5f || var_s < 1e-5f) return 2.0f;
  const float cov = s_rs * rw.inv_wsum - rw.mean_r * m_s;
  const float sq = sqrtf(rw.var_r * var_s);
  const float cost = 1.0f - cov / sq;
  if (!(cost > 0.0f && cost < 2.0f)) return fmaxf(0.0f, fminf(2.0f, cost));
  if (rw.cnt) atomicAdd(rw.cnt, 2ull);  // two passes over the window
  // dC/ds_k = w_k / sum(w) * (-(r_k - mean_r) / sq + cov * (s_k - m_s) / (var_s * sq))
  const float ka = -rw.inv_wsum / sq, kb = rw.inv_wsum * cov / (var_s * sq);
  float gH[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const int W = a.W, Hh = a.H, pw = a.pad_w;
  const float *__restrict__ img = a.img[s];
  int k = 0;
  for (int i = -r; i <= r; i += inc) {
    const float dx = (float)i, x = (float)(px + i);
    const float cx = wp.g03.x * dx, cy = wp.g03.y * dx, cz = wp.h6 * dx + wp.zc;
    for (int j = -r; j <= r; j += inc) {
      const float dy = (float)j, y = (float)(py + j);
      const float X = wp.g14.x * dy + cx, Y = wp.g14.y * dy + cy, Z = wp.h7 * dy + cz;
      const float iz = tap_rcp(Z);
      const float uo = wp.fuv.x + X * iz, vo = wp.fuv.y + Y * iz;  // offsets from (U0, V0)
      const float xc = fminf(fmaxf(uo, wp.lo.x), wp.hi.x), yc = fminf(fmaxf(vo, wp.lo.y), wp.hi.y);
      int ix, iy;
      const float fx = floor_split(xc, &ix), fy = floor_split(yc, &iy);
      const float ax = xc - fx, ay = yc - fy;
      const int x0 = wp.U0 + ix, y0 = wp.V0 + iy;
      const int o = (y0 + 1) * pw + (x0 + 1);
      const float v00 = img[o], v10 = img[o + 1], v01 = img[o + pw], v11 = img[o + pw + 1];
      const float sv = (1.0f - ay) * ((1.0f - ax) * v00 + ax * v10) + ay * ((1.0f - ax) * v01 + ax * v11) - rw.center;
      const float rc = texel(a, 0, px + i, py + j) - rw.center;  // r_k - c
      const float dc = rw.w(k) * (ka * (rc - rw.mean_r) + kb * (sv - m_s));
      // slope of the sample; zero along a clamped coordinate
      const float dsx = (uo > wp.lo.x && uo < wp.hi.x) ? (1.0f - ay) * (v10 - v00) + ay * (v11 - v01) : 0.0f;
      const float dsy = (vo > wp.lo.y && vo < wp.hi.y) ? (1.0f - ax) * (v01 - v00) + ax * (v11 - v10) : 0.0f;
      // u = X' / Z' with X' = H0. p, Z' = H2. p: du/dH0j = p_j / Z', du/dH2j = -u p_j / Z'
      const float u = (float)wp.U0 + uo, v = (float)wp.V0 + vo;
      const float gu = dc * dsx * iz, gv = dc * dsy * iz;
      gH[0] += gu * x; gH[1] += gu * y; gH[2] += gu;
      gH[3] += gv * x; gH[4] += gv * y; gH[5] += gv;
      const float gz = -(gu * u + gv * v);
      gH[6] += gz * x; gH[7] += gz * y; gH[8] += gz;
      if (gimg) {
        const float dcs = dc * gscale;  // the upstream weight of this query's cost
        const int xa = min(max(x0, 0), W - 1), xb = min(max(x0 + 1, 0), W - 1);
        const int ya = min(max(y0, 0), Hh - 1), yb = min(max(y0 + 1, 0), Hh - 1);
        atomicAdd(&gimg[(size_t)ya * W + xa], dcs * (1.0f - ax) * (1.0f - ay));
        atomicAdd(&gimg[(size_t)ya * W + xb], dcs * ax * (1.0f - ay));
        atomicAdd(&gimg[(size_t)yb * W + xa], dcs * (1.0f - ax) * ay);
        atomicAdd(&gimg[(size_t)yb * W + xb], dcs * ax * ay);
      }
      ++k;
    }
  }
  // H = A - (b / w) m^T, m = (nx / fx, ny / fy, nz - nx cx / fx - ny cy / fy):
  // dC/dm_j = -sum_i gH_ij b_i / w and dC/dw = -sum_j (dC/dm_j) m_j / w
  const float m[3] = {pl.x * a.hm[0], pl.y * a.hm[1], pl.x * a.hm[2] + pl.y * a.hm[3] + pl.z};
  const float *b = a.hb[s];
  float gm[3];
  for (int j = 0; j < 3; ++j) gm[j] = -(gH[j] * b[0] + gH[3 + j] * b[1] + gH[6 + j] * b[2]) / pl.w;
  g[0] = gm[0] * a.hm[0] + gm[2] * a.hm[2];
  g[1] = gm[1] * a.hm[1] + gm[2] * a.hm[3];
  g[2] = gm[2];
  g[3] = -(gm[0] * m[0] + gm[1] * m[1] + gm[2] * m[2]) / pl.w;
  return cost;
}

// Strong costs of plane pl against every source: out[j] = cost against source j + 1.
template <int kStage, int kUnroll = 0, class RW>
__device__ __forceinline__ void ncc_all_sources(const PMArgs &a, int px, int py, float4 pl, const RW &rw,
                                                float *out) {
  for (int j = 0; j < a.N - 1; ++j) out[j] = ncc_strong<kStage, kUnroll>(a, px, py, j + 1, pl, rw);
}
// Sum over the listed sources act[0..na) (ascending) of vw[j] * cost(j), in list order.
template <int kStage, class RW, class A>
__device__ __forceinline__ float weighted_ncc(const PMArgs &a, int px, int py, float4 pl, const RW &rw,
                                             const A *act, int na, const uint8_t *vw) {
  float tc = 0.0f;
  for (int q = 0; q < na; ++q) tc += vw[act[q]] * ncc_strong<kStage>(a, px, py, act[q] + 1, pl, rw);
  return tc;
}

__device__ __forceinline__ short2 neighbour(const PMArgs &a, int center, int k) {
  return a.neigh[(size_t)a.nmap[center] * kNeighbours + k];
}

// ------------------------------------------------------------------ deformable (weak) NCC
// ComputeBilateralNCCNew (DPE.cu:561-694): a centre window around the pixel plus eight small
// windows around its stored strong neighbours, all compared through the same homography.  The
// reference side of every window (bilateral weights, w * (r - c), the sums of w, w*(r-c) and
// w*(r-c)^2) does not depend on the hypothesis; k_weak_prepare tabulates it once per pixel and
// pass, and each evaluation reads the table.  Sums are accumulated in the same blocked order
// (per window column, then over columns) in both places.

// Window k's radius and step: the adaptive centre window (k = 0) or a fixed weak window.
__device__ __forceinline__ void weak_window_shape(const PMArgs &a, int center, int k, int *radius, int *inc) {
  int r = k == 0 ? a.P.strong_radius : a.P.weak_radius;
  int s = k == 0 ? a.P.strong_increment : a.P.weak_increment;
  if (a.P.use_radius && k == 0) {
    r = a.radius[center];
    s = cvmax(2, (int)(2.0 * r / 5.0));
  }
  *radius = r;
  *inc = s;
}
__device__ __forceinline__ int weak_window_base(const PMArgs &a, int k) {
  return k == 0 ? 0 : kMaxWin * kMaxWin + (k - 1) * a.wtaps;
}

// The hypothesis-dependent half of one window: sums of w*s, w*s^2, w*(r-c)*s over the taps.
template <class Src>
__device__ __forceinline__ float window_ncc_tab(const PMArgs &a, const float H[9], const Src &src, int cx, int cy,
                                                int radius, int inc, float ref_center, const float2 *__restrict__ tab,
                                                float4 win) {
  float s_s = 0, s_ss = 0, s_rs = 0;
  int t = 0;
  // whole-number tap coordinates stepped by exact float adds (no conversion per tap)
  const float finc = (float)inc, y0 = (float)(cy - radius);
  float x = (float)(cx - radius);
  for (int i = -radius; i <= radius; i += inc, x += finc) {
    float r_s = 0, r_ss = 0, r_rs = 0;
    float y = y0;
    for (int j = -radius; j <= radius; j += inc, y += finc) {
      const float2 sp = project_tap(H, x, y);
      const float sv = bilinear_s(src, a.W, a.H, sp.x, sp.y) - ref_center;
      const float2 m = mul2(tab[t++], make_float2(sv, sv));  // (w s, w (r - c) s)
      r_s += m.x; r_ss += m.x * sv; r_rs += m.y;
    }
    s_s += r_s; s_ss += r_ss; s_rs += r_rs;
  }
  float s_w = win.x, s_r = win.y, s_rr = win.z;
  const float inv = 1.0f / s_w;
  s_r *= inv; s_rr *= inv; s_s *= inv; s_ss *= inv; s_rs *= inv;
  const float var_r = s_rr - s_r * s_r;
  const float var_s = s_ss - s_s * s_s;
  if (var_r < 1e-5f || var_s < 1e-5f) return 2.0f;
  const float cov = s_rs - s_r * s_s;
  return fmaxf(0.0f, fminf(2.0f, 1.0f - cov / sqrtf(var_r * var_s)));
}

// The deformable cost of hypothesis pl against source s for the pixel in `slot`.
template <int kStage>
__device__ __forceinline__ float ncc_weak_tab(const PMArgs &a, int slot, int center, int px, int py, int s, float4 pl,
                                              int kid) {
  float H[9];
  homography(a, s, pl, H);
  const float2 pt = project(H, px, py);
  const dpe_camera &sc = a.cam[s];
  if (pt.x >= sc.width || pt.x < 0.0f || pt.y >= sc.height || pt.y < 0.0f) return 2.0f;
  if (a.counters) atomicAdd(&a.counters[2 * kid + 1], 1ull);
  const float ref_center = texel(a, 0, px, py);
  const float2 *tab = a.wtab + (size_t)slot * a.wtab_stride;
  float center_cost = 0.0f, strong_cost = 0.0f;
  int strong_count = 0;
  for (int k = 0; k < kNeighbours; ++k) {
    const short2 nb = neighbour(a, center, k);
    if (nb.x == -1 || nb.y == -1) continue;
    const float2 np = project(H, nb.x, nb.y);
    if (np.x < 0 || np.y < 0 || np.x >= a.W || np.y >= a.H) {
      if (k != 0) {
        const long idx = (long)nb.x + (long)nb.y * a.W;
        const uint32_t v = (idx >= 0 && idx < (long)a.W * a.H) ? a.views[idx] : 0u;
        if (isSet(v, s - 1)) { strong_cost += 2.0f; strong_count++; }
        continue;
      }
      return 2.0f;
    }
    int radius, inc;
    weak_window_shape(a, center, k, &radius, &inc);
    const float2 *wt = tab + weak_window_base(a, k);
    const float4 win = a.wwin[(size_t)slot * kNeighbours + k];
    const float t = window_ncc_tab(a, H, SrcOf<kStage>::make(a, s), nb.x, nb.y, radius, inc, ref_center, wt, win);
    if (k == 0) center_cost = t;
    else { strong_cost += t; strong_count++; }
  }
  if (strong_count == 0) return center_cost;
  strong_cost /= strong_count;
  strong_cost = cvmin(strong_cost, 2.0f);
  return (float)(0.25 * center_cost + 0.75 * strong_cost);
}

// ComputeGeomConsistencyCost (DPE.cu:919-957)
__device__ __forceinline__ float3 point_world(float x, float y, float depth, const dpe_camera &c) {
  const float px = depth * (x - c.K[2]) / c.K[0];
  const float py = depth * (y - c.K[5]) / c.K[4];
  const float pz = depth;
  const float tx = c.R[0] * px + c.R[3] * py + c.R[6] * pz;
  const float ty = c.R[1] * px + c.R[4] * py + c.R[7] * pz;
  const float tz = c.R[2] * px + c.R[5] * py + c.R[8] * pz;
  return make_float3(tx + c.c[0], ty + c.c[1], tz + c.c[2]);
}
__device__ __forceinline__ void project_camera(float3 X, const dpe_camera &c, float2 &pt, float &depth) {
  const float tx = c.R[0] * X.x + c.R[1] * X.y + c.R[2] * X.z + c.t[0];
  const float ty = c.R[3] * X.x + c.R[4] * X.y + c.R[5] * X.z + c.t[1];
  const float tz = c.R[6] * X.x + c.R[7] * X.y + c.R[8] * X.z + c.t[2];
  depth = c.K[6] * tx + c.K[7] * ty + c.K[8] * tz;
  pt.x = (c.K[0] * tx + c.K[1] * ty + c.K[2] * tz) / depth;
  pt.y = (c.K[3] * tx + c.K[4] * ty + c.K[5] * tz) / depth;
}
__device__ __forceinline__ float geom_cost(const PMArgs &a, int px, int py, int s, float4 pl) {
  const dpe_camera &rc = a.cam[0], &sc = a.cam[s];
  const float depth = depth_from_plane(rc, pl, px, py);
  const float3 fw = point_world((float)px, (float)py, depth, rc);
  float2 sp;
  float sd;
  project_camera(fw, sc, sp, sd);
  int ix = (int)sp.x, iy = (int)sp.y;  // cvt.rzi: truncation, NaN -> 0
  ix = min(max(ix, 0), a.W - 1);
  iy = min(max(iy, 0), a.H - 1);
  const float src_depth = __ldg(a.dep[s] + (size_t)iy * a.W + ix);
  if (src_depth == 0.0f) return 3.0f;
  const float3 sw = point_world(sp.x, sp.y, src_depth, sc);
  float2 bp;
  float rd;
  project_camera(sw, rc, bp, rd);
  const float dx = (float)px - bp.x, dy = (float)py - bp.y;
  return fminf(3.0f, sqrtf(dx * dx + dy * dy));
}

// ------------------------------------------------------------------ packed view weights
// Inlined helpers declare no local arrays: the device compiler once gave such an array the stack
// slot of a still-live array of the calling kernel (found with the DPE_CHECKED build).
__device__ __forceinline__ void store_vweight(uint4 *dst, const uint8_t *vw) {
  uint32_t w0 = 0, w1 = 0, w2 = 0, w3 = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    w0 |= (uint32_t)(vw[i] & 0xF) << (4 * i);
    w1 |= (uint32_t)(vw[8 + i] & 0xF) << (4 * i);
    w2 |= (uint32_t)(vw[16 + i] & 0xF) << (4 * i);
    w3 |= (uint32_t)(vw[24 + i] & 0xF) << (4 * i);
  }
  *dst = make_uint4(w0, w1, w2, w3);
}
__device__ __forceinline__ int vweight_at(const uint4 &p, int i) {
  const uint32_t w = (i >> 3) == 0 ? p.x : (i >> 3) == 1 ? p.y : (i >> 3) == 2 ? p.z : p.w;
  return (w >> (4 * (i & 7))) & 0xF;
}

}  // namespace dpe
