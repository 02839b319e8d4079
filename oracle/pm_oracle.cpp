// pm_oracle.cpp -- CPU restatement of the reference's per-view PatchMatch (DPE.cu:1-3262).
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA kernels in dpe-mvs-fast_b200/csrc.
// PARITY PINNED to the reference itself: the reference's own DPE.cu and DPE.cpp compiled for the
// CPU (oracle/_ref, built by oracle/Makefile behind the stand-ins of oracle/refshim) produce the
// same bits as this restatement on the first-init, weak-texture and geometric paths when the
// switches below select the reference's arithmetic (oracle_set_raw_moments,
// oracle_set_ref_addressing, oracle_set_ref_homography, oracle_set_serial_race);
// tests/test_ref_oracle.py holds that.
// Each function cites the reference lines it restates.  Semantics are FP32 without fast-math
// (the reference build uses --use_fast_math, CMakeLists.txt:26; that rounding is not restated).
// Red/black passes run in the reference's colour order; pixels of one colour are independent and
// run in parallel with OpenMP.  Deviations from the reference, all documented:
//   * random streams: Philox4x32-10 per pixel instead of clock64()-seeded XORWOW (DPE.cu:1036);
//   * the same-colour read race of the edge-aware strong update (direction 4, DPE.cu:1279/1316)
//     reads a snapshot of costs/planes taken before the colour pass (oracle_set_serial_race
//     selects the serial raster-order reading instead);
//   * NCC moments are shifted by the window centre (oracle_set_raw_moments selects the raw ones);
//   * the homography's camera part is composed in double once per call, and each strong window's
//     centre is projected in double with its taps as float offsets (oracle_set_ref_homography
//     selects the reference's per-hypothesis float composition and float projection);
//   * texture reads are exact bilinear with clamp-to-edge addressing at x itself (the hardware
//     path uses 8-bit interpolation weights; oracle_set_ref_addressing adds the rounding of the
//     reference's tex2D(x + 0.5, y + 0.5) coordinate);
//   * radius_cuda starts at strong_radius (the reference may read it uninitialised,
//     DPE.cu:2950-2953 vs :624);
//   * out-of-image linear indices read 0 (the reference reads outside its buffers in
//     BresenhamLine DPE.cu:189-211 and in the edge-mode view prior DPE.cu:1558-1562).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <omp.h>

#include "oracle_common.h"

namespace oracle {

static const float kPi = 3.14159265358979323846f;

// Texture addressing of the reference: its kernels sample tex2D(x + 0.5f, y + 0.5f) and the
// texture unit blends around (u - 0.5, v - 0.5), so a sample position passes through one float
// rounding of x + 0.5 (inexact when x + 0.5 changes binade or x has bits below its ulp).  The
// default samples at x itself (the CUDA kernels' addressing); oracle_set_ref_addressing(1) adds
// the round trip, for bit-for-bit comparisons with the reference's own code compiled for the CPU.
static bool g_ref_addressing = false;
// The reference's float operation order for the homography (homography_ref) instead of the
// double-composed camera part (homography_base).
static bool g_ref_homography = false;

// The same-colour read race of the edge-aware strong update (quirk Q1, DPE.cu:1279/1316): by
// default the edge branch reads a snapshot taken before each colour pass (the CUDA kernels'
// resolution).  oracle_set_serial_race(1) resolves it as a one-thread run in raster order does
// instead -- the up-left same-colour candidate has already been updated when it is read -- which
// is how the reference's own kernels behave when compiled for the CPU and run one thread at a time.
static bool g_serial_race = false;

// A strong window projected into a source (window_projection): its centre as an integer texel
// (U0, V0) plus a float fraction (fu, fv), the per-tap terms, and the texture clamp relative to
// (U0, V0).
struct WinProj {
  int U0, V0;
  float fu, fv, zc, g0, g1, g3, g4, h6, h7, lox, hix, loy, hiy;
};

struct Image {
  const float *data = nullptr;
  int w = 0, h = 0;
  float texel(int x, int y) const {
    x = x < 0 ? 0 : (x >= w ? w - 1 : x);
    y = y < 0 ? 0 : (y >= h ? h - 1 : y);
    return data[(size_t)y * w + x];
  }
  // tex2D(x + 0.5, y + 0.5) with linear filtering and clamp addressing, exact weights.
  float bilinear(float x, float y) const {
    if (g_ref_addressing) {
      volatile float u = x + 0.5f, v = y + 0.5f;
      x = u - 0.5f;
      y = v - 0.5f;
    }
    const float xc = std::fmin(std::fmax(x, -1.0f), (float)(w - 1));
    const float yc = std::fmin(std::fmax(y, -1.0f), (float)(h - 1));
    const float fx = std::floor(xc), fy = std::floor(yc);
    const int x0 = (int)fx, y0 = (int)fy;
    const float ax = xc - fx, ay = yc - fy;
    const float v00 = texel(x0, y0), v10 = texel(x0 + 1, y0);
    const float v01 = texel(x0, y0 + 1), v11 = texel(x0 + 1, y0 + 1);
    const float top = (1.0f - ax) * v00 + ax * v10;
    const float bot = (1.0f - ax) * v01 + ax * v11;
    return (1.0f - ay) * top + ay * bot;
  }
  // bilinear() at (U0 + x, V0 + y), with the clamp to [-1, w-1] x [-1, h-1] taken on the offsets
  // ([lox, hix] x [loy, hiy] = the clamp shifted by (U0, V0)), which equals it on the sum.
  float bilinear_off(const WinProj &wp, float x, float y) const {
    const float xc = std::fmin(std::fmax(x, wp.lox), wp.hix);
    const float yc = std::fmin(std::fmax(y, wp.loy), wp.hiy);
    const float fx = std::floor(xc), fy = std::floor(yc);
    const int x0 = wp.U0 + (int)fx, y0 = wp.V0 + (int)fy;
    const float ax = xc - fx, ay = yc - fy;
    const float v00 = texel(x0, y0), v10 = texel(x0 + 1, y0);
    const float v01 = texel(x0, y0 + 1), v11 = texel(x0 + 1, y0 + 1);
    const float top = (1.0f - ax) * v00 + ax * v10;
    const float bot = (1.0f - ax) * v01 + ax * v11;
    return (1.0f - ay) * top + ay * bot;
  }
  double bilinear_fp64(double x, double y) const {
    const double xc = std::fmin(std::fmax(x, -1.0), (double)(w - 1));
    const double yc = std::fmin(std::fmax(y, -1.0), (double)(h - 1));
    const double fx = std::floor(xc), fy = std::floor(yc);
    const int x0 = (int)fx, y0 = (int)fy;
    const double ax = xc - fx, ay = yc - fy;
    const double v00 = texel(x0, y0), v10 = texel(x0 + 1, y0);
    const double v01 = texel(x0, y0 + 1), v11 = texel(x0 + 1, y0 + 1);
    const double top = (1.0 - ax) * v00 + ax * v10;
    const double bot = (1.0 - ax) * v01 + ax * v11;
    return (1.0 - ay) * top + ay * bot;
  }
};

static inline int isSet(uint32_t v, int n) { return (v >> n) & 1; }
static inline void setBit(uint32_t *v, int n) { *v |= (uint32_t)(1u << n); }
// DPE.cu:81-84: clears bits 0..n (quirk Q3)
static inline void unSetBit(uint32_t *v, int n) { *v &= (uint32_t)(0xFFFFFFFEu << n); }

// ----------------------------------------------------------------------------- camera geometry
// DPE.cu:457-517, in the reference's float operation order: the relative pose, G = Rrel - trel n^T / w,
// then G Kr^-1 and Ks (G Kr^-1), every step in float.
static void homography_ref(const dpe_camera &rc, const dpe_camera &sc, const f4 &pl, float H[9]) {
  float rC[3], sC[3];
  for (int k = 0; k < 3; ++k) {
    rC[k] = -(rc.R[k] * rc.t[0] + rc.R[3 + k] * rc.t[1] + rc.R[6 + k] * rc.t[2]);
    sC[k] = -(sc.R[k] * sc.t[0] + sc.R[3 + k] * sc.t[1] + sc.R[6 + k] * sc.t[2]);
  }
  float Rr[9], Cr[3], tr[3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      Rr[3 * a + b] = sc.R[3 * a] * rc.R[3 * b] + sc.R[3 * a + 1] * rc.R[3 * b + 1] + sc.R[3 * a + 2] * rc.R[3 * b + 2];
  for (int k = 0; k < 3; ++k) Cr[k] = rC[k] - sC[k];
  for (int a = 0; a < 3; ++a) tr[a] = sc.R[3 * a] * Cr[0] + sc.R[3 * a + 1] * Cr[1] + sc.R[3 * a + 2] * Cr[2];
  const float n[3] = {pl.x, pl.y, pl.z};
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) H[3 * a + b] = Rr[3 * a + b] - tr[a] * n[b] / pl.w;
  float T[9];
  for (int a = 0; a < 3; ++a) {
    T[3 * a] = H[3 * a] / rc.K[0];
    T[3 * a + 1] = H[3 * a + 1] / rc.K[4];
    T[3 * a + 2] = -H[3 * a] * rc.K[2] / rc.K[0] - H[3 * a + 1] * rc.K[5] / rc.K[4] + H[3 * a + 2];
  }
  for (int b = 0; b < 3; ++b) {
    H[b] = sc.K[0] * T[b] + sc.K[2] * T[6 + b];
    H[3 + b] = sc.K[4] * T[3 + b] + sc.K[5] * T[6 + b];
    H[6 + b] = sc.K[8] * T[6 + b];
  }
}

// The same homography H = Ks (Rrel - trel n^T / w) Kr^-1 written as A - b m^T / w with
//   A = Ks Rrel Kr^-1,  b = Ks trel,  m = Kr^-T n = (nx / fx, ny / fy, nz - nx cx / fx - ny cy / fy),
// Rrel = Rs Rr^T, trel = Rs (Cr - Cs), C = -R^T t.  The plane-independent A, b and the entries of
// Kr^-1 (dm = (1/fx, 1/fy, -cx/fx, -cy/fy)) are composed in double once per call, kept in double
// for the projection of window centres (window_projection) and rounded once to float for the
// float homography.  Composing the camera products in float, as the reference does, moves the
// entries of H by a few float ulps, which at source coordinates of ~2000 px places a window
// ~1e-4 px off and on low-contrast windows moves the NCC by about as much.
struct HomographyBase {
  double dA[9], db[3], dm[4];
  float A[9], b[3], m[4];
};
static HomographyBase homography_base(const dpe_camera &rc, const dpe_camera &sc) {
  double rC[3], sC[3], Rr[9], Cr[3], tr[3], MK[9];
  for (int k = 0; k < 3; ++k) {
    rC[k] = -((double)rc.R[k] * rc.t[0] + (double)rc.R[3 + k] * rc.t[1] + (double)rc.R[6 + k] * rc.t[2]);
    sC[k] = -((double)sc.R[k] * sc.t[0] + (double)sc.R[3 + k] * sc.t[1] + (double)sc.R[6 + k] * sc.t[2]);
  }
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      Rr[3 * a + b] = (double)sc.R[3 * a] * rc.R[3 * b] + (double)sc.R[3 * a + 1] * rc.R[3 * b + 1] +
                      (double)sc.R[3 * a + 2] * rc.R[3 * b + 2];
  for (int k = 0; k < 3; ++k) Cr[k] = rC[k] - sC[k];
  for (int a = 0; a < 3; ++a)
    tr[a] = (double)sc.R[3 * a] * Cr[0] + (double)sc.R[3 * a + 1] * Cr[1] + (double)sc.R[3 * a + 2] * Cr[2];
  HomographyBase h;
  h.dm[0] = 1.0 / rc.K[0];
  h.dm[1] = 1.0 / rc.K[4];
  h.dm[2] = -(double)rc.K[2] / rc.K[0];
  h.dm[3] = -(double)rc.K[5] / rc.K[4];
  for (int a = 0; a < 3; ++a) {
    MK[3 * a] = Rr[3 * a] * h.dm[0];
    MK[3 * a + 1] = Rr[3 * a + 1] * h.dm[1];
    MK[3 * a + 2] = Rr[3 * a] * h.dm[2] + Rr[3 * a + 1] * h.dm[3] + Rr[3 * a + 2];
  }
  for (int j = 0; j < 3; ++j) {
    h.dA[j] = (double)sc.K[0] * MK[j] + (double)sc.K[2] * MK[6 + j];
    h.dA[3 + j] = (double)sc.K[4] * MK[3 + j] + (double)sc.K[5] * MK[6 + j];
    h.dA[6 + j] = (double)sc.K[8] * MK[6 + j];
  }
  h.db[0] = (double)sc.K[0] * tr[0] + (double)sc.K[2] * tr[2];
  h.db[1] = (double)sc.K[4] * tr[1] + (double)sc.K[5] * tr[2];
  h.db[2] = (double)sc.K[8] * tr[2];
  for (int k = 0; k < 9; ++k) h.A[k] = (float)h.dA[k];
  for (int k = 0; k < 3; ++k) h.b[k] = (float)h.db[k];
  for (int k = 0; k < 4; ++k) h.m[k] = (float)h.dm[k];
  return h;
}
static inline void homography_plane(const HomographyBase &hb, const f4 &pl, float H[9]) {
  const float m[3] = {pl.x * hb.m[0], pl.y * hb.m[1], pl.x * hb.m[2] + pl.y * hb.m[3] + pl.z};
  for (int i = 0; i < 3; ++i) {
    const float bi = hb.b[i] / pl.w;
    for (int j = 0; j < 3; ++j) H[3 * i + j] = hb.A[3 * i + j] - bi * m[j];
  }
}

// Projection of a strong window centred on (px, py) into a source.  The centre goes through the
// homography in double (from the double bases; the plane enters in double); it is kept as an
// integer texel (U0, V0) plus a float fraction, and each tap p0 + (dx, dy) as a float offset:
//   u(p0 + d) - uc = ((H00 - uc H20) dx + (H01 - uc H21) dy) / (Zc + H20 dx + H21 dy),
// whose terms are small, so float arithmetic places the taps to ~1e-6 px.
// false when the centre does not project inside the source (DPE.cu:709-712: cost 2)
static bool window_projection(const HomographyBase &hb, const dpe_camera &sc, int W, int H, const f4 &pl, int px,
                              int py, WinProj &wp) {
  const double *A = hb.dA, *b = hb.db;
  const double m0 = (double)pl.x * hb.dm[0], m1 = (double)pl.y * hb.dm[1];
  const double m2 = (double)pl.x * hb.dm[2] + (double)pl.y * hb.dm[3] + (double)pl.z;
  const double iw = 1.0 / (double)pl.w;
  const double x = (double)px, y = (double)py;
  const double q = (m0 * x + m1 * y + m2) * iw;
  const double X = A[0] * x + A[1] * y + A[2] - b[0] * q;
  const double Y = A[3] * x + A[4] * y + A[5] - b[1] * q;
  const double Z = A[6] * x + A[7] * y + A[8] - b[2] * q;
  const double iz = 1.0 / Z;
  const double uc = X * iz, vc = Y * iz;
  if (!(uc >= 0.0 && uc < (double)sc.width && vc >= 0.0 && vc < (double)sc.height)) return false;
  const double U = std::floor(uc), V = std::floor(vc);
  wp.U0 = (int)U;
  wp.V0 = (int)V;
  wp.fu = (float)(uc - U);
  wp.fv = (float)(vc - V);
  wp.zc = (float)Z;
  const double bw0 = b[0] * iw, bw1 = b[1] * iw, bw2 = b[2] * iw;
  const double h6 = A[6] - bw2 * m0, h7 = A[7] - bw2 * m1;
  wp.g0 = (float)((A[0] - bw0 * m0) - uc * h6);
  wp.g1 = (float)((A[1] - bw0 * m1) - uc * h7);
  wp.g3 = (float)((A[3] - bw1 * m0) - vc * h6);
  wp.g4 = (float)((A[4] - bw1 * m1) - vc * h7);
  wp.h6 = (float)h6;
  wp.h7 = (float)h7;
  wp.lox = (float)(-1 - wp.U0);
  wp.hix = (float)(W - 1 - wp.U0);
  wp.loy = (float)(-1 - wp.V0);
  wp.hiy = (float)(H - 1 - wp.V0);
  return true;
}

// DPE.cu:519-526
static inline f2 project(const float H[9], int x, int y) {
  const float fx = (float)x, fy = (float)y;
  const float X = H[0] * fx + H[1] * fy + H[2];
  const float Y = H[3] * fx + H[4] * fy + H[5];
  const float Z = H[6] * fx + H[7] * fy + H[8];
  return {X / Z, Y / Z};
}

// DPE.cu:528-546
static inline f4 normal_to_world(const dpe_camera &c, const f4 &p) {
  return {c.R[0] * p.x + c.R[3] * p.y + c.R[6] * p.z, c.R[1] * p.x + c.R[4] * p.y + c.R[7] * p.z,
          c.R[2] * p.x + c.R[5] * p.y + c.R[8] * p.z, p.w};
}
static inline f4 normal_to_ref(const dpe_camera &c, const f4 &p) {
  return {c.R[0] * p.x + c.R[1] * p.y + c.R[2] * p.z, c.R[3] * p.x + c.R[4] * p.y + c.R[5] * p.z,
          c.R[6] * p.x + c.R[7] * p.y + c.R[8] * p.z, p.w};
}

// DPE.cu:313-325
static inline void point3d(const dpe_camera &c, int x, int y, float depth, float X[3]) {
  X[0] = depth * ((float)x - c.K[2]) / c.K[0];
  X[1] = depth * ((float)y - c.K[5]) / c.K[4];
  X[2] = depth;
}
// DPE.cu:327-339
static inline f4 view_direction(const dpe_camera &c, int x, int y, float depth) {
  float X[3];
  point3d(c, x, y, depth, X);
  const float norm = std::sqrt(X[0] * X[0] + X[1] * X[1] + X[2] * X[2]);
  return {X[0] / norm, X[1] / norm, X[2] / norm, 0.0f};
}
// DPE.cu:341-346
static inline float dist_to_origin(const dpe_camera &c, int x, int y, float depth, const f4 &n) {
  float X[3];
  point3d(c, x, y, depth, X);
  return -(n.x * X[0] + n.y * X[1] + n.z * X[2]);
}
// DPE.cu:360-363
static inline float depth_from_plane(const dpe_camera &c, const f4 &pl, int x, int y) {
  return -pl.w * c.K[0] /
         (((float)x - c.K[2]) * pl.x + (c.K[0] / c.K[4]) * ((float)y - c.K[5]) * pl.y + c.K[0] * pl.z);
}
// DPE.cu:272-287 (1/sqrt instead of the approximate rsqrtf)
static inline void normalize3(f4 *v) {
  const float inv = 1.0f / std::sqrt(v->x * v->x + v->y * v->y + v->z * v->z);
  v->x *= inv; v->y *= inv; v->z *= inv;
}
static inline void normalize3(f3 *v) {
  const float inv = 1.0f / std::sqrt(v->x * v->x + v->y * v->y + v->z * v->z);
  v->x *= inv; v->y *= inv; v->z *= inv;
}
static inline void normalize2(f2 *v) {
  const float inv = 1.0f / std::sqrt(v->x * v->x + v->y * v->y);
  v->x *= inv; v->y *= inv;
}

// DPE.cu:365-391.  The rejection loop is capped (64 tries; the chance of reaching it is
// (1-pi/4)^64 ~ 1e-43); on the cap the last (q1, q2) pair is used as is.
static f4 random_normal(const dpe_camera &c, int x, int y, PixelRng &rng, float depth) {
  float q1 = 1.0f, q2 = 1.0f, s = 2.0f;
  for (int tries = 0; s >= 1.0f && tries < 64; ++tries) {
    q1 = 2.0f * rng.uniform() - 1.0f;
    q2 = 2.0f * rng.uniform() - 1.0f;
    s = q1 * q1 + q2 * q2;
  }
  const float sq = std::sqrt(std::fmax(1.0f - s, 0.0f));
  f4 n = {2.0f * q1 * sq, 2.0f * q2 * sq, 1.0f - 2.0f * s, 0.0f};
  const f4 v = view_direction(c, x, y, depth);
  if (n.x * v.x + n.y * v.y + n.z * v.z > 0.0f) { n.x = -n.x; n.y = -n.y; n.z = -n.z; }
  normalize3(&n);
  return n;
}

// DPE.cu:393-428
static f4 perturbed_normal(const dpe_camera &c, int x, int y, const f4 &n, PixelRng &rng, float pert) {
  const f4 v = view_direction(c, x, y, 1.0f);
  const float a1 = (rng.uniform() - 0.5f) * pert;
  const float a2 = (rng.uniform() - 0.5f) * pert;
  const float a3 = (rng.uniform() - 0.5f) * pert;
  float s1, s2, s3, c1, c2, c3;
  dpe::dpe_sincos_small(a1, &s1, &c1);
  dpe::dpe_sincos_small(a2, &s2, &c2);
  dpe::dpe_sincos_small(a3, &s3, &c3);
  const float R[9] = {c2 * c3, c3 * s1 * s2 - c1 * s3, s1 * s3 + c1 * c3 * s2,
                      c2 * s3, c1 * c3 + s1 * s2 * s3, c1 * s2 * s3 - c3 * s1,
                      -s2,     c2 * s1,                c1 * c2};
  f4 r = {R[0] * n.x + R[1] * n.y + R[2] * n.z, R[3] * n.x + R[4] * n.y + R[5] * n.z,
          R[6] * n.x + R[7] * n.y + R[8] * n.z, n.w};
  if (r.x * v.x + r.y * v.y + r.z * v.z >= 0.0f) r = n;
  normalize3(&r);
  return r;
}

// DPE.cu:885-917
static inline f3 point_world(float x, float y, float depth, const dpe_camera &c) {
  const float px = depth * (x - c.K[2]) / c.K[0];
  const float py = depth * (y - c.K[5]) / c.K[4];
  const float pz = depth;
  const float tx = c.R[0] * px + c.R[3] * py + c.R[6] * pz;
  const float ty = c.R[1] * px + c.R[4] * py + c.R[7] * pz;
  const float tz = c.R[2] * px + c.R[5] * py + c.R[8] * pz;
  return {tx + c.c[0], ty + c.c[1], tz + c.c[2]};
}
static inline void project_camera(const f3 &X, const dpe_camera &c, f2 &pt, float &depth) {
  const float tx = c.R[0] * X.x + c.R[1] * X.y + c.R[2] * X.z + c.t[0];
  const float ty = c.R[3] * X.x + c.R[4] * X.y + c.R[5] * X.z + c.t[1];
  const float tz = c.R[6] * X.x + c.R[7] * X.y + c.R[8] * X.z + c.t[2];
  depth = c.K[6] * tx + c.K[7] * ty + c.K[8] * tz;
  pt.x = (c.K[0] * tx + c.K[1] * ty + c.K[2] * tz) / depth;
  pt.y = (c.K[3] * tx + c.K[4] * ty + c.K[5] * tz) / depth;
}

// DPE.cu:139-160
static bool point_in_triangle(s2 A, s2 B, s2 C, int px, int py) {
  const f2 AB = {(float)(B.x - A.x), (float)(B.y - A.y)};
  const f2 BC = {(float)(C.x - B.x), (float)(C.y - B.y)};
  const f2 CA = {(float)(A.x - C.x), (float)(A.y - C.y)};
  const float ab = std::sqrt(AB.x * AB.x + AB.y * AB.y);
  const float bc = std::sqrt(BC.x * BC.x + BC.y * BC.y);
  const float ca = std::sqrt(CA.x * CA.x + CA.y * CA.y);
  if (ab <= 2 || bc <= 2 || ca <= 2) return false;
  if (!(ab + bc > ca && bc + ca > ab && ab + ca > bc)) return false;
  const f2 PA = {(float)(A.x - px), (float)(A.y - py)};
  const f2 PB = {(float)(B.x - px), (float)(B.y - py)};
  const f2 PC = {(float)(C.x - px), (float)(C.y - py)};
  const float t1 = PA.x * PB.y - PA.y * PB.x;
  const float t2 = PB.x * PC.y - PB.y * PC.x;
  const float t3 = PC.x * PA.y - PC.y * PA.x;
  return t1 * t2 >= 0 && t1 * t3 >= 0;
}

// ----------------------------------------------------------------------------- per-call state
struct Ctx {
  int W = 0, H = 0, N = 0, lowW = 0, lowH = 0;
  dpe_params P;
  dpe_camera cam[DPE_MAX_IMAGES];
  HomographyBase hbase[DPE_MAX_IMAGES];  // filled by set_cameras()
  Image img[DPE_MAX_IMAGES];
  Image dep[DPE_MAX_IMAGES];
  uint32_t key[2];
  std::vector<f4> plane, plane_snap, fit_plane;
  std::vector<float> cost, cost_snap, complexity;
  std::vector<uint32_t> views, rng_ctr;
  std::vector<uint8_t> weak, reliable, vweight, edge, edge_low;
  std::vector<int32_t> nmap, label, radius;
  std::vector<s2> neigh, lab_bound, edge_neigh, nearest;
  int weak_count = 0;

  PixelRng rng(int center) { return PixelRng{{key[0], key[1]}, (uint32_t)center, &rng_ctr[center]}; }
  uint8_t edge_at(long idx) const { return (idx >= 0 && idx < (long)edge.size()) ? edge[idx] : 0; }
  uint8_t edge_low_at(long idx) const { return (idx >= 0 && idx < (long)edge_low.size()) ? edge_low[idx] : 0; }
  uint32_t views_at(long idx) const { return (idx >= 0 && idx < (long)views.size()) ? views[idx] : 0u; }
  s2 neighbour(int center, int k) const { return neigh[(size_t)nmap[center] * DPE_NEIGHBOUR_NUM + k]; }
  void set_cameras(const dpe_camera *cams) {
    for (int i = 0; i < N; ++i) cam[i] = cams[i];
    for (int i = 1; i < N; ++i) hbase[i] = homography_base(cam[0], cam[i]);
  }
  // Homography of a reference-camera plane into source src (DPE.cu:457-517).
  void homography(int src, const f4 &pl, float H[9]) const {
    if (g_ref_homography) homography_ref(cam[0], cam[src], pl, H);
    else homography_plane(hbase[src], pl, H);
  }
};

// ----------------------------------------------------------------------------- costs
static inline float bilateral_weight(float dx, float dy, float pix, float center, float ss, float sc) {
  const float spatial = std::sqrt(dx * dx + dy * dy);
  const float color = std::fabs(pix - center);
  return dpe::dpe_expf(-spatial / (2.0f * ss * ss) - color / (2.0f * sc * sc));
}

// Moment form of the window NCC.  The reference accumulates raw moments (E[x^2] - E[x]^2,
// DPE.cu:661-662); the default here accumulates on intensities shifted by the reference centre
// value, which leaves variance and covariance unchanged mathematically but avoids FP32
// cancellation (the compensated form the CUDA kernels use).  oracle_set_raw_moments(1) selects
// the reference's raw form.
static bool g_raw_moments = false;

// Window moments of one NCC window (the shared core of DPE.cu:628-672 and :728-778).
static float window_ncc(const Ctx &c, const float H[9], const Image &src, int cx, int cy, int radius, int inc,
                        float ref_center) {
  const Image &ref = c.img[0];
  const float shift = g_raw_moments ? 0.0f : ref_center;
  float s_r = 0, s_rr = 0, s_s = 0, s_ss = 0, s_rs = 0, s_w = 0;
  for (int i = -radius; i <= radius; i += inc) {
    float r_r = 0, r_rr = 0, r_s = 0, r_ss = 0, r_rs = 0, r_w = 0;
    for (int j = -radius; j <= radius; j += inc) {
      const int rx = cx + i, ry = cy + j;
      const float rp0 = ref.texel(rx, ry);
      const f2 sp = project(H, rx, ry);
      const float sv = src.bilinear(sp.x, sp.y) - shift;
      const float w = bilateral_weight((float)i, (float)j, rp0, ref_center, c.P.sigma_spatial, c.P.sigma_color);
      const float rp = rp0 - shift;
      r_r += w * rp; r_rr += w * rp * rp; r_s += w * sv; r_ss += w * sv * sv; r_rs += w * rp * sv; r_w += w;
    }
    s_r += r_r; s_rr += r_rr; s_s += r_s; s_ss += r_ss; s_rs += r_rs; s_w += r_w;
  }
  const float inv = 1.0f / s_w;
  s_r *= inv; s_rr *= inv; s_s *= inv; s_ss *= inv; s_rs *= inv;
  const float var_r = s_rr - s_r * s_r;
  const float var_s = s_ss - s_s * s_s;
  if (var_r < 1e-5f || var_s < 1e-5f) return 2.0f;
  const float cov = s_rs - s_r * s_s;
  const float vrs = std::sqrt(var_r * var_s);
  return std::fmax(0.0f, std::fmin(2.0f, 1.0f - cov / vrs));
}

// ComputeBilateralNCCOld, DPE.cu:696-782.
// Evaluation order: the hypothesis-invariant reference half of the window (bilateral weights,
// weighted reference moments) is summed first, tap by tap; each source tap is then placed at its
// float offset from the window centre projected in double (window_projection).  This is the same mathematics as the
// reference's per-row loop (and the same order as the CUDA kernels); g_raw_moments selects the
// reference's own loop order and raw moments instead.
static float ncc_strong(const Ctx &c, int px, int py, int src, const f4 &pl) {
  const dpe_camera &sc = c.cam[src];
  const float center = c.img[0].texel(px, py);
  const int r = c.P.strong_radius, inc = c.P.strong_increment;
  if (g_raw_moments) {
    float H[9];
    c.homography(src, pl, H);
    const f2 pt = project(H, px, py);
    if (pt.x >= sc.width || pt.x < 0.0f || pt.y >= sc.height || pt.y < 0.0f) return 2.0f;
    return window_ncc(c, H, c.img[src], px, py, r, inc, center);
  }
  WinProj wp;
  if (!window_projection(c.hbase[src], sc, c.W, c.H, pl, px, py, wp)) return 2.0f;
  float w[64], wr[64];
  float sw = 0.f, swr = 0.f, swrr = 0.f;
  int k = 0;
  for (int i = -r; i <= r; i += inc)
    for (int j = -r; j <= r; j += inc) {
      const float rp = c.img[0].texel(px + i, py + j);
      const float wt = bilateral_weight((float)i, (float)j, rp, center, c.P.sigma_spatial, c.P.sigma_color);
      const float rc = rp - center;
      w[k] = wt;
      wr[k] = wt * rc;
      sw += wt; swr += wt * rc; swrr += wt * rc * rc;
      ++k;
    }
  const float inv = 1.0f / sw;
  const float mean_r = swr * inv;
  const float var_r = swrr * inv - mean_r * mean_r;
  float s_s = 0.f, s_ss = 0.f, s_rs = 0.f;
  k = 0;
  for (int i = -r; i <= r; i += inc) {
    const float dx = (float)i;
    const float cx = wp.g0 * dx, cy = wp.g3 * dx, cz = wp.h6 * dx + wp.zc;
    for (int j = -r; j <= r; j += inc) {
      const float dy = (float)j;
      const float X = wp.g1 * dy + cx, Y = wp.g4 * dy + cy, Z = wp.h7 * dy + cz;
      const float iz = 1.0f / Z;
      const float sv = c.img[src].bilinear_off(wp, wp.fu + X * iz, wp.fv + Y * iz) - center;
      const float ws = w[k] * sv;
      s_s += ws;
      s_ss += ws * sv;
      s_rs += wr[k] * sv;
      ++k;
    }
  }
  const float m_s = s_s * inv;
  const float var_s = s_ss * inv - m_s * m_s;
  if (var_r < 1e-5f || var_s < 1e-5f) return 2.0f;
  const float cov = s_rs * inv - mean_r * m_s;
  return std::fmax(0.0f, std::fmin(2.0f, 1.0f - cov / std::sqrt(var_r * var_s)));
}

// ComputeBilateralNCCNew (deformable window), DPE.cu:561-694
static float ncc_weak(const Ctx &c, int px, int py, int src, const f4 &pl) {
  float H[9];
  c.homography(src, pl, H);
  const f2 pt = project(H, px, py);
  const dpe_camera &sc = c.cam[src];
  if (pt.x >= sc.width || pt.x < 0.0f || pt.y >= sc.height || pt.y < 0.0f) return 2.0f;
  const int center = px + py * c.W;
  const float ref_center = c.img[0].texel(px, py);
  float center_cost = 0.0f, strong_cost = 0.0f;
  int strong_count = 0;
  for (int k = 0; k < DPE_NEIGHBOUR_NUM; ++k) {
    const s2 nb = c.neighbour(center, k);
    if (nb.x == -1 || nb.y == -1) continue;
    const f2 np = project(H, nb.x, nb.y);
    if (np.x < 0 || np.y < 0 || np.x >= c.W || np.y >= c.H) {
      if (k != 0) {
        if (isSet(c.views_at((long)nb.x + (long)nb.y * c.W), src - 1)) { strong_cost += 2.0f; strong_count++; }
        continue;
      }
      return 2.0f;
    }
    int radius = k == 0 ? c.P.strong_radius : c.P.weak_radius;
    int inc = k == 0 ? c.P.strong_increment : c.P.weak_increment;
    if (c.P.use_radius && k == 0) {
      radius = c.radius[center];
      inc = CV_MAX(2, f2i(2.0 * radius / 5.0));
    }
    const float t = window_ncc(c, H, c.img[src], nb.x, nb.y, radius, inc, ref_center);
    if (k == 0) center_cost = t;
    else { strong_cost += t; strong_count++; }
  }
  if (strong_count == 0) return center_cost;
  strong_cost /= strong_count;
  strong_cost = CV_MIN(strong_cost, 2.0f);
  return (float)(0.25 * center_cost + 0.75 * strong_cost);
}

// ComputeGeomConsistencyCost, DPE.cu:919-957
static float geom_cost(const Ctx &c, int px, int py, int src, const f4 &pl) {
  const dpe_camera &rc = c.cam[0], &sc = c.cam[src];
  const float depth = depth_from_plane(rc, pl, px, py);
  const f3 fw = point_world((float)px, (float)py, depth, rc);
  f2 sp; float sd;
  project_camera(fw, sc, sp, sd);
  const float src_depth = c.dep[src].texel(f2i(sp.x), f2i(sp.y));
  if (src_depth == 0.0f) return 3.0f;
  const f3 sw = point_world(sp.x, sp.y, src_depth, sc);
  f2 bp; float rd;
  project_camera(sw, rc, bp, rd);
  const float dx = (float)px - bp.x, dy = (float)py - bp.y;
  return std::fmin(3.0f, std::sqrt(dx * dx + dy * dy));
}

static void cost_vector_strong(const Ctx &c, int px, int py, const f4 &pl, float *cv) {
  for (int i = 1; i < c.P.num_images; ++i) cv[i - 1] = ncc_strong(c, px, py, i, pl);
}
static void cost_vector_weak(const Ctx &c, int px, int py, const f4 &pl, float *cv) {
  for (int i = 1; i < c.P.num_images; ++i) cv[i - 1] = ncc_weak(c, px, py, i, pl);
}

static int find_min_cost_index(const float *costs, int n) {
  float m = costs[0];
  int idx = 0;
  for (int i = 1; i < n; ++i)
    if (costs[i] <= m) { m = costs[i]; idx = i; }
  return idx;
}

static void sort_small(float *d, int n) {
  for (int i = 1; i < n; ++i) {
    const float t = d[i];
    int j;
    for (j = i; j >= 1 && t < d[j - 1]; j--) d[j] = d[j - 1];
    d[j] = t;
  }
}

// ----------------------------------------------------------------------------- RandomInitialization
// DPE.cu:784-830
static float initial_cost_and_views(Ctx &c, int px, int py) {
  const int center = px + py * c.W;
  const f4 pl = c.plane[center];
  float cv[32] = {2.0f}, cvc[32] = {2.0f};
  int cnt = 0, valid = 0;
  for (int i = 1; i < c.P.num_images; ++i) {
    const float v = ncc_strong(c, px, py, i, pl);
    cv[i - 1] = v; cvc[i - 1] = v; cnt++;
    if (v < 2.0f) valid++;
  }
  sort_small(cv, cnt);
  c.views[center] = 0;
  const int k = std::min(valid, c.P.top_k);
  if (k > 0) {
    float cost = 0.0f;
    for (int i = 0; i < k; ++i) cost += cv[i];
    const float thr = cv[k - 1];
    for (int i = 0; i < c.P.num_images - 1; ++i)
      if (cvc[i] <= thr) setBit(&c.views[center], i);
    return cost / k;
  }
  return 2.0f;
}
// DPE.cu:832-861
static float initial_cost_selected(Ctx &c, int px, int py) {
  const int center = px + py * c.W;
  const f4 pl = c.plane[center];
  int cnt = 0;
  float cost = 0.0f;
  for (int i = 1; i < c.P.num_images; ++i) {
    if (isSet(c.views[center], i - 1)) {
      const float v = ncc_strong(c, px, py, i, pl);
      if (v < 2.0f) { cnt++; cost += v; }
      else unSetBit(&c.views[center], i - 1);
    }
  }
  return cnt == 0 ? 2.0f : cost / cnt;
}
// DPE.cu:1039-1067
static void random_initialization(Ctx &c, int px, int py) {
  const int center = px + py * c.W;
  const dpe_camera &rc = c.cam[0];
  if (c.P.state == DPE_FIRST_INIT) {
    PixelRng rng = c.rng(center);
    const float depth = rng.uniform() * (c.P.depth_max - c.P.depth_min) + c.P.depth_min;
    f4 pl = random_normal(rc, px, py, rng, depth);
    pl.w = dist_to_origin(rc, px, py, depth, pl);
    c.plane[center] = pl;
    c.cost[center] = initial_cost_and_views(c, px, py);
  } else {
    f4 pl = normal_to_ref(rc, c.plane[center]);
    const float depth = pl.w;
    pl.w = dist_to_origin(rc, px, py, depth, pl);
    c.plane[center] = pl;
    c.cost[center] = initial_cost_selected(c, px, py);
  }
}

// ----------------------------------------------------------------------------- view sampling
// The multi-hypothesis joint view selection shared by both propagation kernels
// (DPE.cu:1551-1619 and :1714-1783).  Returns weight_norm, fills vw and the sampled mask.
static float sample_views(Ctx &c, int center, int iter, const float cost_array[8][32], const float *priors,
                          uint8_t *vw, uint32_t *temp_sel) {
  const int n = c.P.num_images - 1;
  for (int i = 0; i < DPE_MAX_IMAGES; ++i) vw[i] = 0;
  float probs[32] = {0.0f};
  const float thr = (float)(0.8 * (double)dpe::dpe_expf((float)(iter * iter) / (-90.0f)));
  for (int i = 0; i < n; ++i) {
    float count = 0;
    int count_false = 0;
    float tmpw = 0;
    for (int j = 0; j < 8; ++j) {
      const float v = cost_array[j][i];
      if (v < thr) { tmpw += dpe::dpe_expf(v * v / (-0.18f)); count++; }
      if (v > 1.2f) count_false++;
    }
    if (count > 2 && count_false < 3) probs[i] = tmpw / count;
    else if (count_false < 3) probs[i] = dpe::dpe_expf(thr * thr / (-0.32f));
    probs[i] = probs[i] * priors[i];
  }
  // TransformPDFToCDF, DPE.cu:297-311
  float sum = 0.0f;
  for (int i = 0; i < n; ++i) sum += probs[i];
  const float inv = 1.0f / sum;
  float cum = 0.0f;
  for (int i = 0; i < n; ++i) { cum += probs[i] * inv; probs[i] = cum; }
  PixelRng rng = c.rng(center);
  for (int s = 0; s < 15; ++s) {
    const float r = rng.uniform() - FLT_EPSILON;
    for (int id = 0; id < n; ++id)
      if (probs[id] > r) { vw[id] += 1; break; }
  }
  *temp_sel = 0;
  float wn = 0;
  for (int i = 0; i < n; ++i)
    if (vw[i] > 0) { setBit(temp_sel, i); wn += vw[i]; }
  return wn;
}

// PlaneHypothesisRefinementStrong / the random half of ...Weak (DPE.cu:1069-1122, :1173-1215)
static void random_refine(Ctx &c, int px, int py, f4 *pl, float *depth, float *cost, const uint8_t *vw, float wn,
                          bool weak) {
  const dpe_camera &rc = c.cam[0];
  const float dmin = c.P.depth_min, dmax = c.P.depth_max;
  const int center = px + py * c.W;
  PixelRng rng = c.rng(center);
  const float depth_rand = rng.uniform() * (dmax - dmin) + dmin;
  const f4 n_rand = random_normal(rc, px, py, rng, *depth);
  const float lo = (1 - 0.02f) * *depth, hi = (1 + 0.02f) * *depth;
  const float depth_pert = rng.uniform() * (hi - lo) + lo;  // do..while runs once (quirk Q7)
  const f4 n_pert = perturbed_normal(rc, px, py, *pl, rng, (float)(0.02f * 3.14159265358979323846));
  const float depths[5] = {depth_rand, *depth, depth_rand, *depth, depth_pert};
  const f4 normals[5] = {*pl, n_rand, n_rand, n_pert, *pl};
  const int n = c.P.num_images - 1;
  for (int i = 0; i < 5; ++i) {
    float cv[32] = {2.0f};
    f4 t = normals[i];
    t.w = dist_to_origin(rc, px, py, depths[i], t);
    if (weak) cost_vector_weak(c, px, py, t, cv);
    else cost_vector_strong(c, px, py, t, cv);
    float tc = 0.0f;
    for (int j = 0; j < n; ++j) {
      if (vw[j] > 0) {
        if (weak && c.P.geom_consistency) tc += vw[j] * (cv[j] + c.P.geom_factor * geom_cost(c, px, py, j + 1, t));
        else tc += vw[j] * cv[j];
      }
    }
    tc /= wn;
    const float db = depth_from_plane(rc, t, px, py);
    if (db >= dmin && db <= dmax && tc < *cost) { *depth = db; *pl = t; *cost = tc; }
  }
}

// ----------------------------------------------------------------------------- strong update
static const int kDir[8][2] = {{0, -1}, {0, 1}, {-1, 0}, {1, 0}, {-1, -1}, {1, 1}, {-1, 1}, {1, -1}};

// CheckerboardPropagationStrong, DPE.cu:1218-1670
static void strong_update(Ctx &c, int px, int py, int iter) {
  const int W = c.W, H = c.H, n = c.P.num_images - 1;
  const int center = py * W + px;
  const dpe_camera &rc = c.cam[0];
  float cost_array[8][32] = {{2.0f}};
  bool flag[8] = {false};
  int positions[8] = {0};
  // candidate planes are read from `src_plane`/`src_cost`: the live arrays (non-edge branch, only
  // opposite-colour pixels) or the pre-pass snapshot (edge branch, see header).  With
  // g_serial_race the edge branch reads the live arrays too, in a serial raster-order pass.
  const bool snap = c.P.use_edge && !g_serial_race;
  const std::vector<f4> &cand_plane = snap ? c.plane_snap : c.plane;
  const std::vector<float> &cand_cost = snap ? c.cost_snap : c.cost;

  if (c.P.use_edge) {
    const s2 *en = &c.edge_neigh[(size_t)center * 8];
    const float max_edge_dist = CV_MAX(H, W) / 30.0f;
    const int min_step = 2;
    for (int d = 0; d < 8; ++d) {
      const int dx = kDir[d][0], dy = kDir[d][1];
      const int sx = CV_MAX(1, 5 - 2 * iter) * dx, sy = CV_MAX(1, 5 - 2 * iter) * dy;
      const s2 e = en[d];
      float dist = (float)std::sqrt(std::pow((double)(e.x - px), 2) + std::pow((double)(e.y - py), 2));
      if (d >= 4) dist = (float)(dist / std::sqrt(2.0));
      if (c.edge[center]) dist = 11 * min_step;
      else if (e.x == -1 || e.y == -1 || dist > max_edge_dist) {
        dist = max_edge_dist;
        if (d >= 4) dist = (float)(dist / std::sqrt(2.0));
      }
      const int step_num = CV_MIN(CV_MAX(11, f2i(1.0f * dist / min_step)), 22);
      int step_len = CV_MAX(f2i(1.0f * dist / step_num), min_step);
      if (d < 4 && step_len % 2 == 1) step_len -= 1;
      float mc = FLT_MAX;
      int mp = -1;
      for (int s = 0; s < step_num; ++s) {
        int fx = 0, fy = 0;
        if (d > 4) { if (d % 2) fx = dx; else fy = dy; }
        const int tx = px + sx + s * step_len * dx + fx, ty = py + sy + s * step_len * dy + fy;
        if (!(tx >= 0 && ty >= 0 && tx < W && ty < H)) continue;
        const int tc = tx + ty * W;
        if (mc > cand_cost[tc]) { mp = tc; mc = cand_cost[tc]; }
      }
      if (mc < FLT_MAX) {
        flag[d] = true;
        positions[d] = mp;
        cost_vector_strong(c, px, py, cand_plane[mp], cost_array[d]);
      }
    }
    if (!c.edge[center]) {
      const float good_thr = 0.8f * dpe::dpe_expf((float)(iter * iter) / (-90.0f));
      const float bad_thr = 1.2f;
      for (int d = 0; d < 8; ++d) {
        const int dx = kDir[d][0], dy = kDir[d][1];
        const int sx = CV_MAX(1, 5 - 2 * iter) * dx, sy = CV_MAX(1, 5 - 2 * iter) * dy;
        const bool had = flag[d];
        float tca[32] = {2.0f};
        float mc = FLT_MAX;
        int mp = -1;
        for (int s = 0; s < 11; ++s) {
          int fx = 0, fy = 0;
          if (d > 4) { if (d % 2) fx = dx; else fy = dy; }
          const int tx = px + sx + s * min_step * dx + fx, ty = py + sy + s * min_step * dy + fy;
          if (!(tx >= 0 && ty >= 0 && tx < W && ty < H)) continue;
          const int tc = tx + ty * W;
          if (mc > cand_cost[tc]) { mp = tc; mc = cand_cost[tc]; }
        }
        if (mc < FLT_MAX) {
          flag[d] = true;
          cost_vector_strong(c, px, py, cand_plane[mp], tca);
          int good[2] = {0, 0}, bad[2] = {0, 0};
          for (int i = 0; i < 2; ++i)
            for (int j = 0; j < n; ++j) {
              const float v = i == 0 ? cost_array[d][j] : tca[j];
              if (v < good_thr) good[i]++;
              if (v > bad_thr) bad[i]++;
            }
          if (!had || good[1] > good[0] || (good[1] == good[0] && bad[1] < bad[0])) {
            positions[d] = mp;
            for (int j = 0; j < n; ++j) cost_array[d][j] = tca[j];
          }
        }
      }
    }
  } else {
    // 0 up_near, 1 up_far, 2 down_near, 3 down_far, 4 left_near, 5 left_far, 6 right_near, 7 right_far
    auto far_search = [&](int slot, bool ok, int start, int stride, auto cond) {
      if (!ok) return;
      flag[slot] = true;
      float m = c.cost[start];
      int mp = start;
      for (int i = 1; i < 11; ++i)
        if (cond(i)) {
          const int t = start + 2 * i * stride;
          if (c.cost[t] < m) { m = c.cost[t]; mp = t; }
        }
      positions[slot] = mp;
      cost_vector_strong(c, px, py, c.plane[mp], cost_array[slot]);
    };
    far_search(1, py > 2, center - 3 * W, -W, [&](int i) { return py > 2 + 2 * i; });
    far_search(3, py < H - 3, center + 3 * W, W, [&](int i) { return py < H - 3 - 2 * i; });
    far_search(5, px > 2, center - 3, -1, [&](int i) { return px > 2 + 2 * i; });
    far_search(7, px < W - 3, center + 3, 1, [&](int i) { return px < W - 3 - 2 * i; });
    auto near_search = [&](int slot, bool ok, int start, auto cand) {
      if (!ok) return;
      flag[slot] = true;
      float m = c.cost[start];
      int mp = start;
      for (int i = 0; i < 3; ++i)
        for (int side = 0; side < 2; ++side) {
          int t;
          if (cand(i, side, &t) && c.cost[t] < m) { m = c.cost[t]; mp = t; }
        }
      positions[slot] = mp;
      cost_vector_strong(c, px, py, c.plane[mp], cost_array[slot]);
    };
    const int un = center - W, dn = center + W, ln = center - 1, rn = center + 1;
    near_search(0, py > 0, un, [&](int i, int side, int *t) {
      if (side == 0) { *t = un - (1 + i) * W - (1 + i); return py > 1 + i && px > i; }
      *t = un - (1 + i) * W + (1 + i); return py > 1 + i && px < W - 1 - i;
    });
    near_search(2, py < H - 1, dn, [&](int i, int side, int *t) {
      if (side == 0) { *t = dn + (1 + i) * W - (1 + i); return py < H - 2 - i && px > i; }
      *t = dn + (1 + i) * W + (1 + i); return py < H - 2 - i && px < W - 1 - i;
    });
    near_search(4, px > 0, ln, [&](int i, int side, int *t) {
      if (side == 0) { *t = ln - (1 + i) - (1 + i) * W; return px > 1 + i && py > i; }
      *t = ln - (1 + i) + (1 + i) * W; return px > 1 + i && py < H - 1 - i;
    });
    near_search(6, px < W - 1, rn, [&](int i, int side, int *t) {
      if (side == 0) { *t = rn + (1 + i) - (1 + i) * W; return px < W - 2 - i && py > i; }
      *t = rn + (1 + i) + (1 + i) * W; return px < W - 2 - i && py < H - 1 - i;
    });
  }

  // view priors from the four direct neighbours (DPE.cu:1556-1570)
  float priors[32] = {0.0f};
  const long nbr[4] = {(long)center - W, (long)center + W, (long)center - 1, (long)center + 1};
  for (int i = 0; i < 4; ++i)
    if (flag[2 * i]) {
      const uint32_t sv = c.views_at(nbr[i]);
      for (int j = 0; j < n; ++j) priors[j] += isSet(sv, j) == 1 ? 0.9f : 0.1f;
    }
  uint8_t *vw = &c.vweight[(size_t)center * DPE_MAX_IMAGES];
  uint32_t temp_sel = 0;
  const float wn = sample_views(c, center, iter, cost_array, priors, vw, &temp_sel);

  float final_costs[8] = {0.0f};
  for (int i = 0; i < 8; ++i) {
    for (int j = 0; j < n; ++j)
      if (vw[j] > 0) final_costs[i] += vw[j] * cost_array[i][j];
    final_costs[i] /= wn;
  }
  const int mi = find_min_cost_index(final_costs, 8);
  float cvn[32] = {2.0f};
  cost_vector_strong(c, px, py, c.plane[center], cvn);
  float cost_now = 0.0f;
  for (int i = 0; i < n; ++i) cost_now += vw[i] * cvn[i];
  cost_now /= wn;
  const float cost_written = cost_now;  // costs[center] = cost_now (DPE.cu:1643)
  c.cost[center] = cost_written;
  float depth_now = depth_from_plane(rc, c.plane[center], px, py);
  f4 pl_now = c.plane[center];
  if (flag[mi]) {
    const f4 &cand = c.P.use_edge ? cand_plane[positions[mi]] : c.plane[positions[mi]];
    const float db = depth_from_plane(rc, cand, px, py);
    if (db >= c.P.depth_min && db <= c.P.depth_max && final_costs[mi] < cost_now) {
      depth_now = db; pl_now = cand; cost_now = final_costs[mi];
      c.views[center] = temp_sel;
    }
  }
  random_refine(c, px, py, &pl_now, &depth_now, &cost_now, vw, wn, false);
  if (c.P.state == DPE_REFINE_INIT) {
    if ((double)cost_now < (double)cost_written - 0.1) { c.cost[center] = cost_now; c.plane[center] = pl_now; }
  } else {
    c.cost[center] = cost_now;
    c.plane[center] = pl_now;
  }
}

// ----------------------------------------------------------------------------- weak update
// PlaneHypothesisRefinementWeak, DPE.cu:1124-1216
static void weak_refine(Ctx &c, int px, int py, f4 *pl, float *depth, float *cost, const uint8_t *vw, float wn) {
  const int center = px + py * c.W;
  const dpe_camera &rc = c.cam[0];
  const int n = c.P.num_images - 1;
  if (c.weak[center] == DPE_WEAK) {
    const f4 fp = c.fit_plane[center];
    if (fp.x == 0 && fp.y == 0 && fp.z == 0) return;
    float cv[32] = {2.0f};
    cost_vector_weak(c, px, py, fp, cv);
    float tc = 0.0f;
    for (int j = 0; j < n; ++j)
      if (vw[j] > 0) {
        if (c.P.geom_consistency) tc += vw[j] * (cv[j] + c.P.geom_factor * geom_cost(c, px, py, j + 1, fp));
        else tc += vw[j] * cv[j];
      }
    tc /= wn;
    const float db = depth_from_plane(rc, fp, px, py);
    if (db >= c.P.depth_min && db <= c.P.depth_max && tc < *cost) { *depth = db; *pl = fp; *cost = tc; }
  }
  random_refine(c, px, py, pl, depth, cost, vw, wn, true);
}

// CheckerboardPropagationWeak, DPE.cu:1672-1866
static void weak_update(Ctx &c, int px, int py, int iter) {
  const int W = c.W, n = c.P.num_images - 1;
  const int center = py * W + px;
  const dpe_camera &rc = c.cam[0];
  float cost_array[8][32] = {{2.0f}};
  bool flag[8] = {false};
  int positions[8] = {0};
  f4 cand[8] = {};
  for (int i = 0; i < 8; ++i) {
    const s2 nb = c.neighbour(center, i + 1);
    if (nb.x == -1 || nb.y == -1 || c.weak[nb.x + nb.y * W] != DPE_STRONG) { flag[i] = false; continue; }
    positions[i] = nb.x + nb.y * W;
    flag[i] = true;
    cost_vector_weak(c, px, py, c.plane[positions[i]], cost_array[i]);
    cand[i] = c.plane[positions[i]];
  }
  float priors[32] = {0.0f};
  for (int i = 0; i < 8; ++i) {
    const s2 nb = c.neighbour(center, i + 1);
    if (nb.x == -1 || nb.y == -1) continue;
    const uint32_t sv = c.views[nb.x + nb.y * W];
    for (int j = 0; j < n; ++j) priors[j] += isSet(sv, j) == 1 ? 0.9f : 0.1f;
  }
  uint8_t *vw = &c.vweight[(size_t)center * DPE_MAX_IMAGES];
  uint32_t temp_sel = 0;
  const float wn = sample_views(c, center, iter, cost_array, priors, vw, &temp_sel);
  float final_costs[8] = {0.0f};
  for (int i = 0; i < 8; ++i) {
    for (int j = 0; j < n; ++j)
      if (vw[j] > 0) {
        if (c.P.geom_consistency) {
          if (flag[i]) final_costs[i] += vw[j] * (cost_array[i][j] + c.P.geom_factor * geom_cost(c, px, py, j + 1, c.plane[positions[i]]));
          else final_costs[i] += vw[j] * (cost_array[i][j] + c.P.geom_factor * 3.0f);
        } else {
          final_costs[i] += vw[j] * cost_array[i][j];
        }
      }
    final_costs[i] /= wn;
  }
  const int mi = find_min_cost_index(final_costs, 8);
  float cvn[32] = {2.0f};
  cost_vector_weak(c, px, py, c.plane[center], cvn);
  float cost_now = 0.0f;
  for (int i = 0; i < n; ++i) {
    if (c.P.geom_consistency) cost_now += vw[i] * (cvn[i] + c.P.geom_factor * geom_cost(c, px, py, i + 1, c.plane[center]));
    else cost_now += vw[i] * cvn[i];
  }
  cost_now /= wn;
  const float cost_written = cost_now;
  c.cost[center] = cost_written;
  float depth_now = depth_from_plane(rc, c.plane[center], px, py);
  f4 pl_now = c.plane[center];
  if (flag[mi]) {
    const float db = depth_from_plane(rc, cand[mi], px, py);
    if (db >= c.P.depth_min && db <= c.P.depth_max && final_costs[mi] < cost_now) {
      depth_now = db; pl_now = cand[mi]; cost_now = final_costs[mi];
      c.views[center] = temp_sel;
    }
  }
  weak_refine(c, px, py, &pl_now, &depth_now, &cost_now, vw, wn);
  if (c.P.state == DPE_REFINE_INIT) {
    if ((double)cost_now < (double)cost_written - 0.1) { c.cost[center] = cost_now; c.plane[center] = pl_now; }
  } else {
    c.cost[center] = cost_now;
    c.plane[center] = pl_now;
  }
  // final re-cost with the strong window (DPE.cu:1849-1865); the radius swap has no effect on it
  float cv2[32] = {2.0f};
  cost_vector_strong(c, px, py, c.plane[center], cv2);
  float cn = 0.0f;
  for (int i = 0; i < n; ++i) cn += vw[i] * cv2[i];
  cn /= wn;
  c.cost[center] = cn;
}

// ----------------------------------------------------------------------------- support kernels
// BresenhamLine, DPE.cu:162-248
static bool bresenham(const Ctx &c, int ax, int ay, int bx, int by) {
  if (c.edge_at((long)ax + (long)ay * c.W) || c.edge_at((long)bx + (long)by * c.W)) return false;
  const float scale_x = 1.0f * c.lowW / (float)c.W;
  const float scale_y = 1.0f * c.lowH / (float)c.H;
  const int h = c.lowH, w = c.lowW;
  const int max_step = c.P.high_res_img ? (int)std::round(CV_MAX(h, w) / 60.0) : CV_MAX(h, w);
  for (int pass = 0; pass < 2; ++pass) {
    const int fx = pass == 0 ? bx : ax, fy = pass == 0 ? by : ay;
    const int tx = pass == 0 ? ax : bx, ty = pass == 0 ? ay : by;
    int x0 = (int)CV_MIN(std::round(fx * scale_x), (float)(w - 1));
    int y0 = (int)CV_MIN(std::round(fy * scale_y), (float)(h - 1));
    const int x1 = (int)CV_MIN(std::round(tx * scale_x), (float)(w - 1));
    const int y1 = (int)CV_MIN(std::round(ty * scale_y), (float)(h - 1));
    const int dx = std::abs(x1 - x0), sx = x0 < x1 ? 1 : -1;
    const int dy = std::abs(y1 - y0), sy = y0 < y1 ? 1 : -1;
    int err = (dx > dy ? dx : dy) / 2;
    int step = 0;
    bool tagx = true, tagy = true;
    while (tagx || tagy) {
      if (x0 == x1) tagx = false;
      if (y0 == y1) tagy = false;
      const int e2 = err;
      if (e2 > -dx) { err -= dy; x0 += sx; }
      if (e2 < dy) { err += dx; y0 += sy; }
      if (c.edge_low_at((long)x0 + (long)y0 * w)) return true;
      step += 1;
      if (step >= max_step) break;
    }
  }
  return false;
}

// GenEdgeInform, DPE.cu:2487-2595
static void gen_edge_inform(Ctx &c, int px, int py) {
  const int W = c.W, H = c.H, center = px + py * W;
  if (c.P.use_edge) {
    s2 *en = &c.edge_neigh[(size_t)center * 8];
    for (int i = 0; i < 8; ++i) {
      en[i] = {-1, -1};
      const int dx = kDir[i][0], dy = kDir[i][1];
      int nx = px + dx, ny = py + dy;
      while (nx >= 0 && nx < W && ny >= 0 && ny < H) {
        if (c.edge[nx + ny * W]) { en[i] = {(int16_t)nx, (int16_t)ny}; break; }
        nx += dx; ny += dy;
      }
    }
    const int r = c.P.strong_radius;
    int edge_pix = 0, tot_pix = 0;
    for (int i = -r; i <= r; ++i)
      for (int j = -r; j <= r; ++j) {
        const int nx = px + i, ny = py + j;
        if (nx < 0 || nx >= W || ny < 0 || ny >= H) continue;
        if (c.edge[ny * W + nx]) edge_pix++;
        tot_pix++;
      }
    float density = 1.0f * edge_pix / tot_pix;
    if (c.P.use_label) {
      int bound_pix = 0;
      for (int i = -r; i <= r; ++i)
        for (int j = -r; j <= r; ++j) {
          const int nx = px + i, ny = py + j;
          if (nx < 0 || nx >= W || ny < 0 || ny >= H) continue;
          if (c.label[ny * W + nx] == 0) bound_pix++;
        }
      density = CV_MAX(density, bound_pix / tot_pix);  // integer division (quirk Q6)
    }
    c.complexity[center] = (float)(1.0f / (1.0f + std::exp(-25.0 * (density - 0.35))));
  }
  if (c.P.use_label && c.weak[center] == DPE_WEAK) {
    s2 *lb = &c.lab_bound[(size_t)c.nmap[center] * 8];
    const int cl = c.label[center];
    if (cl > 0) {
      for (int i = 0; i < 8; ++i) {
        const int dx = kDir[i][0], dy = kDir[i][1];
        int nx = px + dx, ny = py + dy, lx = -1, ly = -1;
        while (nx >= 0 && nx < W && ny >= 0 && ny < H) {
          const int nl = c.label[nx + ny * W];
          if (nl == cl) { lx = nx; ly = ny; }
          else if (nl == -1) break;
          nx += dx; ny += dy;
        }
        lb[i] = {(int16_t)lx, (int16_t)ly};
      }
    }
  }
}

// FindNearestStrongPoint, DPE.cu:2859-2893
static void find_nearest_strong(Ctx &c, int px, int py) {
  const int W = c.W, H = c.H, center = px + py * W;
  c.nearest[center] = {-1, -1};
  if (c.weak[center] != DPE_WEAK) return;
  for (int r = 0; r <= 100; ++r)
    for (int x = -r; x <= r; ++x)
      for (int y = -r; y <= r; ++y) {
        if (std::abs(x) != r && std::abs(y) != r) continue;
        const int nx = px + x, ny = py + y;
        if (nx < 0 || ny < 0 || nx >= W || ny >= H) continue;
        if (c.weak[nx + ny * W] == DPE_STRONG) { c.nearest[center] = {(int16_t)nx, (int16_t)ny}; return; }
      }
}

// GenNeighbours, DPE.cu:2107-2467
static void gen_neighbours(Ctx &c, int px, int py) {
  const int W = c.W, H = c.H, center = px + py * W;
  if (c.weak[center] != DPE_WEAK) return;
  const int kMaxPts = 64, margin = 6;
  const float depth_diff = c.P.depth_max - c.P.depth_min;
  const dpe_camera &cam = c.cam[0];
  PixelRng rng = c.rng(center);
  s2 *nbs = &c.neigh[(size_t)c.nmap[center] * DPE_NEIGHBOUR_NUM];
  for (int i = 0; i < DPE_NEIGHBOUR_NUM; ++i) nbs[i] = {-1, -1};
  nbs[0] = {(int16_t)px, (int16_t)py};
  s2 pts[kMaxPts];
  bool valid[kMaxPts];
  for (int i = 0; i < kMaxPts; ++i) { pts[i] = {-1, -1}; valid[i] = false; }
  int odi = -1, npts = 0;
  const int rt = c.P.rotate_time;
  // the angle arithmetic promotes to double through M_PI (DPE.cu:2152-2156)
  const float angle = 45.0f / rt;
  const float cos_a = (float)std::cos(angle * 3.14159265358979323846 / 180.f);
  const float sin_a = (float)std::sin(angle * 3.14159265358979323846 / 180.f);
  const float thr = (float)std::cos((angle / 2.0f) * 3.14159265358979323846 / 180.0f);
  const int shift_range = CV_MAX(f2i(std::tan((angle / 2.0f) * 3.14159265358979323846 / 180.0f) * 20), 1);
  const float ransac_thr = c.P.ransac_threshold * depth_diff;
  bool edge_limit = false;
  if (c.P.use_limit) {
    edge_limit = true;
    if (c.P.use_edge) {
      const float cv = c.complexity[center];
      const float rp = rng.uniform() - FLT_EPSILON;
      if (rp < cv) edge_limit = false;
      else c.complexity[center] = CV_MAX(0.99f, cv);
    }
  }
  for (int odx = -1; odx <= 1; ++odx)
    for (int ody = -1; ody <= 1; ++ody) {
      if (odx == 0 && ody == 0) continue;
      f2 od = {(float)odx, (float)ody};
      normalize2(&od);
      odi++;
      for (int ri = 0; ri < rt; ++ri) {
        const int di = odi * 4 + ri;
        for (int radius = 2; radius <= 4096; radius = CV_MIN(radius * 2, radius + 25)) {
          const f2 tp = {px + od.x * radius, py + od.y * radius};
          if (tp.x < 0 || tp.y < 0 || tp.x >= W || tp.y >= H) break;
          for (int k = 0; k < 4; ++k) {
            // ((sign) * curand()) % shift_range evaluated in unsigned arithmetic, sign drawn first
            uint32_t sgn = (rng.next_u32() % 2 == 0) ? 1u : 0xFFFFFFFFu;
            const int rxs = (int)((sgn * rng.next_u32()) % (uint32_t)shift_range);
            sgn = (rng.next_u32() % 2 == 0) ? 1u : 0xFFFFFFFFu;
            const int rys = (int)((sgn * rng.next_u32()) % (uint32_t)shift_range);
            f2 dir = {od.x * 20 + rxs, od.y * 20 + rys};
            normalize2(&dir);
            s2 nb = {(int16_t)f2i(px + dir.x * radius), (int16_t)f2i(py + dir.y * radius)};
            if (nb.x < margin || nb.y < margin || nb.x >= W - margin || nb.y >= H - margin) continue;
            int nbc = nb.x + nb.y * W;
            if (c.weak[nbc] != DPE_STRONG) {
              nb = c.nearest[nbc];
              if (nb.x == -1 || nb.y == -1) continue;
              nbc = nb.x + nb.y * W;
            }
            f2 td = {(float)(nb.x - px), (float)(nb.y - py)};
            normalize2(&td);
            const float ca = td.x * od.x + td.y * od.y;
            if (ca > thr && (!edge_limit || !bresenham(c, px, py, nb.x, nb.y))) {
              pts[di] = nb; valid[di] = true; npts++;
              break;
            }
          }
          if (valid[di]) break;
        }
        f2 rd = {od.x * cos_a - od.y * sin_a, od.x * sin_a + od.y * cos_a};
        normalize2(&rd);
        od = rd;
      }
    }
  int ext = 31;
  if (c.P.use_label && c.label[center] > 0) {
    const s2 *lb = &c.lab_bound[(size_t)c.nmap[center] * 8];
    float bd[8] = {0};
    int ds[8] = {0};
    for (int i = 0; i < 8; ++i) {
      const s2 b = lb[i];
      float dist = 0.0f;
      if (b.x != -1 && b.y != -1) {
        dist = (float)std::sqrt(std::pow((double)(px - b.x), 2) + std::pow((double)(py - b.y), 2));
        if (i >= 4) dist = (float)(dist / std::sqrt(2.0));
      }
      bd[i] = dist;
      if (i % 2 == 1) {
        const float od2 = bd[i - 1];
        const int step = CV_MIN(1, CV_MAX(2 * rt - 1, f2i(2 * rt * dist / (dist + od2))));  // quirk Q5
        ds[i - 1] = 2 * rt - step;
        ds[i] = step;
      }
    }
    for (int i = 0; i < 8; ++i) {
      const float dist = bd[i];
      const int gap = ds[i] + 1;
      const int step_len = CV_MAX(1, f2i(std::floor(1.0 * dist / gap)));
      for (int s = 1; s <= ds[i]; ++s) {
        s2 nb = {(int16_t)(px + s * step_len * kDir[i][0]), (int16_t)(py + s * step_len * kDir[i][1])};
        if (nb.x < margin || nb.y < margin || nb.x >= W - margin || nb.y >= H - margin) continue;
        int nbc = nb.x + nb.y * W;
        if (c.weak[nbc] != DPE_STRONG) {
          nb = c.nearest[nbc];
          if (nb.x == -1 || nb.y == -1) continue;
          nbc = nb.x + nb.y * W;
        }
        if (c.label[nbc] != 0 && c.label[nbc] != c.label[center]) continue;
        ext++;
        pts[ext] = nb; valid[ext] = true; npts++;
      }
    }
  }
  if (npts <= 3) { c.reliable[center] = 0; return; }

  s2 sv[kMaxPts];
  f3 sv3[kMaxPts], svn[kMaxPts];
  int vc = 0;
  float X[3];
  point3d(cam, px, py, c.plane[center].w, X);
  const f3 cw = {X[0], X[1], X[2]};
  for (int i = 0; i < kMaxPts; ++i) {
    sv[i] = {-1, -1};
    if (valid[i]) {
      const s2 sp = pts[i];
      const int spc = sp.x + sp.y * W;
      sv[vc] = sp;
      point3d(cam, sp.x, sp.y, c.plane[spc].w, X);
      sv3[vc] = {X[0], X[1], X[2]};
      const f4 n4 = normal_to_ref(cam, c.plane[spc]);
      svn[vc] = {n4.x, n4.y, n4.z};
      vc++;
    }
  }
  f4 best = {0, 0, 0, 0};
  bool has_valid = false;
  {
    int iteration = 50, max_iter = c.P.high_res_img ? 200 : 125, max_count = 3;
    float min_cost = FLT_MAX, residuals[kMaxPts] = {0.0f};
    float tthr = ransac_thr;
    bool has_consist = false;
    bool must_tri = (c.P.use_label && c.label[center] > 0 && edge_limit) ? false : true;
    while (iteration > 0 && max_iter > 0) {
      max_iter--;
      const int a = (int)(rng.next_u32() % (uint32_t)vc);
      const int b = (int)(rng.next_u32() % (uint32_t)vc);
      const int cc = (int)(rng.next_u32() % (uint32_t)vc);
      if (a == b || b == cc || a == cc) continue;
      if (must_tri && !point_in_triangle(sv[a], sv[b], sv[cc], px, py)) continue;
      if (edge_limit) {
        // the reference caches these tests in edge_test[][]; the test is a pure function
        if (bresenham(c, sv[a].x, sv[a].y, sv[b].x, sv[b].y) || bresenham(c, sv[b].x, sv[b].y, sv[cc].x, sv[cc].y) ||
            bresenham(c, sv[cc].x, sv[cc].y, sv[a].x, sv[a].y))
          continue;
      }
      bool nc = false;
      if (c.P.geom_consistency && edge_limit) {
        const f3 &AN = svn[a], &BN = svn[b], &CN = svn[cc];
        nc = true;
        if ((double)(AN.x * BN.x + AN.y * BN.y + AN.z * BN.z) < 0.8660254 ||
            (double)(AN.x * CN.x + AN.y * CN.y + AN.z * CN.z) < 0.8660254 ||
            (double)(BN.x * CN.x + BN.y * CN.y + BN.z * CN.z) < 0.8660254)
          nc = false;
        if (has_consist && !nc) continue;
      }
      iteration--;
      const f3 &A = sv3[a], &B = sv3[b], &C = sv3[cc];
      const f3 AC = {A.x - C.x, A.y - C.y, A.z - C.z}, BC = {B.x - C.x, B.y - C.y, B.z - C.z};
      f4 cr;
      cr.x = AC.y * BC.z - BC.y * AC.z;
      cr.y = -(AC.x * BC.z - BC.x * AC.z);
      cr.z = AC.x * BC.y - BC.x * AC.y;
      if ((cr.x == 0 && cr.y == 0 && cr.z == 0) || std::isnan(cr.x) || std::isnan(cr.y) || std::isnan(cr.z)) continue;
      normalize3(&cr);
      cr.w = -(cr.x * A.x + cr.y * A.y + cr.z * A.z);
      int tcount = 0;
      float sdist = 0.0f;
      for (int s = 0; s < vc; ++s) {
        const float fx = (sv[s].x - cam.K[2]) / cam.K[0];
        const float fy = (sv[s].y - cam.K[5]) / cam.K[4];
        const float fd = -cr.w / (cr.x * fx + cr.y * fy + cr.z);
        const float dist = std::fabs(fd - sv3[s].z);
        residuals[s] = dist;
        if (dist < tthr) { tcount++; sdist += dist; }
      }
      if (tcount < 6) continue;
      const float fx = (px - cam.K[2]) / cam.K[0], fy = (py - cam.K[5]) / cam.K[4];
      if (tcount > max_count) {
        if (!must_tri && point_in_triangle(sv[a], sv[b], sv[cc], px, py)) must_tri = true;
        if (!has_consist && nc) has_consist = true;
        const float fd = -cr.w / (cr.x * fx + cr.y * fy + cr.z);
        const float cd = std::fabs(fd - cw.z);
        best = cr; max_count = tcount; sdist /= tcount; min_cost = cd; has_valid = true;
        if (tthr > (c.P.high_res_img ? 0.05 : 0.005)) {
          sort_small(residuals, vc);
          if (tthr < residuals[DPE_NEIGHBOUR_NUM]) continue;
          tthr = (float)(residuals[DPE_NEIGHBOUR_NUM] - 1e-6);
          tcount = 0;
          for (int s = 0; s < vc; ++s) {
            if (residuals[s] < tthr) tcount++;
            else break;
          }
          max_count = tcount;
        }
      } else if (tcount == max_count) {
        if (!must_tri && point_in_triangle(sv[a], sv[b], sv[cc], px, py)) must_tri = true;
        const float fd = -cr.w / (cr.x * fx + cr.y * fy + cr.z);
        const float cd = std::fabs(fd - cw.z);
        if (cd < min_cost) { best = cr; max_count = tcount; sdist /= tcount; min_cost = cd; }
      }
    }
  }
  if (!has_valid) { c.reliable[center] = 0; return; }
  float weight[kMaxPts];
  for (int i = 0; i < vc; ++i) {
    const float fx = (sv[i].x - cam.K[2]) / cam.K[0];
    const float fy = (sv[i].y - cam.K[5]) / cam.K[4];
    const float fd = -best.w / (best.x * fx + best.y * fy + best.z);
    const float dist = std::fabs(fd - sv3[i].z);
    if (dist >= ransac_thr) { sv[i] = {-1, -1}; weight[i] = FLT_MAX; continue; }
    weight[i] = dist;
  }
  // sort_small_weighted (insertion sort by weight), DPE.cu:20-33
  for (int i = 1; i < vc; ++i) {
    const s2 tp = sv[i];
    const float tw = weight[i];
    int j;
    for (j = i; j >= 1 && tw < weight[j - 1]; j--) { sv[j] = sv[j - 1]; weight[j] = weight[j - 1]; }
    sv[j] = tp; weight[j] = tw;
  }
  for (int i = 1; i < DPE_NEIGHBOUR_NUM; ++i) nbs[i] = sv[i - 1];
  c.reliable[center] = 1;
}

// RANSACToGetFitPlane, DPE.cu:2895-3128
static void ransac_fit_plane(Ctx &c, int px, int py) {
  const int W = c.W, center = px + py * W;
  if (c.weak[center] != DPE_WEAK) { c.fit_plane[center] = c.plane[center]; return; }
  PixelRng rng = c.rng(center);
  const dpe_camera &cam = c.cam[0];
  bool edge_limit = false;
  if (c.P.use_limit) {
    edge_limit = true;
    if (c.P.use_edge) {
      const float cv = c.complexity[center];
      const float rp = rng.uniform() - FLT_EPSILON;
      if (rp < cv) edge_limit = false;
    }
  }
  s2 sp[DPE_NEIGHBOUR_NUM - 1];
  f3 sp3[DPE_NEIGHBOUR_NUM - 1], spn[DPE_NEIGHBOUR_NUM - 1];
  int sc = 0;
  float X[3];
  for (int i = 1; i < DPE_NEIGHBOUR_NUM; ++i) {
    const s2 t = c.neighbour(center, i);
    if (t.x == -1 || t.y == -1) continue;
    sp[sc] = t;
    const int tc = t.x + t.y * W;
    const float d = depth_from_plane(cam, c.plane[tc], t.x, t.y);
    point3d(cam, t.x, t.y, d, X);
    sp3[sc] = {X[0], X[1], X[2]};
    const f4 n4 = c.plane[tc];
    spn[sc] = {n4.x, n4.y, n4.z};
    sc++;
  }
  if (sc < 3) { c.fit_plane[center] = c.plane[center]; return; }
  int ua = -1, ub = -1, uc = -1;
  float min_cost = FLT_MAX;
  f4 best = {0, 0, 0, 0};
  bool has_best = false, has_strong = false;
  bool must_tri = (c.P.use_label && c.label[center] > 0 && edge_limit) ? false : true;
  int iteration = 50;
  while (iteration--) {
    const int a = (int)(rng.next_u32() % (uint32_t)sc);
    const int b = (int)(rng.next_u32() % (uint32_t)sc);
    const int cc = (int)(rng.next_u32() % (uint32_t)sc);
    if (a == b || b == cc || a == cc) continue;
    bool is_strong = false;
    if (c.P.geom_consistency && edge_limit) {
      const f3 &AN = spn[a], &BN = spn[b], &CN = spn[cc];
      is_strong = true;
      if ((double)(AN.x * BN.x + AN.y * BN.y + AN.z * BN.z) < 0.8660254 ||
          (double)(AN.x * CN.x + AN.y * CN.y + AN.z * CN.z) < 0.8660254 ||
          (double)(BN.x * CN.x + BN.y * CN.y + BN.z * CN.z) < 0.8660254)
        is_strong = false;
      if (has_strong && !is_strong) continue;
    }
    if (must_tri && !point_in_triangle(sp[a], sp[b], sp[cc], px, py)) continue;
    if (edge_limit) {
      if (bresenham(c, sp[a].x, sp[a].y, sp[b].x, sp[b].y) || bresenham(c, sp[b].x, sp[b].y, sp[cc].x, sp[cc].y) ||
          bresenham(c, sp[cc].x, sp[cc].y, sp[a].x, sp[a].y))
        continue;
    }
    const f3 &A = sp3[a], &B = sp3[b], &C = sp3[cc];
    const f3 AC = {A.x - C.x, A.y - C.y, A.z - C.z}, BC = {B.x - C.x, B.y - C.y, B.z - C.z};
    f4 cr;
    cr.x = AC.y * BC.z - BC.y * AC.z;
    cr.y = -(AC.x * BC.z - BC.x * AC.z);
    cr.z = AC.x * BC.y - BC.x * AC.y;
    if ((cr.x == 0 && cr.y == 0 && cr.z == 0) || std::isnan(cr.x) || std::isnan(cr.y) || std::isnan(cr.z)) continue;
    normalize3(&cr);
    cr.w = -(cr.x * A.x + cr.y * A.y + cr.z * A.z);
    if (!has_strong && is_strong) has_strong = true;
    float tc = 0.0f;
    for (int s = 0; s < sc; ++s) {
      if (s == a || s == b || s == cc) continue;
      const float fx = (sp[s].x - cam.K[2]) / cam.K[0];
      const float fy = (sp[s].y - cam.K[5]) / cam.K[4];
      const float fd = -cr.w / (cr.x * fx + cr.y * fy + cr.z);
      tc += std::fabs(fd - sp3[s].z);
    }
    if (tc < min_cost) {
      if (!must_tri && point_in_triangle(sp[a], sp[b], sp[cc], px, py)) must_tri = true;
      min_cost = tc; best = cr; has_best = true; ua = a; ub = b; uc = cc;
    }
  }
  if (has_best) {
    const float depth = depth_from_plane(cam, c.plane[center], px, py);
    const f4 v = view_direction(cam, px, py, depth);
    if (best.x * v.x + best.y * v.y + best.z * v.z > 0) { best.x = -best.x; best.y = -best.y; best.z = -best.z; best.w = -best.w; }
    c.fit_plane[center] = best;
    if (c.P.use_radius) {
      if (must_tri) {
        const s2 A = sp[ua], B = sp[ub], C = sp[uc];
        const float a = std::sqrt((float)((A.x - B.x) * (A.x - B.x) + (A.y - B.y) * (A.y - B.y)));
        const float b = std::sqrt((float)((B.x - C.x) * (B.x - C.x) + (B.y - C.y) * (B.y - C.y)));
        const float cl = std::sqrt((float)((C.x - A.x) * (C.x - A.x) + (C.y - A.y) * (C.y - A.y)));
        const float p = (float)((a + b + cl) / 2.0);
        const float S = std::sqrt(p * (p - a) * (p - b) * (p - cl));
        int radius = f2i(std::floor(std::sqrt(S) / 2.0));
        const float ad = std::sqrt((float)((A.x - px) * (A.x - px) + (A.y - py) * (A.y - py)));
        const float bd = std::sqrt((float)((B.x - px) * (B.x - px) + (B.y - py) * (B.y - py)));
        const float cd = std::sqrt((float)((C.x - px) * (C.x - px) + (C.y - py) * (C.y - py)));
        const float md = CV_MIN(CV_MIN(ad, bd), cd);
        if (2.5 * md < radius) radius = f2i(md);
        if (edge_limit) {
          if (c.P.use_edge) {
            float med = FLT_MAX;
            const s2 *en = &c.edge_neigh[(size_t)center * 8];
            for (int d = 0; d < 8; ++d) {
              const s2 e = en[d];
              if (e.x == -1 || e.y == -1) continue;
              const float dist = std::sqrt((float)((e.x - px) * (e.x - px) + (e.y - py) * (e.y - py)));
              med = CV_MIN(med, dist);
            }
            if (med < radius) radius = f2i(med);
          }
          if (c.P.use_label && c.label[center] > 0) {
            float mbd = FLT_MAX;
            const s2 *lb = &c.lab_bound[(size_t)c.nmap[center] * 8];
            for (int d = 0; d < 8; ++d) {
              const s2 bb = lb[d];
              if (bb.x == -1 || bb.y == -1) continue;
              const float dist = (float)std::sqrt(std::pow((double)(px - bb.x), 2) + std::pow((double)(py - bb.y), 2));
              mbd = CV_MIN(mbd, dist);
            }
            if (mbd < radius) radius = f2i(mbd);
          }
        }
        while ((radius << 1) % 5 != 0) radius--;
        if (!edge_limit) c.radius[center] = radius > c.P.strong_radius ? 0 : c.P.strong_radius;
        else c.radius[center] = radius > c.P.strong_radius ? radius : c.P.strong_radius;
      } else {
        c.radius[center] = c.P.strong_radius;
      }
    }
  } else {
    c.fit_plane[center] = {0, 0, 0, 0};
    if (c.P.use_radius) c.radius[center] = c.P.strong_radius;
  }
}

// GetDepthandNormal, DPE.cu:1944-1959
static void get_depth_normal(Ctx &c, int px, int py) {
  const int center = py * c.W + px;
  f4 pl = c.plane[center];
  pl.w = depth_from_plane(c.cam[0], pl, px, py);
  c.plane[center] = normal_to_world(c.cam[0], pl);
}

// CheckerboardFilterStrong, DPE.cu:1961-2071
static void filter_strong(Ctx &c, int px, int py) {
  const int W = c.W, H = c.H, center = py * W + px;
  float f[21];
  int k = 0;
  f[k++] = c.plane[center].w;
  if (c.cost[center] < 0.001f) return;
  auto take = [&](bool ok, int idx) {
    if (ok && c.weak[idx] == DPE_STRONG) f[k++] = c.plane[idx].w;
  };
  const int up = center - W, upup = center - 3 * W, dn = center + W, dndn = center + 3 * W;
  const int lf = center - 1, lflf = center - 3, rt = center + 1, rtrt = center + 3;
  take(py > 0, up);
  take(py > 2, upup);
  take(py > 4, upup - 2 * W);
  take(py < H - 1, dn);
  take(py < H - 3, dndn);
  take(py < H - 5, dndn + 2 * W);
  take(px > 0, lf);
  take(px > 2, lflf);
  take(px > 4, lflf - 2);
  take(px < W - 1, rt);
  take(px < W - 3, rtrt);
  take(px < W - 5, rtrt + 2);
  take(py > 0 && px < W - 2, up + 2);
  take(py < H - 1 && px < W - 2, dn + 2);
  take(py > 0 && px > 1, up - 2);
  take(py < H - 1 && px > 1, dn - 2);
  take(px > 0 && py > 2, lf - 2 * W);
  take(px < W - 1 && py > 2, rt - 2 * W);
  take(px > 0 && py < H - 2, lf + 2 * W);
  take(px < W - 1 && py < H - 2, rt + 2 * W);
  sort_small(f, k);
  const int m = k / 2;
  c.plane[center].w = (k % 2 == 0) ? (f[m - 1] + f[m]) / 2 : f[m];
}

// Shared prologue of DepthToWeak / LocalRefine (DPE.cu:2619-2660, :2767-2806)
struct SweepSetup {
  f4 pl;
  float depth, cost_now, base_line, weight_normal;
  int valid;
};
static SweepSetup sweep_setup(Ctx &c, int px, int py) {
  const int center = px + py * c.W;
  const dpe_camera *cams = c.cam;
  const uint8_t *vw = &c.vweight[(size_t)center * DPE_MAX_IMAGES];
  SweepSetup s;
  s.pl = normal_to_ref(cams[0], c.plane[center]);
  s.depth = s.pl.w;
  s.cost_now = 0.0f; s.base_line = 0.0f; s.weight_normal = 0.0f; s.valid = 0;
  if (s.depth == 0) return s;
  for (int si = 1; si < c.P.num_images; ++si) {
    const int vi = si - 1;
    if (!isSet(c.views[center], vi)) continue;
    f4 t = s.pl;
    t.w = dist_to_origin(cams[0], px, py, s.depth, t);
    float tc = ncc_strong(c, px, py, si, t);
    if (c.P.geom_consistency) tc += c.P.geom_factor * geom_cost(c, px, py, si, t);
    s.cost_now += tc * vw[vi];
    s.weight_normal += vw[vi];
    const float d0 = cams[0].c[0] - cams[si].c[0], d1 = cams[0].c[1] - cams[si].c[1], d2 = cams[0].c[2] - cams[si].c[2];
    const double tv = d0 * d0 + d1 * d1 + d2 * d2;
    s.base_line += std::sqrt((float)tv);
    s.valid++;
  }
  return s;
}

// DepthToWeak, DPE.cu:2597-2751
static void depth_to_weak(Ctx &c, int px, int py) {
  const int W = c.W, H = c.H, center = px + py * W, margin = 6;
  if (px < margin || py < margin || px >= W - margin || py >= H - margin) { c.weak[center] = DPE_UNKNOWN; return; }
  const dpe_camera &rc = c.cam[0];
  const uint8_t *vw = &c.vweight[(size_t)center * DPE_MAX_IMAGES];
  SweepSetup s = sweep_setup(c, px, py);
  if (s.depth == 0) { c.weak[center] = DPE_UNKNOWN; return; }
  if (s.valid == 0) { c.weak[center] = DPE_UNKNOWN; return; }
  s.cost_now /= s.weight_normal;
  s.base_line /= s.valid;
  const float disp = rc.K[0] * s.base_line / s.depth;
  const int R = 30, NS = 61;
  float pc[NS];
  for (int pd = -R; pd <= R; ++pd) {
    const float pdep = rc.K[0] * s.base_line / (disp + pd);
    if (pdep < c.P.depth_min || pdep > c.P.depth_max) { pc[pd + R] = 2.0f; continue; }
    f4 t = s.pl;
    t.w = dist_to_origin(rc, px, py, pdep, t);
    float cost = 0.0f;
    for (int si = 1; si < c.P.num_images; ++si) {
      const int vi = si - 1;
      float tc = 0.0f;
      if (isSet(c.views[center], vi)) {
        tc += ncc_strong(c, px, py, si, t);
        if (c.P.geom_consistency) tc += c.P.geom_factor * geom_cost(c, px, py, si, t);
        cost += tc * vw[vi];
      }
    }
    cost /= s.weight_normal;
    pc[pd + R] = CV_MIN(2.0f, cost);
  }
  bool peak[NS];
  for (int i = 0; i < NS; ++i) peak[i] = false;
  int peaks = 0, min_peak = 0;
  float min_cost = 2.0f;
  for (int i = 2; i < NS - 2; ++i)
    if (pc[i - 1] > pc[i] && pc[i + 1] > pc[i]) {
      peak[i] = true; peaks++;
      if (pc[i] < min_cost) { min_peak = i; min_cost = pc[i]; }
    }
  if (std::abs(min_peak - R) > c.P.weak_peak_radius || pc[min_peak] > 0.5f) { c.weak[center] = DPE_WEAK; return; }
  if (peaks == 1) { c.weak[center] = pc[min_peak] <= 0.15f ? DPE_STRONG : DPE_WEAK; return; }
  float var = 0.0f;
  for (int i = 2; i < NS - 2; ++i)
    if (peak[i] && i != min_peak) { const float d = pc[i] - min_cost; var += d * d; }
  var = std::sqrt(var);
  var /= (peaks - 1);
  c.weak[center] = var > 0.2f ? DPE_STRONG : DPE_WEAK;
}

// LocalRefine, DPE.cu:2753-2839
static void local_refine(Ctx &c, int px, int py) {
  const int center = px + py * c.W;
  const dpe_camera &rc = c.cam[0];
  const uint8_t *vw = &c.vweight[(size_t)center * DPE_MAX_IMAGES];
  SweepSetup s = sweep_setup(c, px, py);
  if (s.depth == 0) return;
  if (s.weight_normal == 0 || s.valid == 0) return;
  s.cost_now /= s.weight_normal;
  s.base_line /= s.valid;
  const float disp = rc.K[0] * s.base_line / s.depth;
  float min_cost = 2.0f, best = s.depth;
  for (int pd = -5; pd <= 5; ++pd) {
    const float pdep = rc.K[0] * s.base_line / (disp + pd);
    if (pdep < c.P.depth_min || pdep > c.P.depth_max) continue;
    f4 t = s.pl;
    t.w = dist_to_origin(rc, px, py, pdep, t);
    float tc = 0.0f;
    for (int si = 1; si < c.P.num_images; ++si) {
      const int vi = si - 1;
      if (isSet(c.views[center], vi)) {
        tc += ncc_strong(c, px, py, si, t) * vw[vi];
        if (c.P.geom_consistency) tc += c.P.geom_factor * geom_cost(c, px, py, si, t) * vw[vi];
      }
    }
    tc /= s.weight_normal;
    if (tc < min_cost) { min_cost = tc; best = pdep; }
  }
  if ((double)(s.cost_now - min_cost) > 0.1) c.plane[center].w = best;
}

// ----------------------------------------------------------------------------- driver
template <class F> static void for_all(Ctx &c, F f, int threads) {
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads)
  for (int y = 0; y < c.H; ++y)
    for (int x = 0; x < c.W; ++x) f(x, y);
}
// pixels with (x + y) % 2 == parity; black = 0, red = 1 (DPE.cu:1904-1942 thread mapping)
template <class F> static void for_colour(Ctx &c, int parity, F f, int threads) {
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads)
  for (int y = 0; y < c.H; ++y)
    for (int x = (y + parity) & 1; x < c.W; x += 2) f(x, y);
}

}  // namespace oracle

using namespace oracle;

extern "C" {

void oracle_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) { philox4x32_10(ctr, key, out); }

void oracle_set_raw_moments(int on) { g_raw_moments = on != 0; }

void oracle_set_ref_addressing(int on) { g_ref_addressing = on != 0; }

void oracle_set_ref_homography(int on) { g_ref_homography = on != 0; }

void oracle_set_serial_race(int on) { g_serial_race = on != 0; }

// Strong NCC at explicit queries.  fp64 != 0 evaluates the cost in double precision end to end
// (homography from the float cameras, exact bilinear, double exp/sqrt).
void oracle_ncc_strong(const dpe_ncc_query *q, int fp64, double *out) {
  Ctx c;
  c.W = q->width; c.H = q->height; c.N = q->num_images; c.P = q->params;
  c.set_cameras(q->cameras);
  for (int i = 0; i < c.N; ++i) { c.img[i].data = q->images[i]; c.img[i].w = c.W; c.img[i].h = c.H; }
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < q->count; ++k) {
    const f4 pl = {q->plane[4 * k], q->plane[4 * k + 1], q->plane[4 * k + 2], q->plane[4 * k + 3]};
    const int px = q->px[k], py = q->py[k], s = q->src[k];
    if (!fp64) { out[k] = ncc_strong(c, px, py, s, pl); continue; }
    // ---- FP64 path: same algorithm, double arithmetic throughout
    const dpe_camera &rc = c.cam[0], &sc = c.cam[s];
    double rC[3], sC[3], Rr[9], Cr[3], tr[3], H[9], T[9];
    for (int i = 0; i < 3; ++i) {
      rC[i] = -((double)rc.R[i] * rc.t[0] + (double)rc.R[3 + i] * rc.t[1] + (double)rc.R[6 + i] * rc.t[2]);
      sC[i] = -((double)sc.R[i] * sc.t[0] + (double)sc.R[3 + i] * sc.t[1] + (double)sc.R[6 + i] * sc.t[2]);
    }
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        Rr[3 * a + b] = (double)sc.R[3 * a] * rc.R[3 * b] + (double)sc.R[3 * a + 1] * rc.R[3 * b + 1] + (double)sc.R[3 * a + 2] * rc.R[3 * b + 2];
    for (int i = 0; i < 3; ++i) Cr[i] = rC[i] - sC[i];
    for (int a = 0; a < 3; ++a) tr[a] = (double)sc.R[3 * a] * Cr[0] + (double)sc.R[3 * a + 1] * Cr[1] + (double)sc.R[3 * a + 2] * Cr[2];
    const double n[3] = {pl.x, pl.y, pl.z};
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) H[3 * a + b] = Rr[3 * a + b] - tr[a] * n[b] / (double)pl.w;
    for (int a = 0; a < 3; ++a) {
      T[3 * a] = H[3 * a] / rc.K[0];
      T[3 * a + 1] = H[3 * a + 1] / rc.K[4];
      T[3 * a + 2] = -H[3 * a] * rc.K[2] / rc.K[0] - H[3 * a + 1] * rc.K[5] / rc.K[4] + H[3 * a + 2];
    }
    for (int b = 0; b < 3; ++b) {
      H[b] = (double)sc.K[0] * T[b] + (double)sc.K[2] * T[6 + b];
      H[3 + b] = (double)sc.K[4] * T[3 + b] + (double)sc.K[5] * T[6 + b];
      H[6 + b] = (double)sc.K[8] * T[6 + b];
    }
    auto proj = [&](double x, double y, double *ox, double *oy) {
      const double X = H[0] * x + H[1] * y + H[2], Y = H[3] * x + H[4] * y + H[5], Z = H[6] * x + H[7] * y + H[8];
      *ox = X / Z; *oy = Y / Z;
    };
    double cx, cy;
    proj(px, py, &cx, &cy);
    if (cx >= sc.width || cx < 0.0 || cy >= sc.height || cy < 0.0) { out[k] = 2.0; continue; }
    const double center = c.img[0].texel(px, py);
    const int r = c.P.strong_radius, inc = c.P.strong_increment;
    double s_r = 0, s_rr = 0, s_s = 0, s_ss = 0, s_rs = 0, s_w = 0;
    for (int i = -r; i <= r; i += inc)
      for (int j = -r; j <= r; j += inc) {
        const double rp = c.img[0].texel(px + i, py + j);
        double sx, sy;
        proj(px + i, py + j, &sx, &sy);
        const double sv = c.img[s].bilinear_fp64(sx, sy);
        const double w = std::exp(-std::sqrt((double)(i * i + j * j)) / (2.0 * c.P.sigma_spatial * c.P.sigma_spatial) -
                                  std::fabs(rp - center) / (2.0 * c.P.sigma_color * c.P.sigma_color));
        s_r += w * rp; s_rr += w * rp * rp; s_s += w * sv; s_ss += w * sv * sv; s_rs += w * rp * sv; s_w += w;
      }
    s_r /= s_w; s_rr /= s_w; s_s /= s_w; s_ss /= s_w; s_rs /= s_w;
    const double vr = s_rr - s_r * s_r, vs = s_ss - s_s * s_s;
    if (vr < 1e-5 || vs < 1e-5) { out[k] = 2.0; continue; }
    out[k] = std::fmax(0.0, std::fmin(2.0, 1.0 - (s_rs - s_r * s_s) / std::sqrt(vr * vs)));
  }
}

// ----------------------------------------------------------------------------- FP64 gradient
// Reference gradient of the strong NCC (ComputeBilateralNCCOld, DPE.cu:696-782, evaluated as
// above in double) for checking the adjoint kernel.  The plane derivatives come from forward-mode
// dual numbers over (nx, ny, nz, w), independent of any hand-derived adjoint; the source-image
// derivative follows from dC/ds_k (the cost's sensitivity to each bilinear sample) times the
// bilinear weights of the sample's four texels (clamped to the image like the sample itself).
namespace {
struct D4 {
  double v = 0, d[4] = {0, 0, 0, 0};
  D4() = default;
  D4(double x) : v(x) {}
};
inline D4 operator+(const D4 &a, const D4 &b) { D4 r(a.v + b.v); for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] + b.d[i]; return r; }
inline D4 operator-(const D4 &a, const D4 &b) { D4 r(a.v - b.v); for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] - b.d[i]; return r; }
inline D4 operator*(const D4 &a, const D4 &b) {
  D4 r(a.v * b.v);
  for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
inline D4 operator/(const D4 &a, const D4 &b) {
  D4 r(a.v / b.v);
  for (int i = 0; i < 4; ++i) r.d[i] = (a.d[i] * b.v - a.v * b.d[i]) / (b.v * b.v);
  return r;
}
inline D4 dsqrt(const D4 &a) {
  D4 r(std::sqrt(a.v));
  for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] / (2.0 * r.v);
  return r;
}
}  // namespace

// cost_out[k] and grad_plane[4k..4k+3] = dC/d(nx, ny, nz, w) per query.  grad_images, when not
// null, holds num_images pointers (entry 0 unused) to W*H double buffers that receive the
// gradient of the SUM of all query costs with respect to that source image's pixels.
void oracle_ncc_strong_grad(const dpe_ncc_query *q, double *cost_out, double *grad_plane, double **grad_images) {
  Ctx c;
  c.W = q->width; c.H = q->height; c.N = q->num_images; c.P = q->params;
  c.set_cameras(q->cameras);
  for (int i = 0; i < c.N; ++i) { c.img[i].data = q->images[i]; c.img[i].w = c.W; c.img[i].h = c.H; }
  const int r = c.P.strong_radius, inc = c.P.strong_increment;
#pragma omp parallel for schedule(static) if (!grad_images)
  for (int64_t k = 0; k < q->count; ++k) {
    const int px = q->px[k], py = q->py[k], s = q->src[k];
    const dpe_camera &rc = c.cam[0], &sc = c.cam[s];
    double *g = grad_plane + 4 * k;
    g[0] = g[1] = g[2] = g[3] = 0.0;
    cost_out[k] = 2.0;
    double rC[3], sC[3], Rr[9], Cr[3], tr[3];
    for (int i = 0; i < 3; ++i) {
      rC[i] = -((double)rc.R[i] * rc.t[0] + (double)rc.R[3 + i] * rc.t[1] + (double)rc.R[6 + i] * rc.t[2]);
      sC[i] = -((double)sc.R[i] * sc.t[0] + (double)sc.R[3 + i] * sc.t[1] + (double)sc.R[6 + i] * sc.t[2]);
    }
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        Rr[3 * a + b] = (double)sc.R[3 * a] * rc.R[3 * b] + (double)sc.R[3 * a + 1] * rc.R[3 * b + 1] + (double)sc.R[3 * a + 2] * rc.R[3 * b + 2];
    for (int i = 0; i < 3; ++i) Cr[i] = rC[i] - sC[i];
    for (int a = 0; a < 3; ++a) tr[a] = (double)sc.R[3 * a] * Cr[0] + (double)sc.R[3 * a + 1] * Cr[1] + (double)sc.R[3 * a + 2] * Cr[2];
    D4 n[3], w;
    for (int b = 0; b < 3; ++b) { n[b] = D4(q->plane[4 * k + b]); n[b].d[b] = 1.0; }
    w = D4(q->plane[4 * k + 3]); w.d[3] = 1.0;
    D4 H[9], T[9];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) H[3 * a + b] = D4(Rr[3 * a + b]) - D4(tr[a]) * n[b] / w;
    for (int a = 0; a < 3; ++a) {
      T[3 * a] = H[3 * a] / D4(rc.K[0]);
      T[3 * a + 1] = H[3 * a + 1] / D4(rc.K[4]);
      T[3 * a + 2] = D4(0.0) - H[3 * a] * D4((double)rc.K[2] / rc.K[0]) - H[3 * a + 1] * D4((double)rc.K[5] / rc.K[4]) +
                     H[3 * a + 2];
    }
    for (int b = 0; b < 3; ++b) {
      H[b] = D4(sc.K[0]) * T[b] + D4(sc.K[2]) * T[6 + b];
      H[3 + b] = D4(sc.K[4]) * T[3 + b] + D4(sc.K[5]) * T[6 + b];
      H[6 + b] = D4(sc.K[8]) * T[6 + b];
    }
    auto proj = [&](double x, double y, D4 *ox, D4 *oy) {
      const D4 X = H[0] * D4(x) + H[1] * D4(y) + H[2], Y = H[3] * D4(x) + H[4] * D4(y) + H[5];
      const D4 Z = H[6] * D4(x) + H[7] * D4(y) + H[8];
      *ox = X / Z; *oy = Y / Z;
    };
    D4 cx, cy;
    proj(px, py, &cx, &cy);
    if (cx.v >= sc.width || cx.v < 0.0 || cy.v >= sc.height || cy.v < 0.0) continue;
    const double center = c.img[0].texel(px, py);
    constexpr int kMaxTaps = 256;
    double wk[kMaxTaps], rk[kMaxTaps], svk[kMaxTaps];
    int tx0[kMaxTaps], ty0[kMaxTaps];
    double tax[kMaxTaps], tay[kMaxTaps];
    int nt = 0;
    D4 s_s(0.0), s_ss(0.0), s_rs(0.0);
    double s_r = 0, s_rr = 0, s_w = 0;
    for (int i = -r; i <= r; i += inc)
      for (int j = -r; j <= r; j += inc) {
        const double rp = c.img[0].texel(px + i, py + j);
        D4 sx, sy;
        proj(px + i, py + j, &sx, &sy);
        const Image &im = c.img[s];
        // bilinear with clamp-to-edge: a clamped coordinate does not move the sample
        D4 xc = sx, yc = sy;
        if (sx.v < -1.0) xc = D4(-1.0);
        if (sx.v > (double)(im.w - 1)) xc = D4((double)(im.w - 1));
        if (sy.v < -1.0) yc = D4(-1.0);
        if (sy.v > (double)(im.h - 1)) yc = D4((double)(im.h - 1));
        const double fx = std::floor(xc.v), fy = std::floor(yc.v);
        const int x0 = (int)fx, y0 = (int)fy;
        D4 ax = xc - D4(fx), ay = yc - D4(fy);
        const double v00 = im.texel(x0, y0), v10 = im.texel(x0 + 1, y0);
        const double v01 = im.texel(x0, y0 + 1), v11 = im.texel(x0 + 1, y0 + 1);
        const D4 top = (D4(1.0) - ax) * D4(v00) + ax * D4(v10);
        const D4 bot = (D4(1.0) - ax) * D4(v01) + ax * D4(v11);
        const D4 sv = (D4(1.0) - ay) * top + ay * bot;
        const double wt = std::exp(-std::sqrt((double)(i * i + j * j)) / (2.0 * c.P.sigma_spatial * c.P.sigma_spatial) -
                                   std::fabs(rp - center) / (2.0 * c.P.sigma_color * c.P.sigma_color));
        s_r += wt * rp; s_rr += wt * rp * rp; s_w += wt;
        s_s = s_s + D4(wt) * sv; s_ss = s_ss + D4(wt) * sv * sv; s_rs = s_rs + D4(wt * rp) * sv;
        if (nt < kMaxTaps) {
          wk[nt] = wt; rk[nt] = rp; svk[nt] = sv.v; tx0[nt] = x0; ty0[nt] = y0; tax[nt] = ax.v; tay[nt] = ay.v;
          nt++;
        }
      }
    s_r /= s_w; s_rr /= s_w;
    const D4 ms = s_s / D4(s_w), mss = s_ss / D4(s_w), mrs = s_rs / D4(s_w);
    const double vr = s_rr - s_r * s_r;
    const D4 vs = mss - ms * ms;
    if (vr < 1e-5 || vs.v < 1e-5) continue;
    const D4 cov = mrs - D4(s_r) * ms;
    const D4 cst = D4(1.0) - cov / dsqrt(D4(vr) * vs);
    cost_out[k] = std::fmax(0.0, std::fmin(2.0, cst.v));
    if (cst.v <= 0.0 || cst.v >= 2.0) continue;  // clamped: flat
    for (int i = 0; i < 4; ++i) g[i] = cst.d[i];
    if (grad_images && grad_images[s]) {
      const double sq = std::sqrt(vr * vs.v);
      for (int t = 0; t < nt; ++t) {
        const double dcov = wk[t] * (rk[t] - s_r) / s_w;
        const double dvs = 2.0 * wk[t] * (svk[t] - ms.v) / s_w;
        const double dc = -dcov / sq + cov.v * dvs / (2.0 * vs.v * sq);
        const int xs[2] = {tx0[t], tx0[t] + 1}, ys[2] = {ty0[t], ty0[t] + 1};
        const double bx[2] = {1.0 - tax[t], tax[t]}, by[2] = {1.0 - tay[t], tay[t]};
        for (int yy = 0; yy < 2; ++yy)
          for (int xx = 0; xx < 2; ++xx) {
            const int X = std::min(std::max(xs[xx], 0), c.W - 1), Y = std::min(std::max(ys[yy], 0), c.H - 1);
            grad_images[s][(size_t)Y * c.W + X] += dc * bx[xx] * by[yy];
          }
      }
    }
  }
}

// One per-view PatchMatch call with the kernel order of DPE::RunPatchMatch (DPE.cu:3157-3234).
// Host memory only.  Returns 0 on success.
int oracle_pm_run(const dpe_problem *pr, dpe_pm_out *out, int threads) {
  if (!pr || !out || pr->memory != DPE_MEM_HOST) return DPE_ERR_INVALID_ARGUMENT;
  if (threads <= 0) threads = omp_get_max_threads();
  Ctx c;
  c.W = pr->width; c.H = pr->height; c.N = pr->num_images; c.P = pr->params;
  c.P.num_images = c.N;
  const size_t L = (size_t)c.W * c.H;
  c.set_cameras(pr->cameras);
  for (int i = 0; i < c.N; ++i) {
    c.img[i].data = pr->images[i]; c.img[i].w = c.W; c.img[i].h = c.H;
    if (c.P.geom_consistency) { c.dep[i].data = pr->depths[i]; c.dep[i].w = c.W; c.dep[i].h = c.H; }
  }
  c.key[0] = (uint32_t)pr->seed; c.key[1] = (uint32_t)(pr->seed >> 32);
  c.plane.assign(L, f4{0, 0, 0, 0});
  if (c.P.state != DPE_FIRST_INIT && pr->plane_in) std::memcpy(c.plane.data(), pr->plane_in, L * sizeof(f4));
  c.cost.assign(L, 0.0f);
  c.views.assign(L, 0u);
  if (c.P.state != DPE_FIRST_INIT && pr->selected_views_in) std::memcpy(c.views.data(), pr->selected_views_in, L * 4);
  c.rng_ctr.assign(L, 0u);
  c.weak.assign(L, (uint8_t)DPE_STRONG);
  if (c.P.use_APD) std::memcpy(c.weak.data(), pr->weak_in, L);
  c.nmap.assign(L, 0);
  c.weak_count = 0;
  if (c.P.use_APD)
    for (size_t i = 0; i < L; ++i)
      if (c.weak[i] == DPE_WEAK) c.nmap[i] = c.weak_count++;
  c.neigh.assign((size_t)c.weak_count * DPE_NEIGHBOUR_NUM, s2{-1, -1});
  c.lab_bound.assign((size_t)c.weak_count * 8, s2{-1, -1});
  c.reliable.assign(L, 0);
  c.nearest.assign(L, s2{-1, -1});
  c.fit_plane.assign(L, f4{0, 0, 0, 0});
  c.vweight.assign(L * DPE_MAX_IMAGES, 0);
  c.radius.assign(L, c.P.strong_radius);
  c.complexity.assign(L, 0.0f);
  c.edge_neigh.assign(L * 8, s2{-1, -1});
  if (c.P.use_edge || c.P.use_limit) {
    c.edge.assign(pr->edge, pr->edge + L);
    c.lowW = pr->low_width; c.lowH = pr->low_height;
    c.edge_low.assign(pr->edge_low_res, pr->edge_low_res + (size_t)c.lowW * c.lowH);
  }
  if (c.P.use_label) c.label.assign(pr->label, pr->label + L);
  else c.label.assign(L, 0);

  for_all(c, [&](int x, int y) { gen_edge_inform(c, x, y); }, threads);
  for_all(c, [&](int x, int y) { find_nearest_strong(c, x, y); }, threads);
  for_all(c, [&](int x, int y) { gen_neighbours(c, x, y); }, threads);
  for_all(c, [&](int x, int y) {
    const int ctr = x + y * c.W;
    if (c.weak[ctr] == DPE_WEAK && c.reliable[ctr] != 1) c.weak[ctr] = DPE_UNKNOWN;
  }, threads);
  for_all(c, [&](int x, int y) { random_initialization(c, x, y); }, threads);
  for (int it = 0; it < c.P.max_iterations; ++it) {
    for (int colour = 0; colour < 2; ++colour) {
      if (c.P.use_edge && !g_serial_race) { c.plane_snap = c.plane; c.cost_snap = c.cost; }
      for_colour(c, colour, [&](int x, int y) {
        if (c.weak[x + y * c.W] != DPE_WEAK) strong_update(c, x, y, it);
      }, c.P.use_edge && g_serial_race ? 1 : threads);
    }
    for_all(c, [&](int x, int y) { ransac_fit_plane(c, x, y); }, threads);
    for (int colour = 0; colour < 2; ++colour)
      for_colour(c, colour, [&](int x, int y) {
        if (c.weak[x + y * c.W] == DPE_WEAK) weak_update(c, x, y, it);
      }, threads);
  }
  for_all(c, [&](int x, int y) { get_depth_normal(c, x, y); }, threads);
  for (int colour = 0; colour < 2; ++colour)
    for_colour(c, colour, [&](int x, int y) {
      if (c.weak[x + y * c.W] != DPE_WEAK) filter_strong(c, x, y);
    }, threads);
  for_all(c, [&](int x, int y) { depth_to_weak(c, x, y); }, threads);
  for_all(c, [&](int x, int y) { local_refine(c, x, y); }, threads);

  if (out->plane) std::memcpy(out->plane, c.plane.data(), L * sizeof(f4));
  if (out->weak) std::memcpy(out->weak, c.weak.data(), L);
  if (out->selected_views) std::memcpy(out->selected_views, c.views.data(), L * 4);
  if (out->costs) std::memcpy(out->costs, c.cost.data(), L * 4);
  out->gpu_ms = 0.0f;
  return DPE_OK;
}

}  // extern "C"
