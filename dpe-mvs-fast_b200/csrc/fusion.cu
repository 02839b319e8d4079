// fusion.cu -- depth-map fusion (RunFusion, DPE.cpp:1387-1548) on the GPU with the reference's
// order-dependent result.
//
// The reference walks views in pair.txt order and pixels in raster order; an accepted pixel
// masks the source pixels it used, and a masked source pixel is skipped by every later pixel.
// Views run one after another here as well (a view's own pixels are masked only by earlier
// views).  Within one reference view, a (source, pixel) entry of pixel p is live iff no earlier
// pixel of the view that is ACCEPTED tests the same source pixel consistent; p's acceptance
// depends on which of its entries are live.  The kernels compute every pixel's consistency
// entries in parallel, then find the decisions as the fixed point of a Jacobi iteration:
//   * start from every pixel's decision with all its entries live;
//   * a round stamps each currently accepted pixel on the source pixels it tests consistent
//     (atomicMin, the first accepted claimant wins) and re-decides every candidate from those
//     claims;
//   * stop after a round that changes no decision.
// The decisions of the sequential loop satisfy every round (each depends only on earlier
// pixels), and they are the only assignment that does: induction over raster order.  After k
// rounds every pixel whose chain of earlier dependencies is k long is final, so the rounds end;
// on the 10-view 1600x1200 scene they end after 5-10 rounds per view, because a changed decision
// rarely changes a later one.  Decisions, counts, point order and colours are those of the
// sequential loop.
//
// This file is compiled with -fmad=false so that its float and double arithmetic rounds like the
// CPU restatement of the same loop.
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <cstring>
#include <vector>

#include "ctx.h"

namespace {

struct FuseView {
  int W, H;
  const float *depth;
  const float *normal;
  const uint8_t *weak;
  const uint8_t *bgr;
  const uint8_t *block;
  uint8_t *mask;
  // per pixel: the first accepted claimant of the current round, as (stamp << 32 | pixel) with
  // stamp = 0xFFFFFFFF - round number (counted over the whole call): a round's keys are smaller
  // than every earlier round's, so no reset between rounds is needed, and a key belongs to the
  // current round exactly when its stamp is the current one.
  unsigned long long *claim;
  dpe_camera cam;
};

constexpr int kMaxSrc = 32;

struct FuseArgs {
  int mode;
  int min_consistent;
  int ref;
  int ns;
  int src[kMaxSrc];
  const FuseView *views;  // device array
  int *entry_q;           // W*H*ns: source pixel index, -1 when the entry is not consistent
  double *entry_score;    // W*H*ns: exp(-(e + 200 dd + 10 angle)) of a consistent entry
  uint8_t *status;        // W*H: 1 accepted, 3 rejected (this round), 2 not a candidate
  int *changes;           // decisions a round changed
};

// RunFusion's acceptance rule (DPE.cpp:1517-1520) over the live entries of one pixel, summed in
// source order; min_consistent > 1 raises the reference's n >= 1.
__device__ __forceinline__ bool fuse_accept(const FuseArgs &f, const FuseView &V, int pix, int n, double dyn_d,
                                            float dyn_f) {
  const float factor = V.weak[pix] == DPE_WEAK ? 0.45f : 0.3f;
  const int need = f.min_consistent > 1 ? f.min_consistent : 1;
  return f.mode == DPE_FUSE_FP64 ? (n >= need && dyn_d > (double)factor * n) : (n >= need && dyn_f > factor * n);
}

template <class T> __device__ __forceinline__ void world_point(T x, T y, T depth, const dpe_camera &c, T out[3]) {
  const T px = depth * (x - (T)c.K[2]) / (T)c.K[0];
  const T py = depth * (y - (T)c.K[5]) / (T)c.K[4];
  const T pz = depth;
  const T tx = (T)c.R[0] * px + (T)c.R[3] * py + (T)c.R[6] * pz;
  const T ty = (T)c.R[1] * px + (T)c.R[4] * py + (T)c.R[7] * pz;
  const T tz = (T)c.R[2] * px + (T)c.R[5] * py + (T)c.R[8] * pz;
  const T Cx = -((T)c.R[0] * (T)c.t[0] + (T)c.R[3] * (T)c.t[1] + (T)c.R[6] * (T)c.t[2]);
  const T Cy = -((T)c.R[1] * (T)c.t[0] + (T)c.R[4] * (T)c.t[1] + (T)c.R[7] * (T)c.t[2]);
  const T Cz = -((T)c.R[2] * (T)c.t[0] + (T)c.R[5] * (T)c.t[1] + (T)c.R[8] * (T)c.t[2]);
  out[0] = tx + Cx; out[1] = ty + Cy; out[2] = tz + Cz;
}
template <class T> __device__ __forceinline__ void project(const T X[3], const dpe_camera &c, T &u, T &v, T &d) {
  const T tx = (T)c.R[0] * X[0] + (T)c.R[1] * X[1] + (T)c.R[2] * X[2] + (T)c.t[0];
  const T ty = (T)c.R[3] * X[0] + (T)c.R[4] * X[1] + (T)c.R[5] * X[2] + (T)c.t[1];
  const T tz = (T)c.R[6] * X[0] + (T)c.R[7] * X[1] + (T)c.R[8] * X[2] + (T)c.t[2];
  d = (T)c.K[6] * tx + (T)c.K[7] * ty + (T)c.K[8] * tz;
  u = ((T)c.K[0] * tx + (T)c.K[1] * ty + (T)c.K[2] * tz) / d;
  v = ((T)c.K[3] * tx + (T)c.K[4] * ty + (T)c.K[5] * tz) / d;
}

// Per reference pixel: candidate test and every source entry (DPE.cpp:1468-1516).
__global__ void k_entries(const __grid_constant__ FuseArgs f) {
  const FuseView &V = f.views[f.ref];
  const int pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= V.W * V.H) return;
  const int c = pix % V.W, r = pix / V.W;
  int *eq = f.entry_q + (size_t)pix * f.ns;
  double *es = f.entry_score + (size_t)pix * f.ns;
  for (int j = 0; j < f.ns; ++j) eq[j] = -1;
  uint8_t st = 2;
  const float ref_depth = V.depth[pix];
  if (!(V.block && V.block[pix] < 128) && V.mask[pix] != 1 && !(ref_depth <= 0.0)) {
    const float rn0 = V.normal[3 * pix], rn1 = V.normal[3 * pix + 1], rn2 = V.normal[3 * pix + 2];
    double Xd[3];
    float Xf[3];
    world_point<double>((double)c, (double)r, (double)ref_depth, V.cam, Xd);
    world_point<float>((float)c, (float)r, ref_depth, V.cam, Xf);
    int n_pass = 0;
    double dyn_d = 0.0;
    float dyn_f = 0.0f;
    for (int j = 0; j < f.ns; ++j) {
      const FuseView &S = f.views[f.src[j]];
      int sr, sc;
      if (f.mode == DPE_FUSE_FP64) {
        double u, v, pd;
        project<double>(Xd, S.cam, u, v, pd);
        sr = (int)(v + 0.5); sc = (int)(u + 0.5);
      } else {
        float u, v, pd;
        project<float>(Xf, S.cam, u, v, pd);
        sr = (int)(v + 0.5f); sc = (int)(u + 0.5f);
      }
      if (!(sc >= 0 && sc < S.W && sr >= 0 && sr < S.H)) continue;
      const int sp = sr * S.W + sc;
      if (S.mask[sp] == 1) continue;
      const float sd = S.depth[sp];
      if (sd <= 0.0) continue;
      const float sn0 = S.normal[3 * sp], sn1 = S.normal[3 * sp + 1], sn2 = S.normal[3 * sp + 2];
      bool ok;
      double score;
      if (f.mode == DPE_FUSE_FP64) {
        double T[3], u, v, pd;
        world_point<double>((double)sc, (double)sr, (double)sd, S.cam, T);
        project<double>(T, V.cam, u, v, pd);
        const double ex = (double)c - u, ey = (double)r - v;
        const double reproj = sqrt(ex * ex + ey * ey);
        const double rel = fabs(pd - (double)ref_depth) / (double)ref_depth;
        const double dot = (double)rn0 * sn0 + (double)rn1 * sn1 + (double)rn2 * sn2;
        double ang = acos(dot);
        if (ang != ang) ang = 0.0;
        ok = reproj < 2.0 && rel < 0.01 && ang < (double)0.174533f;
        score = exp(-(reproj + 200.0 * rel + ang * 10.0));
      } else {
        float T[3], u, v, pd;
        world_point<float>((float)sc, (float)sr, sd, S.cam, T);
        project<float>(T, V.cam, u, v, pd);
        const float ex = (float)c - u, ey = (float)r - v;
        const float reproj = (float)sqrt((double)ex * (double)ex + (double)ey * (double)ey);
        const float rel = fabsf(pd - ref_depth) / ref_depth;
        const float dot = rn0 * sn0 + rn1 * sn1 + rn2 * sn2;
        float ang = acosf(dot);
        if (ang != ang) ang = 0.0f;
        ok = reproj < 2.0f && rel < 0.01f && ang < 0.174533f;
        score = (double)(float)exp(-(double)(reproj + 200 * rel + ang * 10));
      }
      if (!ok) continue;
      eq[j] = sp;
      es[j] = score;
      n_pass++;
      dyn_d += score;
      dyn_f += (float)score;
    }
    // the starting point of the rounds: the decision with every entry live
    if (n_pass > 0) st = fuse_accept(f, V, pix, n_pass, dyn_d, dyn_f) ? 1 : 3;
  }
  f.status[pix] = st;
}

// One round, first half: every accepted pixel stamps itself on the source pixels it tests
// consistent; the smallest key of the round on a source pixel is its first accepted claimant.
// Also clears the round's change count (k_redecide, next in the stream, counts).
__global__ void k_claim(const __grid_constant__ FuseArgs f, int npix, unsigned stamp) {
  const int pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix == 0) *f.changes = 0;
  if (pix >= npix || f.status[pix] != 1) return;
  const int *eq = f.entry_q + (size_t)pix * f.ns;
  const unsigned long long key = ((unsigned long long)stamp << 32) | (unsigned)pix;
  for (int j = 0; j < f.ns; ++j)
    if (eq[j] >= 0) atomicMin(&f.views[f.src[j]].claim[eq[j]], key);
}

// One round, second half: every candidate's decision from the round's claims.  An entry is live
// unless an earlier accepted pixel claims its source pixel.
__global__ void k_redecide(const __grid_constant__ FuseArgs f, int npix, unsigned stamp) {
  const FuseView &V = f.views[f.ref];
  const int pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= npix) return;
  const uint8_t st = f.status[pix];
  if (st != 1 && st != 3) return;
  const int *eq = f.entry_q + (size_t)pix * f.ns;
  const double *es = f.entry_score + (size_t)pix * f.ns;
  int n = 0;
  double dyn_d = 0.0;
  float dyn_f = 0.0f;
  for (int j = 0; j < f.ns; ++j) {
    if (eq[j] < 0) continue;
    const unsigned long long u = f.views[f.src[j]].claim[eq[j]];
    if ((unsigned)(u >> 32) == stamp && (int)(unsigned)u < pix) continue;  // claimed earlier
    n++;
    dyn_d += es[j];
    dyn_f += (float)es[j];
  }
  const uint8_t now = fuse_accept(f, V, pix, n, dyn_d, dyn_f) ? 1 : 3;
  if (now != st) {
    f.status[pix] = now;
    atomicAdd(f.changes, 1);
  }
}

__global__ void k_accept_flags(const uint8_t *status, int *flags, int npix) {
  const int pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix < npix) flags[pix] = status[pix] == 1 ? 1 : 0;
}

// Emit accepted points in raster order and mask the source pixels they used (DPE.cpp:1519-1541).
__global__ void k_emit(const __grid_constant__ FuseArgs f, const int *offsets, long long *base, long long capacity,
                       float *xyz, uint8_t *bgr, int32_t *origin, uint8_t *ncons, int view_index, unsigned stamp) {
  const FuseView &V = f.views[f.ref];
  const int npix = V.W * V.H;
  const int pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= npix || f.status[pix] != 1) return;
  const int *eq = f.entry_q + (size_t)pix * f.ns;
  const int c = pix % V.W, r = pix / V.W;
  float col0 = V.bgr[3 * pix], col1 = V.bgr[3 * pix + 1], col2 = V.bgr[3 * pix + 2];
  int n = 0;
  for (int j = 0; j < f.ns; ++j) {
    if (eq[j] < 0) continue;
    const FuseView &S = f.views[f.src[j]];
    const unsigned long long u = S.claim[eq[j]];
    if ((unsigned)(u >> 32) != stamp || (int)(unsigned)u != pix) continue;  // claimed by an earlier pixel
    S.mask[eq[j]] = 1;
    col0 += S.bgr[3 * eq[j]]; col1 += S.bgr[3 * eq[j] + 1]; col2 += S.bgr[3 * eq[j] + 2];
    n++;
  }
  col0 /= (n + 1); col1 /= (n + 1); col2 /= (n + 1);
  float X[3];
  world_point<float>((float)c, (float)r, V.depth[pix], V.cam, X);
  const long long k = *base + offsets[pix];
  if (k >= capacity) return;
  xyz[3 * k] = X[0]; xyz[3 * k + 1] = X[1]; xyz[3 * k + 2] = X[2];
  bgr[3 * k] = (uint8_t)col0; bgr[3 * k + 1] = (uint8_t)col1; bgr[3 * k + 2] = (uint8_t)col2;
  if (origin) { origin[2 * k] = view_index; origin[2 * k + 1] = pix; }
  if (ncons) ncons[k] = (uint8_t)n;
}

__global__ void k_advance_base(long long *base, const int *offsets, const uint8_t *status, int npix) {
  *base += offsets[npix - 1] + (status[npix - 1] == 1 ? 1 : 0);
}

// ---------------------------------------------------------------------------------------------
// TAT fusion variants (RunFusion_TAT_Intermediate, DPE.cpp:1550-1718; RunFusion_TAT_advanced,
// DPE.cpp:1720-1867).
//
// Within one reference view these read only the masks of its sources, which earlier views set, so
// all pixels of the view are independent but for one carried quantity: each source's last
// differences (the reference's per-view `diff` vector, DPE.cpp:1640 / 1804), which a pixel
// overwrites only for the sources it can test.  Pixel p therefore sees, for source j, the entry
// of the last pixel q <= p (raster order) at which j was tested.  k_tat_entries tests every
// (source, pixel) pair and writes a marker per pair; one inclusive max-scan over the markers,
// laid out source-major with an offset per source so the scan cannot carry across sources,
// gives every pixel that q; k_tat_decide then runs the reference's k loop.
// ---------------------------------------------------------------------------------------------
struct TatEntry {
  double dist, depth, angle;  // reprojection error, relative depth difference, normal angle
  int sp;                     // source pixel index
  int pad;
};

struct TatArgs {
  int mode;
  int variant;
  int ref;
  int ns;
  int npix;
  int src[kMaxSrc];
  const FuseView *views;
  TatEntry *entry;        // ns*npix, source-major: the differences where the pair was tested
  int *marker;            // ns*npix: j*(npix+1) + 1 + p where tested, j*(npix+1) otherwise
  const int *last;        // ns*npix: inclusive max-scan of marker
  uint8_t *status;        // npix: 1 kept, 2 not
  uint32_t *used;         // npix: sources counted at the accepting k
  uint8_t *count;         // npix: their number
};

// The consistency bounds at k (DPE.cpp:1555-1559, 1686; 1725-1726, 1849), in the reference's
// float arithmetic; the FP64 mode compares the double differences with the same float bounds.
struct TatBounds {
  float dist, depth, angle;
};
__device__ __forceinline__ TatBounds tat_bounds(int variant, int k) {
  const float dist_base = 0.25f;
  const float depth_base = variant == DPE_TAT_INTERMEDIATE ? 1.0f / 3500.0f : 1.0f / 3000.0f;
  const float angle_base = 0.06981317007977318f;  // 4 degrees
  const float angle_grad = 0.05235987755982988f;  // 3 degrees
  TatBounds b;
  b.dist = (float)k * dist_base;
  b.depth = (float)k * depth_base;
  b.angle = (float)k * angle_grad + angle_base;
  return b;
}

// Per (source, pixel): the reference's per-source test (DPE.cpp:1653-1681 / 1819-1845).
__global__ void k_tat_entries(const __grid_constant__ TatArgs t) {
  const FuseView &V = t.views[t.ref];
  const int pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= t.npix) return;
  const int c = pix % V.W, r = pix / V.W;
  const float ref_depth = V.depth[pix];
  const bool visited = !(V.block && V.block[pix] < 128) && !(ref_depth <= 0.0);
  float Xf[3];
  double Xd[3];
  float rn0 = 0.f, rn1 = 0.f, rn2 = 0.f;
  if (visited) {
    rn0 = V.normal[3 * pix]; rn1 = V.normal[3 * pix + 1]; rn2 = V.normal[3 * pix + 2];
    world_point<float>((float)c, (float)r, ref_depth, V.cam, Xf);
    if (t.mode == DPE_FUSE_FP64) world_point<double>((double)c, (double)r, (double)ref_depth, V.cam, Xd);
  }
  for (int j = 0; j < t.ns; ++j) {
    const size_t at = (size_t)j * t.npix + pix;
    const int seg = j * (t.npix + 1);
    int mark = seg;
    if (visited) {
      const FuseView &S = t.views[t.src[j]];
      int sr, sc;
      if (t.mode == DPE_FUSE_FP64) {
        double u, v, pd;
        project<double>(Xd, S.cam, u, v, pd);
        sr = (int)(v + 0.5); sc = (int)(u + 0.5);
      } else {
        float u, v, pd;
        project<float>(Xf, S.cam, u, v, pd);
        sr = (int)(v + 0.5f); sc = (int)(u + 0.5f);
      }
      if (sc >= 0 && sc < S.W && sr >= 0 && sr < S.H) {
        const int sp = sr * S.W + sc;
        const float sd = S.depth[sp];
        if (S.mask[sp] != 1 && !(sd <= 0.0)) {
          const float sn0 = S.normal[3 * sp], sn1 = S.normal[3 * sp + 1], sn2 = S.normal[3 * sp + 2];
          TatEntry e;
          if (t.mode == DPE_FUSE_FP64) {
            double T[3], u, v, pd;
            world_point<double>((double)sc, (double)sr, (double)sd, S.cam, T);
            project<double>(T, V.cam, u, v, pd);
            const double ex = (double)c - u, ey = (double)r - v;
            e.dist = sqrt(ex * ex + ey * ey);
            e.depth = fabs(pd - (double)ref_depth) / (double)ref_depth;
            double ang = acos((double)rn0 * sn0 + (double)rn1 * sn1 + (double)rn2 * sn2);
            e.angle = ang != ang ? 0.0 : ang;
          } else {
            float T[3], u, v, pd;
            world_point<float>((float)sc, (float)sr, sd, S.cam, T);
            project<float>(T, V.cam, u, v, pd);
            const float ex = (float)c - u, ey = (float)r - v;
            e.dist = (float)sqrt((double)ex * (double)ex + (double)ey * (double)ey);
            e.depth = fabsf(pd - ref_depth) / ref_depth;
            const float ang = acosf(rn0 * sn0 + rn1 * sn1 + rn2 * sn2);
            e.angle = ang != ang ? 0.0f : ang;
          }
          e.sp = sp;
          e.pad = 0;
          t.entry[at] = e;
          mark = seg + 1 + pix;
        }
      }
    }
    t.marker[at] = mark;
  }
}

struct MaxInt {
  __device__ __forceinline__ int operator()(int a, int b) const { return a > b ? a : b; }
};

// The entry source j carries into pixel pix; false while j has not been tested in this view.
__device__ __forceinline__ bool tat_carried(const TatArgs &t, int j, int pix, TatEntry &e) {
  const int seg = j * (t.npix + 1);
  const int m = t.last[(size_t)j * t.npix + pix];
  if (m <= seg) return false;
  e = t.entry[(size_t)j * t.npix + (m - seg - 1)];
  return true;
}

__device__ __forceinline__ bool tat_passes(const TatArgs &t, const TatEntry &e, int k) {
  const TatBounds b = tat_bounds(t.variant, k);
  if (t.mode == DPE_FUSE_FP64) {
    const bool ok = e.dist < (double)b.dist && e.depth < (double)b.depth;
    return t.variant == DPE_TAT_ADVANCED ? ok : ok && e.angle < (double)b.angle;
  }
  const bool ok = (float)e.dist < b.dist && (float)e.depth < b.depth;
  return t.variant == DPE_TAT_ADVANCED ? ok : ok && (float)e.angle < b.angle;
}

// Per pixel: the k loop (DPE.cpp:1682-1712 / 1846-1861).  The bounds grow with k, so a source
// that passes at k passes at every larger k: each source's first passing k is found once, and
// the count at k is the number of sources whose first passing k is <= k.
__global__ void k_tat_decide(const __grid_constant__ TatArgs t) {
  const FuseView &V = t.views[t.ref];
  const int pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= t.npix) return;
  uint8_t st = 2;
  uint32_t used = 0;
  int count = 0;
  const float ref_depth = V.depth[pix];
  if (!(V.block && V.block[pix] < 128) && !(ref_depth <= 0.0) && t.ns >= 2) {
    uint8_t first[kMaxSrc];
    for (int j = 0; j < t.ns; ++j) {
      first[j] = (uint8_t)(t.ns + 1);
      TatEntry e;
      if (!tat_carried(t, j, pix, e)) continue;
      for (int k = 2; k <= t.ns; ++k)
        if (tat_passes(t, e, k)) { first[j] = (uint8_t)k; break; }
    }
    for (int k = 2; k <= t.ns; ++k) {
      uint32_t m = 0;
      int n = 0;
      for (int j = 0; j < t.ns; ++j)
        if (first[j] <= k) { m |= 1u << j; n++; }
      if (n >= k) { st = 1; used = m; count = n; break; }
    }
  }
  t.status[pix] = st;
  t.used[pix] = used;
  t.count[pix] = (uint8_t)count;
}

// Emit kept pixels in raster order (DPE.cpp:1697-1710 / 1852-1859) and mask them.
__global__ void k_tat_emit(const __grid_constant__ TatArgs t, const int *offsets, long long *base, long long capacity,
                           float *xyz, uint8_t *bgr, int32_t *origin, uint8_t *ncons, int view_index) {
  const FuseView &V = t.views[t.ref];
  const int pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= t.npix || t.status[pix] != 1) return;
  V.mask[pix] = 1;
  const int c = pix % V.W, r = pix / V.W;
  float col0 = V.bgr[3 * pix], col1 = V.bgr[3 * pix + 1], col2 = V.bgr[3 * pix + 2];
  const int n = t.count[pix];
  if (t.variant == DPE_TAT_INTERMEDIATE) {
    const uint32_t used = t.used[pix];
    for (int j = 0; j < t.ns; ++j) {
      if (!(used >> j & 1u)) continue;
      TatEntry e;
      tat_carried(t, j, pix, e);
      const uint8_t *sc = t.views[t.src[j]].bgr + 3 * (size_t)e.sp;
      col0 += (float)sc[0]; col1 += (float)sc[1]; col2 += (float)sc[2];
    }
    col0 /= (n + 1.0f); col1 /= (n + 1.0f); col2 /= (n + 1.0f);
  }
  float X[3];
  world_point<float>((float)c, (float)r, V.depth[pix], V.cam, X);
  const long long k = *base + offsets[pix];
  if (k >= capacity) return;
  xyz[3 * k] = X[0]; xyz[3 * k + 1] = X[1]; xyz[3 * k + 2] = X[2];
  bgr[3 * k] = (uint8_t)col0; bgr[3 * k + 1] = (uint8_t)col1; bgr[3 * k + 2] = (uint8_t)col2;
  if (origin) { origin[2 * k] = view_index; origin[2 * k + 1] = pix; }
  if (ncons) ncons[k] = (uint8_t)n;
}

// Device buffers shared by both fusion rules: every view's arrays and consumed-pixel mask, the
// per-view decision and scan buffers, and the point output.
struct FuseBuffers {
  std::vector<FuseView> hv;
  unsigned round = 0;  // rounds run in this call (the claim keys' stamps)
  long long rounds = 0;
  FuseView *d_views = nullptr;
  size_t max_pix = 0, total_pix = 0;
  int max_ns = 1;
  uint8_t *status = nullptr;
  int *flags = nullptr, *offsets = nullptr;
  long long *base = nullptr;
  void *scan_tmp = nullptr;
  size_t scan_bytes = 0;
  long long cap_dev = 0;
  float *xyz = nullptr;
  uint8_t *rgb = nullptr;
  int32_t *origin = nullptr;
  uint8_t *ncons = nullptr;
};

// Checks the views, places their arrays on the device, clears the masks and starts the timer.
static int fuse_prepare(dpe_ctx *ctx, const dpe_fusion_in *in, const dpe_fusion_out *out, bool need_weak,
                        FuseBuffers &B) {
  if (!ctx || !in || !out || in->num_views < 1 || !in->views) return DPE_ERR_INVALID_ARGUMENT;
  if (in->mode != DPE_FUSE_FP64 && in->mode != DPE_FUSE_FLOAT) return DPE_ERR_INVALID_ARGUMENT;
  if (in->memory != DPE_MEM_HOST && in->memory != DPE_MEM_DEVICE) return DPE_ERR_INVALID_ARGUMENT;
  if (out->capacity < 0 || (out->capacity > 0 && (!out->xyz || !out->bgr))) return DPE_ERR_INVALID_ARGUMENT;
  const int nv = in->num_views;
  for (int i = 0; i < nv; ++i) {
    const dpe_fusion_view &v = in->views[i];
    if (v.width <= 0 || v.height <= 0 || !v.depth || !v.normal || !v.bgr || (need_weak && !v.weak))
      return DPE_ERR_INVALID_ARGUMENT;
    if ((size_t)v.width * v.height > (size_t)INT_MAX / 2) return DPE_ERR_INVALID_ARGUMENT;
    if (v.num_src < 0 || v.num_src > kMaxSrc || (v.num_src > 0 && !v.src_views)) return DPE_ERR_INVALID_ARGUMENT;
    for (int j = 0; j < v.num_src; ++j)
      if (v.src_views[j] < 0 || v.src_views[j] >= nv || v.src_views[j] == i) return DPE_ERR_INVALID_ARGUMENT;
    B.max_pix = std::max(B.max_pix, (size_t)v.width * v.height);
    B.total_pix += (size_t)v.width * v.height;
    B.max_ns = std::max(B.max_ns, v.num_src);
  }
  DPE_TRY(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  Arena &A = ctx->arena;
  const bool host = in->memory == DPE_MEM_HOST;
  const size_t total_pix = B.total_pix, max_pix = B.max_pix;

  B.hv.resize(nv);
  uint8_t *masks = A.get<uint8_t>("f_mask", total_pix);
  unsigned long long *claim = A.get<unsigned long long>("f_claim", total_pix);
  // all ones: the stamp of round 0, older than every round of this call
  if (claim) DPE_TRY(cudaMemsetAsync(claim, 0xFF, total_pix * sizeof(unsigned long long), ctx->stream));
  float *d_depth = host ? A.get<float>("f_depth", total_pix) : nullptr;
  float *d_normal = host ? A.get<float>("f_normal", total_pix * 3) : nullptr;
  uint8_t *d_weak = host && need_weak ? A.get<uint8_t>("f_weak", total_pix) : nullptr;
  uint8_t *d_bgr = host ? A.get<uint8_t>("f_bgr", total_pix * 3) : nullptr;
  uint8_t *d_block = host ? A.get<uint8_t>("f_block", total_pix) : nullptr;
  B.d_views = A.get<FuseView>("f_views", nv);
  B.status = A.get<uint8_t>("f_status", max_pix);
  B.flags = A.get<int>("f_flags", max_pix);
  B.offsets = A.get<int>("f_offsets", max_pix);
  B.base = A.get<long long>("f_base", 1);
  cub::DeviceScan::ExclusiveSum(nullptr, B.scan_bytes, B.flags, B.offsets, (int)max_pix, s);
  B.scan_tmp = A.get<uint8_t>("f_scan_tmp", B.scan_bytes + 16);
  B.cap_dev = (long long)std::min<size_t>((size_t)std::max<int64_t>(out->capacity, 0), total_pix);
  B.xyz = A.get<float>("f_xyz", (size_t)B.cap_dev * 3 + 3);
  B.rgb = A.get<uint8_t>("f_rgb", (size_t)B.cap_dev * 3 + 3);
  B.origin = out->origin ? A.get<int32_t>("f_origin", (size_t)B.cap_dev * 2 + 2) : nullptr;
  B.ncons = out->num_consistent ? A.get<uint8_t>("f_ncons", (size_t)B.cap_dev + 1) : nullptr;
  if (!A.ok()) return DPE_ERR_OUT_OF_MEMORY;

  size_t off = 0;
  for (int i = 0; i < nv; ++i) {
    const dpe_fusion_view &v = in->views[i];
    const size_t n = (size_t)v.width * v.height;
    FuseView &f = B.hv[i];
    f.W = v.width; f.H = v.height; f.cam = v.camera;
    f.mask = masks + off; f.claim = claim + off;
    if (host) {
      DPE_TRY(cudaMemcpyAsync(d_depth + off, v.depth, n * 4, cudaMemcpyHostToDevice, s));
      DPE_TRY(cudaMemcpyAsync(d_normal + 3 * off, v.normal, n * 12, cudaMemcpyHostToDevice, s));
      DPE_TRY(cudaMemcpyAsync(d_bgr + 3 * off, v.bgr, n * 3, cudaMemcpyHostToDevice, s));
      f.depth = d_depth + off; f.normal = d_normal + 3 * off; f.bgr = d_bgr + 3 * off;
      f.weak = nullptr;
      if (need_weak) {
        DPE_TRY(cudaMemcpyAsync(d_weak + off, v.weak, n, cudaMemcpyHostToDevice, s));
        f.weak = d_weak + off;
      }
      f.block = nullptr;
      if (v.block_mask) {
        DPE_TRY(cudaMemcpyAsync(d_block + off, v.block_mask, n, cudaMemcpyHostToDevice, s));
        f.block = d_block + off;
      }
    } else {
      f.depth = v.depth; f.normal = v.normal; f.weak = v.weak; f.bgr = v.bgr; f.block = v.block_mask;
    }
    off += n;
  }
  DPE_TRY(cudaMemcpyAsync(B.d_views, B.hv.data(), sizeof(FuseView) * nv, cudaMemcpyHostToDevice, s));
  DPE_TRY(cudaMemsetAsync(masks, 0, total_pix, s));
  DPE_TRY(cudaMemsetAsync(B.base, 0, sizeof(long long), s));
  DPE_TRY(cudaEventRecord(ctx->ev0, s));
  return DPE_OK;
}

// Raster-order offsets of the kept pixels of one view (status 1).
static int fuse_offsets(dpe_ctx *ctx, FuseBuffers &B, int npix) {
  cudaStream_t s = ctx->stream;
  const unsigned blocks = (unsigned)((npix + 255) / 256);
  k_accept_flags<<<blocks, 256, 0, s>>>(B.status, B.flags, npix);
  DPE_LAUNCHED("k_accept_flags", s);
  DPE_TRY(cub::DeviceScan::ExclusiveSum(B.scan_tmp, B.scan_bytes, B.flags, B.offsets, npix, s));
  return DPE_OK;
}

static int fuse_advance(dpe_ctx *ctx, FuseBuffers &B, int npix) {
  cudaStream_t s = ctx->stream;
  k_advance_base<<<1, 1, 0, s>>>(B.base, B.offsets, B.status, npix);
  DPE_LAUNCHED("k_advance_base", s);
  return DPE_OK;
}

// Stops the timer and copies the points back.
static int fuse_finish(dpe_ctx *ctx, FuseBuffers &B, dpe_fusion_out *out) {
  cudaStream_t s = ctx->stream;
  DPE_TRY(cudaEventRecord(ctx->ev1, s));
  long long count = 0;
  DPE_TRY(cudaMemcpyAsync(&count, B.base, sizeof(long long), cudaMemcpyDeviceToHost, s));
  DPE_TRY(cudaStreamSynchronize(s));
  const long long ncopy = std::min<long long>(count, B.cap_dev);
  if (ncopy > 0) {
    DPE_TRY(cudaMemcpyAsync(out->xyz, B.xyz, (size_t)ncopy * 12, cudaMemcpyDeviceToHost, s));
    DPE_TRY(cudaMemcpyAsync(out->bgr, B.rgb, (size_t)ncopy * 3, cudaMemcpyDeviceToHost, s));
    if (out->origin) DPE_TRY(cudaMemcpyAsync(out->origin, B.origin, (size_t)ncopy * 8, cudaMemcpyDeviceToHost, s));
    if (out->num_consistent)
      DPE_TRY(cudaMemcpyAsync(out->num_consistent, B.ncons, (size_t)ncopy, cudaMemcpyDeviceToHost, s));
  }
  DPE_TRY(cudaStreamSynchronize(s));
  ctx->collect();
  float ms = 0.f;
  DPE_TRY(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  out->gpu_ms = ms;
  out->count = count;
  return count > out->capacity ? DPE_ERR_CAPACITY : DPE_OK;
}

}  // namespace

extern "C" int dpe_fuse(dpe_ctx *ctx, const dpe_fusion_in *in, dpe_fusion_out *out) {
  FuseBuffers B;
  int st = fuse_prepare(ctx, in, out, true, B);
  if (st != DPE_OK) return st;
  cudaStream_t s = ctx->stream;
  Arena &A = ctx->arena;
  int *entry_q = A.get<int>("f_eq", B.max_pix * B.max_ns);
  double *entry_s = A.get<double>("f_es", B.max_pix * B.max_ns);
  int *changes = A.get<int>("f_changes", 1);
  if (!A.ok()) return DPE_ERR_OUT_OF_MEMORY;

  FuseArgs f;
  std::memset(&f, 0, sizeof(f));
  f.mode = in->mode;
  f.min_consistent = in->min_consistent;
  f.views = B.d_views;
  f.entry_q = entry_q;
  f.entry_score = entry_s;
  f.status = B.status;
  f.changes = changes;
  for (int i = 0; i < in->num_views; ++i) {
    const dpe_fusion_view &v = in->views[i];
    const int npix = v.width * v.height;
    const unsigned blocks = (unsigned)((npix + 255) / 256);
    f.ref = i;
    f.ns = v.num_src;
    for (int j = 0; j < v.num_src; ++j) f.src[j] = v.src_views[j];
    unsigned stamp = 0xFFFFFFFFu;
    if (v.num_src > 0) {
      DPE_TIMED(ctx, KID_FUSE_ENTRIES, s, k_entries<<<blocks, 256, 0, s>>>(f));
      DPE_LAUNCHED("k_entries", s);
      // Jacobi rounds until one changes nothing.  Each round makes at least the first undecided
      // pixel of the dependency order final, so npix + 1 rounds always suffice.
      for (int round = 0; round < npix + 1; ++round) {
        stamp = 0xFFFFFFFFu - (unsigned)(++B.round);
        DPE_TIMED(ctx, KID_FUSE_ROUNDS, s, k_claim<<<blocks, 256, 0, s>>>(f, npix, stamp));
        DPE_LAUNCHED("k_claim", s);
        DPE_TIMED(ctx, KID_FUSE_ROUNDS, s, k_redecide<<<blocks, 256, 0, s>>>(f, npix, stamp));
        DPE_LAUNCHED("k_redecide", s);
        int changed = 0;
        DPE_TRY(cudaMemcpyAsync(&changed, changes, 4, cudaMemcpyDeviceToHost, s));
        DPE_TRY(cudaStreamSynchronize(s));
        B.rounds++;
        if (changed == 0) break;
      }
    } else {
      DPE_TRY(cudaMemsetAsync(B.status, 2, npix, s));
    }
    if ((st = fuse_offsets(ctx, B, npix)) != DPE_OK) return st;
    DPE_TIMED(ctx, KID_FUSE_EMIT, s,
              k_emit<<<blocks, 256, 0, s>>>(f, B.offsets, B.base, B.cap_dev, B.xyz, B.rgb, B.origin, B.ncons, i,
                                            stamp));
    DPE_LAUNCHED("k_emit", s);
    if ((st = fuse_advance(ctx, B, npix)) != DPE_OK) return st;
  }
  return fuse_finish(ctx, B, out);
}

extern "C" int dpe_fuse_tat(dpe_ctx *ctx, const dpe_fusion_in *in, int variant, dpe_fusion_out *out) {
  if (variant != DPE_TAT_INTERMEDIATE && variant != DPE_TAT_ADVANCED) return DPE_ERR_INVALID_ARGUMENT;
  FuseBuffers B;
  int st = fuse_prepare(ctx, in, out, false, B);
  if (st != DPE_OK) return st;
  // the scan markers of a view must fit an int: ns * (npix + 1) <= INT_MAX
  if ((size_t)B.max_ns * (B.max_pix + 1) > (size_t)INT_MAX) return DPE_ERR_INVALID_ARGUMENT;
  cudaStream_t s = ctx->stream;
  Arena &A = ctx->arena;
  const size_t pairs = B.max_pix * B.max_ns;
  TatEntry *entry = A.get<TatEntry>("f_tat_entry", pairs);
  int *marker = A.get<int>("f_tat_marker", pairs);
  int *last = A.get<int>("f_tat_last", pairs);
  uint32_t *used = A.get<uint32_t>("f_tat_used", B.max_pix);
  uint8_t *count = A.get<uint8_t>("f_tat_count", B.max_pix);
  size_t max_scan_bytes = 0;
  cub::DeviceScan::InclusiveScan(nullptr, max_scan_bytes, marker, last, MaxInt(), (int)pairs, s);
  void *max_scan_tmp = A.get<uint8_t>("f_tat_scan_tmp", max_scan_bytes + 16);
  if (!A.ok()) return DPE_ERR_OUT_OF_MEMORY;

  TatArgs t;
  std::memset(&t, 0, sizeof(t));
  t.mode = in->mode;
  t.variant = variant;
  t.views = B.d_views;
  t.entry = entry;
  t.marker = marker;
  t.last = last;
  t.status = B.status;
  t.used = used;
  t.count = count;
  for (int i = 0; i < in->num_views; ++i) {
    const dpe_fusion_view &v = in->views[i];
    const int npix = v.width * v.height;
    const unsigned blocks = (unsigned)((npix + 255) / 256);
    t.ref = i;
    t.ns = v.num_src;
    t.npix = npix;
    for (int j = 0; j < v.num_src; ++j) t.src[j] = v.src_views[j];
    if (v.num_src >= 2) {
      DPE_TIMED(ctx, KID_FUSE_ENTRIES, s, k_tat_entries<<<blocks, 256, 0, s>>>(t));
      DPE_LAUNCHED("k_tat_entries", s);
      size_t nb = max_scan_bytes;
      DPE_TRY(cub::DeviceScan::InclusiveScan(max_scan_tmp, nb, marker, last, MaxInt(), npix * v.num_src, s));
      DPE_TIMED(ctx, KID_FUSE_TAT, s, k_tat_decide<<<blocks, 256, 0, s>>>(t));
      DPE_LAUNCHED("k_tat_decide", s);
    } else {  // the k loop of 2..num_src is empty: nothing is kept
      DPE_TRY(cudaMemsetAsync(B.status, 2, npix, s));
    }
    if ((st = fuse_offsets(ctx, B, npix)) != DPE_OK) return st;
    DPE_TIMED(ctx, KID_FUSE_EMIT, s,
              k_tat_emit<<<blocks, 256, 0, s>>>(t, B.offsets, B.base, B.cap_dev, B.xyz, B.rgb, B.origin, B.ncons, i));
    DPE_LAUNCHED("k_tat_emit", s);
    if ((st = fuse_advance(ctx, B, npix)) != DPE_OK) return st;
  }
  return fuse_finish(ctx, B, out);
}
