// fusion.cu -- depth-map fusion (RunFusion, DPE.cpp:1387-1548) on the GPU with the reference's
// order-dependent result.
//
// The reference walks views in pair.txt order and pixels in raster order; an accepted pixel
// masks the source pixels it used, and a masked source pixel is skipped by every later pixel.
// Equivalently, for one reference view: a (source, pixel) entry of pixel p is masked iff an
// earlier pixel of the same view that lists the same entry was accepted (or a previous view
// masked it).  The kernels below compute every pixel's consistency entries in parallel, then
// decide pixels in "waves": a pixel is decided once every earlier contender for each of its
// entries is decided.  The globally first undecided pixel is always decidable, so the waves end;
// in practice contention is sparse and a handful of waves suffice.  Decisions, counts, point
// order and colours are those of the sequential loop.
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
  int *acc_min;  // per pixel: smallest accepted contender of the current reference view
  int *und_min;  // per pixel: smallest undecided contender in the current wave
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
  uint8_t *status;        // W*H: 0 undecided, 1 accepted, 2 rejected / not a candidate
  int *remaining;
};

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
    }
    if (n_pass > 0) st = 0;
  }
  f.status[pix] = st;
}

__global__ void k_mark_undecided(const __grid_constant__ FuseArgs f, int npix) {
  const int pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= npix || f.status[pix] != 0) return;
  const int *eq = f.entry_q + (size_t)pix * f.ns;
  for (int j = 0; j < f.ns; ++j)
    if (eq[j] >= 0) atomicMin(&f.views[f.src[j]].und_min[eq[j]], pix);
}

__global__ void k_decide(const __grid_constant__ FuseArgs f, int npix) {
  const FuseView &V = f.views[f.ref];
  const int pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= npix || f.status[pix] != 0) return;
  const int *eq = f.entry_q + (size_t)pix * f.ns;
  const double *es = f.entry_score + (size_t)pix * f.ns;
  int n = 0;
  double dyn_d = 0.0;
  float dyn_f = 0.0f;
  for (int j = 0; j < f.ns; ++j) {
    if (eq[j] < 0) continue;
    const FuseView &S = f.views[f.src[j]];
    if (S.acc_min[eq[j]] < pix) continue;  // masked by an earlier accepted pixel of this view
    if (S.und_min[eq[j]] < pix) { atomicAdd(f.remaining, 1); return; }  // an earlier contender is undecided
    n++;
    dyn_d += es[j];
    dyn_f += (float)es[j];
  }
  const float factor = V.weak[pix] == DPE_WEAK ? 0.45f : 0.3f;
  const int need = f.min_consistent > 1 ? f.min_consistent : 1;
  const bool accept = f.mode == DPE_FUSE_FP64 ? (n >= need && dyn_d > (double)factor * n) : (n >= need && dyn_f > factor * n);
  f.status[pix] = accept ? 1 : 2;
  if (accept)
    for (int j = 0; j < f.ns; ++j)
      if (eq[j] >= 0) atomicMin(&f.views[f.src[j]].acc_min[eq[j]], pix);
}

__global__ void k_accept_flags(const uint8_t *status, int *flags, int npix) {
  const int pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix < npix) flags[pix] = status[pix] == 1 ? 1 : 0;
}

// Emit accepted points in raster order and mask the source pixels they used (DPE.cpp:1519-1541).
__global__ void k_emit(const __grid_constant__ FuseArgs f, const int *offsets, long long *base, long long capacity,
                       float *xyz, uint8_t *bgr, int32_t *origin, uint8_t *ncons, int view_index) {
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
    if (S.acc_min[eq[j]] != pix) continue;  // masked by an earlier accepted pixel
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

}  // namespace

extern "C" int dpe_fuse(dpe_ctx *ctx, const dpe_fusion_in *in, dpe_fusion_out *out) {
  if (!ctx || !in || !out || in->num_views < 1 || !in->views) return DPE_ERR_INVALID_ARGUMENT;
  if (in->mode != DPE_FUSE_FP64 && in->mode != DPE_FUSE_FLOAT) return DPE_ERR_INVALID_ARGUMENT;
  if (in->memory != DPE_MEM_HOST && in->memory != DPE_MEM_DEVICE) return DPE_ERR_INVALID_ARGUMENT;
  if (out->capacity < 0 || (out->capacity > 0 && (!out->xyz || !out->bgr))) return DPE_ERR_INVALID_ARGUMENT;
  const int nv = in->num_views;
  size_t max_pix = 0, total_pix = 0;
  int max_ns = 1;
  for (int i = 0; i < nv; ++i) {
    const dpe_fusion_view &v = in->views[i];
    if (v.width <= 0 || v.height <= 0 || !v.depth || !v.normal || !v.weak || !v.bgr) return DPE_ERR_INVALID_ARGUMENT;
    if (v.num_src < 0 || v.num_src > kMaxSrc || (v.num_src > 0 && !v.src_views)) return DPE_ERR_INVALID_ARGUMENT;
    for (int j = 0; j < v.num_src; ++j)
      if (v.src_views[j] < 0 || v.src_views[j] >= nv || v.src_views[j] == i) return DPE_ERR_INVALID_ARGUMENT;
    max_pix = std::max(max_pix, (size_t)v.width * v.height);
    total_pix += (size_t)v.width * v.height;
    max_ns = std::max(max_ns, v.num_src);
  }
  DPE_TRY(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  Arena &A = ctx->arena;
  const bool host = in->memory == DPE_MEM_HOST;

  // ---- per-view device data
  std::vector<FuseView> hv(nv);
  uint8_t *masks = A.get<uint8_t>("f_mask", total_pix);
  int *acc = A.get<int>("f_acc", total_pix);
  int *und = A.get<int>("f_und", total_pix);
  float *d_depth = host ? A.get<float>("f_depth", total_pix) : nullptr;
  float *d_normal = host ? A.get<float>("f_normal", total_pix * 3) : nullptr;
  uint8_t *d_weak = host ? A.get<uint8_t>("f_weak", total_pix) : nullptr;
  uint8_t *d_bgr = host ? A.get<uint8_t>("f_bgr", total_pix * 3) : nullptr;
  uint8_t *d_block = host ? A.get<uint8_t>("f_block", total_pix) : nullptr;
  FuseView *d_views = A.get<FuseView>("f_views", nv);
  int *entry_q = A.get<int>("f_eq", max_pix * max_ns);
  double *entry_s = A.get<double>("f_es", max_pix * max_ns);
  uint8_t *status = A.get<uint8_t>("f_status", max_pix);
  int *flags = A.get<int>("f_flags", max_pix);
  int *offsets = A.get<int>("f_offsets", max_pix);
  int *remaining = A.get<int>("f_remaining", 1);
  long long *base = A.get<long long>("f_base", 1);
  size_t scan_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, flags, offsets, (int)max_pix, s);
  void *scan_tmp = A.get<uint8_t>("f_scan_tmp", scan_bytes + 16);
  const long long cap_dev = (long long)std::min<size_t>((size_t)std::max<int64_t>(out->capacity, 0), total_pix);
  float *d_xyz = A.get<float>("f_xyz", (size_t)cap_dev * 3 + 3);
  uint8_t *d_rgb = A.get<uint8_t>("f_rgb", (size_t)cap_dev * 3 + 3);
  int32_t *d_origin = out->origin ? A.get<int32_t>("f_origin", (size_t)cap_dev * 2 + 2) : nullptr;
  uint8_t *d_ncons = out->num_consistent ? A.get<uint8_t>("f_ncons", (size_t)cap_dev + 1) : nullptr;
  if (!A.ok()) return DPE_ERR_OUT_OF_MEMORY;

  size_t off = 0;
  for (int i = 0; i < nv; ++i) {
    const dpe_fusion_view &v = in->views[i];
    const size_t n = (size_t)v.width * v.height;
    FuseView &f = hv[i];
    f.W = v.width; f.H = v.height; f.cam = v.camera;
    f.mask = masks + off; f.acc_min = acc + off; f.und_min = und + off;
    if (host) {
      DPE_TRY(cudaMemcpyAsync(d_depth + off, v.depth, n * 4, cudaMemcpyHostToDevice, s));
      DPE_TRY(cudaMemcpyAsync(d_normal + 3 * off, v.normal, n * 12, cudaMemcpyHostToDevice, s));
      DPE_TRY(cudaMemcpyAsync(d_weak + off, v.weak, n, cudaMemcpyHostToDevice, s));
      DPE_TRY(cudaMemcpyAsync(d_bgr + 3 * off, v.bgr, n * 3, cudaMemcpyHostToDevice, s));
      f.depth = d_depth + off; f.normal = d_normal + 3 * off; f.weak = d_weak + off; f.bgr = d_bgr + 3 * off;
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
  DPE_TRY(cudaMemcpyAsync(d_views, hv.data(), sizeof(FuseView) * nv, cudaMemcpyHostToDevice, s));
  DPE_TRY(cudaMemsetAsync(masks, 0, total_pix, s));
  DPE_TRY(cudaMemsetAsync(base, 0, sizeof(long long), s));
  DPE_TRY(cudaEventRecord(ctx->ev0, s));

  FuseArgs f;
  std::memset(&f, 0, sizeof(f));
  f.mode = in->mode;
  f.min_consistent = in->min_consistent;
  f.views = d_views;
  f.entry_q = entry_q;
  f.entry_score = entry_s;
  f.status = status;
  f.remaining = remaining;
  for (int i = 0; i < nv; ++i) {
    const dpe_fusion_view &v = in->views[i];
    const int npix = v.width * v.height;
    const unsigned blocks = (unsigned)((npix + 255) / 256);
    f.ref = i;
    f.ns = v.num_src;
    for (int j = 0; j < v.num_src; ++j) f.src[j] = v.src_views[j];
    for (int j = 0; j < v.num_src; ++j) {
      const FuseView &S = hv[v.src_views[j]];
      DPE_TRY(cudaMemsetAsync(S.acc_min, 0x7F, (size_t)S.W * S.H * 4, s));
    }
    if (v.num_src > 0) {
      DPE_TIMED(ctx, KID_FUSE_ENTRIES, s, k_entries<<<blocks, 256, 0, s>>>(f));
      DPE_LAUNCHED("k_entries", s);
      // waves until every candidate pixel is decided; each wave decides at least the first one
      for (int wave = 0; wave < npix + 1; ++wave) {
        for (int j = 0; j < v.num_src; ++j) {
          const FuseView &S = hv[v.src_views[j]];
          DPE_TRY(cudaMemsetAsync(S.und_min, 0x7F, (size_t)S.W * S.H * 4, s));
        }
        DPE_TRY(cudaMemsetAsync(remaining, 0, 4, s));
        DPE_TIMED(ctx, KID_FUSE_WAVES, s, k_mark_undecided<<<blocks, 256, 0, s>>>(f, npix));
        DPE_LAUNCHED("k_mark_undecided", s);
        DPE_TIMED(ctx, KID_FUSE_WAVES, s, k_decide<<<blocks, 256, 0, s>>>(f, npix));
        DPE_LAUNCHED("k_decide", s);
        int rem = 0;
        DPE_TRY(cudaMemcpyAsync(&rem, remaining, 4, cudaMemcpyDeviceToHost, s));
        DPE_TRY(cudaStreamSynchronize(s));
        if (rem == 0) break;
      }
    } else {
      DPE_TRY(cudaMemsetAsync(status, 2, npix, s));
    }
    k_accept_flags<<<blocks, 256, 0, s>>>(status, flags, npix);
    DPE_LAUNCHED("k_accept_flags", s);
    DPE_TRY(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, flags, offsets, npix, s));
    DPE_TIMED(ctx, KID_FUSE_EMIT, s, k_emit<<<blocks, 256, 0, s>>>(f, offsets, base, cap_dev, d_xyz, d_rgb, d_origin, d_ncons, i));
    DPE_LAUNCHED("k_emit", s);
    k_advance_base<<<1, 1, 0, s>>>(base, offsets, status, npix);
    DPE_LAUNCHED("k_advance_base", s);
  }
  DPE_TRY(cudaEventRecord(ctx->ev1, s));
  long long count = 0;
  DPE_TRY(cudaMemcpyAsync(&count, base, sizeof(long long), cudaMemcpyDeviceToHost, s));
  DPE_TRY(cudaStreamSynchronize(s));
  const long long ncopy = std::min<long long>(count, cap_dev);
  if (ncopy > 0) {
    DPE_TRY(cudaMemcpyAsync(out->xyz, d_xyz, (size_t)ncopy * 12, cudaMemcpyDeviceToHost, s));
    DPE_TRY(cudaMemcpyAsync(out->bgr, d_rgb, (size_t)ncopy * 3, cudaMemcpyDeviceToHost, s));
    if (out->origin) DPE_TRY(cudaMemcpyAsync(out->origin, d_origin, (size_t)ncopy * 8, cudaMemcpyDeviceToHost, s));
    if (out->num_consistent) DPE_TRY(cudaMemcpyAsync(out->num_consistent, d_ncons, (size_t)ncopy, cudaMemcpyDeviceToHost, s));
  }
  DPE_TRY(cudaStreamSynchronize(s));
  ctx->collect();
  float ms = 0.f;
  DPE_TRY(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  out->gpu_ms = ms;
  out->count = count;
  return count > out->capacity ? DPE_ERR_CAPACITY : DPE_OK;
}
