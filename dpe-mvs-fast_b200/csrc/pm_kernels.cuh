// pm_kernels.cuh -- the per-view PatchMatch kernels (one thread per pixel of a pass).
//
// Kernel order and per-pixel semantics follow DPE::RunPatchMatch (DPE.cu:3130-3262).  B200
// design points: all per-call constants (cameras, relative poses, params, pointers) live in one
// argument block in device memory (one per problem of a batch); state is structure-of-arrays; view weights are packed as
// 4-bit counts (16 B per pixel instead of 32); the strong NCC's reference window is built once
// per thread and reused by every hypothesis and source view; the same-colour race of the
// edge-aware update is removed by reading candidates from a pre-pass snapshot.
#pragma once

#include "dpe_device.cuh"

namespace dpe {

__device__ __constant__ const int kDir[8][2] = {{0, -1}, {0, 1}, {-1, 0}, {1, 0}, {-1, -1}, {1, 1}, {-1, 1}, {1, -1}};

// ------------------------------------------------------------------ launch geometry
// A kernel runs either for one problem (a 2D grid over its pixels, or a 1D grid over a work list)
// or for a batch of problems in one launch (dpe_pm_run_batch): the batch's grid is the problems'
// grids laid end to end in one dimension, and each block finds its problem in a prefix table of
// block counts.
enum GridKind { kGridFull = 0, kGridHalf = 1, kGridList = 2 };
struct Launch {
  const PMArgs *args;  // [nprob] per-problem argument blocks
  const int *start;    // batched: [nprob + 1] first block of each problem; null for one problem
  int nprob;
};
// This block's problem, its coordinates in the problem's own grid, and that grid's width.
struct Blk {
  const PMArgs *a;
  int x, y, gx;
};
template <int kKind>
__device__ __forceinline__ Blk resolve(const Launch &L) {
  if (!L.start) return Blk{L.args, (int)blockIdx.x, (int)blockIdx.y, (int)gridDim.x};
  const int f = (int)blockIdx.x;
  int lo = 0, hi = L.nprob;  // the last problem whose first block is <= f
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (L.start[mid] <= f) lo = mid;
    else hi = mid;
  }
  const PMArgs *a = L.args + lo;
  const int local = f - L.start[lo];
  const int gx = kKind == kGridFull ? (a->W + 15) / 16 : kKind == kGridHalf ? (a->W + 31) / 32
                                                                            : L.start[lo + 1] - L.start[lo];
  return Blk{a, local % gx, local / gx, gx};
}

// pixel of colour `parity` ((x + y) % 2) handled by this thread of a half-height grid
__device__ __forceinline__ bool colour_pixel(const PMArgs &a, const Blk &B, int parity, int *px, int *py) {
  const int x = B.x * blockDim.x + threadIdx.x;
  const int yy = B.y * blockDim.y + threadIdx.y;
  const int y = 2 * yy + ((x + parity) & 1);
  *px = x; *py = y;
  return x < a.W && y < a.H;
}
__device__ __forceinline__ bool full_pixel(const PMArgs &a, const Blk &B, int *px, int *py) {
  *px = B.x * blockDim.x + threadIdx.x;
  *py = B.y * blockDim.y + threadIdx.y;
  return *px < a.W && *py < a.H;
}

// ------------------------------------------------------------------ setup
#ifdef DPE_CHECKED
// How the device reads the per-call block (checked builds compare it with the host's values).
__global__ void k_echo_args(const PMArgs *__restrict__ pa, long long *out) {
  out[0] = pa->W; out[1] = pa->H; out[2] = pa->N; out[3] = pa->P.strong_radius; out[4] = pa->P.strong_increment;
  out[5] = pa->P.use_edge; out[6] = pa->P.num_images; out[7] = (long long)sizeof(PMArgs);
}
#endif
__global__ void k_pad_image(const float *__restrict__ src, float *__restrict__ dst, int W, int H) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x - 1;
  const int y = blockIdx.y * blockDim.y + threadIdx.y - 1;
  if (x > W || y > H) return;
  const int sx = min(max(x, 0), W - 1), sy = min(max(y, 0), H - 1);
  dst[(size_t)(y + 1) * (W + 2) + (x + 1)] = src[(size_t)sy * W + sx];
}

// Staged copy of one padded source image (PMArgs::pair): word o packs P[o] (low 16 bits) and
// P[o+1] (high 16 bits) as FP16 or BF16, rounded to nearest-even.  The last word repeats P[o].
template <bool kBF16>
__global__ void k_stage_pairs(const float *__restrict__ pad, uint32_t *__restrict__ out, long long n) {
  const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= n) return;
  const float lo = pad[o], hi = pad[o + 1 < n ? o + 1 : o];
  uint32_t a, b;
  if (kBF16) {
    a = __bfloat16_as_ushort(__float2bfloat16_rn(lo));
    b = __bfloat16_as_ushort(__float2bfloat16_rn(hi));
  } else {
    a = __half_as_ushort(__float2half_rn(lo));
    b = __half_as_ushort(__float2half_rn(hi));
  }
  out[o] = a | (b << 16);
}

// Sets *flag when any of the n floats is not exact in BF16 (a float is exact when its low 16
// bits are zero: 8-bit images are).  One atomic per block.
__global__ void k_bf16_exact(const float *__restrict__ p, long long n, unsigned *flag) {
  unsigned bits = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    bits |= __float_as_uint(p[i]) & 0xFFFFu;
  if (__syncthreads_or(bits != 0) && threadIdx.x == 0) atomicOr(flag, 1u);
}

__global__ void k_init_state(const Launch lc, const float4 *plane_in, const uint32_t *views_in,
                             const uint8_t *weak_in, int *weak_flag) {
  const Blk B = resolve<kGridFull>(lc);
  const PMArgs &a = *B.a;
  int px, py;
  if (!full_pixel(a, B, &px, &py)) return;
  const int c = px + py * a.W;
  a.plane[c] = (a.P.state != DPE_FIRST_INIT && plane_in) ? plane_in[c] : make_float4(0, 0, 0, 0);
  a.views[c] = (a.P.state != DPE_FIRST_INIT && views_in) ? views_in[c] : 0u;
  const uint8_t wk = a.P.use_APD ? weak_in[c] : (uint8_t)DPE_STRONG;
  a.weak[c] = wk;
  weak_flag[c] = (a.P.use_APD && wk == DPE_WEAK) ? 1 : 0;
  a.rng_ctr[c] = 0u;
  a.radius[c] = a.P.strong_radius;
  a.fit_plane[c] = make_float4(0, 0, 0, 0);
  a.reliable[c] = 0;
  a.complexity[c] = 0.0f;
  a.vweight[c] = make_uint4(0, 0, 0, 0);
  a.cost[c] = 0.0f;
}

// ------------------------------------------------------------------ GenEdgeInform (DPE.cu:2487-2595)
__global__ void k_gen_edge_inform(const Launch lc) {
  const Blk B = resolve<kGridFull>(lc);
  const PMArgs &a = *B.a;
  int px, py;
  if (!full_pixel(a, B, &px, &py)) return;
  const int W = a.W, H = a.H, center = px + py * W;
  if (a.P.use_edge) {
    short2 *en = &a.edge_neigh[(size_t)center * 8];
    for (int i = 0; i < 8; ++i) {
      short2 found = make_short2(-1, -1);
      const int dx = kDir[i][0], dy = kDir[i][1];
      int nx = px + dx, ny = py + dy;
      while (nx >= 0 && nx < W && ny >= 0 && ny < H) {
        if (a.edge[nx + ny * W]) { found = make_short2(nx, ny); break; }
        nx += dx; ny += dy;
      }
      en[i] = found;
    }
    const int r = a.P.strong_radius;
    int edge_pix = 0, tot_pix = 0, bound_pix = 0;
    for (int i = -r; i <= r; ++i)
      for (int j = -r; j <= r; ++j) {
        const int nx = px + i, ny = py + j;
        if (nx < 0 || nx >= W || ny < 0 || ny >= H) continue;
        if (a.edge[ny * W + nx]) edge_pix++;
        if (a.P.use_label && a.label[ny * W + nx] == 0) bound_pix++;
        tot_pix++;
      }
    float density = 1.0f * edge_pix / tot_pix;
    if (a.P.use_label) density = cvmax(density, bound_pix / tot_pix);  // integer division (quirk Q6)
    a.complexity[center] = (float)(1.0f / (1.0f + exp(-25.0 * (density - 0.35))));
  }
  if (a.P.use_label && a.weak[center] == DPE_WEAK) {
    const int cl = a.label[center];
    if (cl > 0) {
      short2 *lb = &a.lab_bound[(size_t)a.nmap[center] * 8];
      for (int i = 0; i < 8; ++i) {
        const int dx = kDir[i][0], dy = kDir[i][1];
        int nx = px + dx, ny = py + dy, lx = -1, ly = -1;
        while (nx >= 0 && nx < W && ny >= 0 && ny < H) {
          const int nl = a.label[nx + ny * W];
          if (nl == cl) { lx = nx; ly = ny; }
          else if (nl == -1) break;
          nx += dx; ny += dy;
        }
        lb[i] = make_short2(lx, ly);
      }
    }
  }
}

// ------------------------------------------------------------------ FindNearestStrongPoint (DPE.cu:2859-2893)
__device__ __forceinline__ void find_nearest_strong_pixel(const PMArgs &a, int px, int py) {
  const int W = a.W, H = a.H, center = px + py * W;
  short2 res = make_short2(-1, -1);
  if (a.weak[center] == DPE_WEAK) {
    for (int r = 1; r <= 100; ++r) {
      bool found = false;
      for (int x = -r; x <= r && !found; ++x) {
        const int nx = px + x;
        const bool edge_col = (x == -r || x == r);
        // inner loop over y: full column on the ring's left/right edges, else only y = -r and y = r
        for (int y = -r; y <= r; y += edge_col ? 1 : 2 * r) {
          const int ny = py + y;
          if (nx < 0 || ny < 0 || nx >= W || ny >= H) continue;
          if (a.weak[nx + ny * W] == DPE_STRONG) { res = make_short2(nx, ny); found = true; break; }
        }
      }
      if (found) break;
    }
  }
  a.nearest[center] = res;
}
// Resident blocks requested for the one-thread-per-pixel searches (nearest strong point,
// GenNeighbours, the plane fit): measured on the 10-view 1600x1200 schedule with fixed 16x8
// blocks, 6 blocks (80 registers) make GenNeighbours 9 % faster than its unbounded 104 registers
// (4 blocks) and 4 % faster than 8 blocks (64 registers, more stack traffic).
#ifndef DPE_LATENCY_MIN_BLOCKS
#define DPE_LATENCY_MIN_BLOCKS 6
#endif
// One thread per pixel of a 2D grid: the tiles keep the rays of neighbouring pixels together
// (measured faster than a work list over the WEAK pixels).
__global__ void __launch_bounds__(128, DPE_LATENCY_MIN_BLOCKS) k_find_nearest_strong(const Launch lc) {
  const Blk B = resolve<kGridFull>(lc);
  const PMArgs &a = *B.a;
  int px, py;
  if (!full_pixel(a, B, &px, &py)) return;
  find_nearest_strong_pixel(a, px, py);
}

// ------------------------------------------------------------------ geometry helpers for GenNeighbours
__device__ __forceinline__ uint8_t edge_at(const PMArgs &a, long idx) {
  return (idx >= 0 && idx < (long)a.W * a.H) ? a.edge[idx] : (uint8_t)0;
}
__device__ __forceinline__ uint8_t edge_low_at(const PMArgs &a, long idx) {
  return (idx >= 0 && idx < (long)a.lowW * a.lowH) ? a.edge_low[idx] : (uint8_t)0;
}

// BresenhamLine (DPE.cu:162-248); out-of-image linear indices read 0.
__device__ bool bresenham(const PMArgs &a, int ax, int ay, int bx, int by) {
  if (edge_at(a, (long)ax + (long)ay * a.W) || edge_at(a, (long)bx + (long)by * a.W)) return false;
  const float scale_x = 1.0f * a.lowW / (float)a.W;
  const float scale_y = 1.0f * a.lowH / (float)a.H;
  const int h = a.lowH, w = a.lowW;
  const int max_step = a.P.high_res_img ? (int)round(cvmax(h, w) / 60.0) : cvmax(h, w);
  for (int pass = 0; pass < 2; ++pass) {
    const int fx = pass == 0 ? bx : ax, fy = pass == 0 ? by : ay;
    const int tx = pass == 0 ? ax : bx, ty = pass == 0 ? ay : by;
    int x0 = (int)cvmin(roundf(fx * scale_x), (float)(w - 1));
    int y0 = (int)cvmin(roundf(fy * scale_y), (float)(h - 1));
    const int x1 = (int)cvmin(roundf(tx * scale_x), (float)(w - 1));
    const int y1 = (int)cvmin(roundf(ty * scale_y), (float)(h - 1));
    const int dx = abs(x1 - x0), sx = x0 < x1 ? 1 : -1;
    const int dy = abs(y1 - y0), sy = y0 < y1 ? 1 : -1;
    int err = (dx > dy ? dx : dy) / 2;
    int step = 0;
    bool tagx = true, tagy = true;
    while (tagx || tagy) {
      if (x0 == x1) tagx = false;
      if (y0 == y1) tagy = false;
      const int e2 = err;
      if (e2 > -dx) { err -= dy; x0 += sx; }
      if (e2 < dy) { err += dx; y0 += sy; }
      if (edge_low_at(a, (long)x0 + (long)y0 * w)) return true;
      step += 1;
      if (step >= max_step) break;
    }
  }
  return false;
}

// PointinTriangle (DPE.cu:139-160)
__device__ __forceinline__ bool point_in_triangle(short2 A, short2 B, short2 C, int px, int py) {
  const float2 AB = make_float2(B.x - A.x, B.y - A.y), BC = make_float2(C.x - B.x, C.y - B.y), CA = make_float2(A.x - C.x, A.y - C.y);
  const float ab = sqrtf(AB.x * AB.x + AB.y * AB.y), bc = sqrtf(BC.x * BC.x + BC.y * BC.y), ca = sqrtf(CA.x * CA.x + CA.y * CA.y);
  if (ab <= 2 || bc <= 2 || ca <= 2) return false;
  if (!(ab + bc > ca && bc + ca > ab && ab + ca > bc)) return false;
  const float2 PA = make_float2(A.x - px, A.y - py), PB = make_float2(B.x - px, B.y - py), PC = make_float2(C.x - px, C.y - py);
  const float t1 = PA.x * PB.y - PA.y * PB.x, t2 = PB.x * PC.y - PB.y * PC.x, t3 = PC.x * PA.y - PC.y * PA.x;
  return t1 * t2 >= 0 && t1 * t3 >= 0;
}

__device__ __forceinline__ void sort_small(float *d, int n) {
  for (int i = 1; i < n; ++i) {
    const float t = d[i];
    int j;
    for (j = i; j >= 1 && t < d[j - 1]; j--) d[j] = d[j - 1];
    d[j] = t;
  }
}

// ------------------------------------------------------------------ GenNeighbours (DPE.cu:2107-2467)
__device__ __forceinline__ void gen_neighbours_pixel(const PMArgs &a, int px, int py) {
  const int W = a.W, H = a.H, center = px + py * W;
  if (a.weak[center] != DPE_WEAK) return;
  constexpr int kMaxPts = 64;
  const int margin = 6;
  const float depth_diff = a.P.depth_max - a.P.depth_min;
  const dpe_camera &cam = a.cam[0];
  Rng rng = make_rng(a, center);
  short2 *nbs = &a.neigh[(size_t)a.nmap[center] * kNeighbours];
  nbs[0] = make_short2(px, py);
  for (int i = 1; i < kNeighbours; ++i) nbs[i] = make_short2(-1, -1);
  short2 pts[kMaxPts];
  uint64_t valid = 0;
  int odi = -1, npts = 0;
  const int rt = a.P.rotate_time;
  const float angle = 45.0f / rt;
  const float cos_a = (float)cos(angle * 3.14159265358979323846 / 180.f);
  const float sin_a = (float)sin(angle * 3.14159265358979323846 / 180.f);
  const float thr = (float)cos((angle / 2.0f) * 3.14159265358979323846 / 180.0f);
  const int shift_range = cvmax((int)(tan((angle / 2.0f) * 3.14159265358979323846 / 180.0f) * 20), 1);
  const float ransac_thr = a.P.ransac_threshold * depth_diff;
  bool edge_limit = false;
  if (a.P.use_limit) {
    edge_limit = true;
    if (a.P.use_edge) {
      const float cv = a.complexity[center];
      const float rp = rng.uniform() - FLT_EPSILON;
      if (rp < cv) edge_limit = false;
      else a.complexity[center] = cvmax(0.99f, cv);
    }
  }
  for (int odx = -1; odx <= 1; ++odx)
    for (int ody = -1; ody <= 1; ++ody) {
      if (odx == 0 && ody == 0) continue;
      float2 od = make_float2((float)odx, (float)ody);
      normalize2(&od);
      odi++;
      for (int ri = 0; ri < rt; ++ri) {
        const int di = odi * 4 + ri;
        for (int radius = 2; radius <= 4096; radius = cvmin(radius * 2, radius + 25)) {
          const float2 tp = make_float2(px + od.x * radius, py + od.y * radius);
          if (tp.x < 0 || tp.y < 0 || tp.x >= W || tp.y >= H) break;
          for (int k = 0; k < 4; ++k) {
            uint32_t sgn = (rng.u32() % 2 == 0) ? 1u : 0xFFFFFFFFu;
            const int rxs = (int)((sgn * rng.u32()) % (uint32_t)shift_range);
            sgn = (rng.u32() % 2 == 0) ? 1u : 0xFFFFFFFFu;
            const int rys = (int)((sgn * rng.u32()) % (uint32_t)shift_range);
            float2 dir = make_float2(od.x * 20 + rxs, od.y * 20 + rys);
            normalize2(&dir);
            short2 nb = make_short2((short)(int)(px + dir.x * radius), (short)(int)(py + dir.y * radius));
            if (nb.x < margin || nb.y < margin || nb.x >= W - margin || nb.y >= H - margin) continue;
            int nbc = nb.x + nb.y * W;
            if (a.weak[nbc] != DPE_STRONG) {
              nb = a.nearest[nbc];
              if (nb.x == -1 || nb.y == -1) continue;
              nbc = nb.x + nb.y * W;
            }
            float2 td = make_float2((float)(nb.x - px), (float)(nb.y - py));
            normalize2(&td);
            const float ca = td.x * od.x + td.y * od.y;
            if (ca > thr && (!edge_limit || !bresenham(a, px, py, nb.x, nb.y))) {
              pts[di] = nb; valid |= 1ull << di; npts++;
              break;
            }
          }
          if ((valid >> di) & 1ull) break;
        }
        float2 rd = make_float2(od.x * cos_a - od.y * sin_a, od.x * sin_a + od.y * cos_a);
        normalize2(&rd);
        od = rd;
      }
    }
  int ext = 31;
  if (a.P.use_label && a.label[center] > 0) {
    const short2 *lb = &a.lab_bound[(size_t)a.nmap[center] * 8];
    float bd[8];
    int ds[8];
    for (int i = 0; i < 8; ++i) {
      const short2 b = lb[i];
      float dist = 0.0f;
      if (b.x != -1 && b.y != -1) {
        const double ddx = (double)(px - b.x), ddy = (double)(py - b.y);
        dist = (float)sqrt(ddx * ddx + ddy * ddy);
        if (i >= 4) dist = (float)(dist / sqrt(2.0));
      }
      bd[i] = dist;
      if (i % 2 == 1) {
        const float od2 = bd[i - 1];
        const int step = cvmin(1, cvmax(2 * rt - 1, (int)(2 * rt * dist / (dist + od2))));  // quirk Q5
        ds[i - 1] = 2 * rt - step;
        ds[i] = step;
      }
    }
    for (int i = 0; i < 8; ++i) {
      const float dist = bd[i];
      const int gap = ds[i] + 1;
      const int step_len = cvmax(1, (int)floor(1.0 * dist / gap));
      for (int s = 1; s <= ds[i]; ++s) {
        short2 nb = make_short2((short)(px + s * step_len * kDir[i][0]), (short)(py + s * step_len * kDir[i][1]));
        if (nb.x < margin || nb.y < margin || nb.x >= W - margin || nb.y >= H - margin) continue;
        int nbc = nb.x + nb.y * W;
        if (a.weak[nbc] != DPE_STRONG) {
          nb = a.nearest[nbc];
          if (nb.x == -1 || nb.y == -1) continue;
          nbc = nb.x + nb.y * W;
        }
        if (a.label[nbc] != 0 && a.label[nbc] != a.label[center]) continue;
        ext++;
        pts[ext] = nb; valid |= 1ull << ext; npts++;
      }
    }
  }
  if (npts <= 3) { a.reliable[center] = 0; a.rng_ctr[center] = rng.ctr; return; }

  short2 sv[kMaxPts];
  float3 sv3[kMaxPts], svn[kMaxPts];
  int vc = 0;
  float X[3];
  point3d(cam, px, py, a.plane[center].w, X);
  const float cwz = X[2];
  for (int i = 0; i < kMaxPts; ++i) {
    if ((valid >> i) & 1ull) {
      const short2 sp = pts[i];
      const int spc = sp.x + sp.y * W;
      const float4 spl = a.plane[spc];
      sv[vc] = sp;
      point3d(cam, sp.x, sp.y, spl.w, X);
      sv3[vc] = make_float3(X[0], X[1], X[2]);
      const float4 n4 = normal_to_ref(cam, spl);
      svn[vc] = make_float3(n4.x, n4.y, n4.z);
      vc++;
    }
  }
  float4 best = make_float4(0, 0, 0, 0);
  bool has_valid = false;
  {
    int iteration = 50, max_iter = a.P.high_res_img ? 200 : 125, max_count = 3;
    float min_cost = FLT_MAX;
    float residuals[kMaxPts];
    for (int i = 0; i < kMaxPts; ++i) residuals[i] = 0.0f;
    float tthr = ransac_thr;
    bool has_consist = false;
    bool must_tri = (a.P.use_label && a.label[center] > 0 && edge_limit) ? false : true;
    while (iteration > 0 && max_iter > 0) {
      max_iter--;
      const int ia = (int)(rng.u32() % (uint32_t)vc);
      const int ib = (int)(rng.u32() % (uint32_t)vc);
      const int ic = (int)(rng.u32() % (uint32_t)vc);
      if (ia == ib || ib == ic || ia == ic) continue;
      if (must_tri && !point_in_triangle(sv[ia], sv[ib], sv[ic], px, py)) continue;
      if (edge_limit) {
        if (bresenham(a, sv[ia].x, sv[ia].y, sv[ib].x, sv[ib].y) || bresenham(a, sv[ib].x, sv[ib].y, sv[ic].x, sv[ic].y) ||
            bresenham(a, sv[ic].x, sv[ic].y, sv[ia].x, sv[ia].y))
          continue;
      }
      bool nc = false;
      if (a.P.geom_consistency && edge_limit) {
        const float3 AN = svn[ia], BN = svn[ib], CN = svn[ic];
        nc = true;
        if ((double)(AN.x * BN.x + AN.y * BN.y + AN.z * BN.z) < 0.8660254 ||
            (double)(AN.x * CN.x + AN.y * CN.y + AN.z * CN.z) < 0.8660254 ||
            (double)(BN.x * CN.x + BN.y * CN.y + BN.z * CN.z) < 0.8660254)
          nc = false;
        if (has_consist && !nc) continue;
      }
      iteration--;
      const float3 A = sv3[ia], B = sv3[ib], C = sv3[ic];
      const float3 AC = make_float3(A.x - C.x, A.y - C.y, A.z - C.z), BC = make_float3(B.x - C.x, B.y - C.y, B.z - C.z);
      float4 cr;
      cr.x = AC.y * BC.z - BC.y * AC.z;
      cr.y = -(AC.x * BC.z - BC.x * AC.z);
      cr.z = AC.x * BC.y - BC.x * AC.y;
      if ((cr.x == 0 && cr.y == 0 && cr.z == 0) || isnan(cr.x) || isnan(cr.y) || isnan(cr.z)) continue;
      normalize3(&cr);
      cr.w = -(cr.x * A.x + cr.y * A.y + cr.z * A.z);
      int tcount = 0;
      float sdist = 0.0f;
      for (int s = 0; s < vc; ++s) {
        const float fx = (sv[s].x - cam.K[2]) / cam.K[0];
        const float fy = (sv[s].y - cam.K[5]) / cam.K[4];
        const float fd = -cr.w / (cr.x * fx + cr.y * fy + cr.z);
        const float dist = fabsf(fd - sv3[s].z);
        residuals[s] = dist;
        if (dist < tthr) { tcount++; sdist += dist; }
      }
      if (tcount < 6) continue;
      const float fx = (px - cam.K[2]) / cam.K[0], fy = (py - cam.K[5]) / cam.K[4];
      if (tcount > max_count) {
        if (!must_tri && point_in_triangle(sv[ia], sv[ib], sv[ic], px, py)) must_tri = true;
        if (!has_consist && nc) has_consist = true;
        const float fd = -cr.w / (cr.x * fx + cr.y * fy + cr.z);
        const float cd = fabsf(fd - cwz);
        best = cr; max_count = tcount; sdist /= tcount; min_cost = cd; has_valid = true;
        if (tthr > (a.P.high_res_img ? 0.05 : 0.005)) {
          sort_small(residuals, vc);
          if (tthr < residuals[kNeighbours]) continue;
          tthr = (float)(residuals[kNeighbours] - 1e-6);
          tcount = 0;
          for (int s = 0; s < vc; ++s) {
            if (residuals[s] < tthr) tcount++;
            else break;
          }
          max_count = tcount;
        }
      } else if (tcount == max_count) {
        if (!must_tri && point_in_triangle(sv[ia], sv[ib], sv[ic], px, py)) must_tri = true;
        const float fd = -cr.w / (cr.x * fx + cr.y * fy + cr.z);
        const float cd = fabsf(fd - cwz);
        if (cd < min_cost) { best = cr; max_count = tcount; sdist /= tcount; min_cost = cd; }
      }
    }
  }
  a.rng_ctr[center] = rng.ctr;
  if (!has_valid) { a.reliable[center] = 0; return; }
  float weight[kMaxPts];
  for (int i = 0; i < vc; ++i) {
    const float fx = (sv[i].x - cam.K[2]) / cam.K[0];
    const float fy = (sv[i].y - cam.K[5]) / cam.K[4];
    const float fd = -best.w / (best.x * fx + best.y * fy + best.z);
    const float dist = fabsf(fd - sv3[i].z);
    if (dist >= ransac_thr) { sv[i] = make_short2(-1, -1); weight[i] = FLT_MAX; continue; }
    weight[i] = dist;
  }
  for (int i = 1; i < vc; ++i) {
    const short2 tp = sv[i];
    const float tw = weight[i];
    int j;
    for (j = i; j >= 1 && tw < weight[j - 1]; j--) { sv[j] = sv[j - 1]; weight[j] = weight[j - 1]; }
    sv[j] = tp; weight[j] = tw;
  }
  for (int i = 1; i < kNeighbours; ++i) nbs[i] = (i - 1 < vc) ? sv[i - 1] : make_short2(-1, -1);
  a.reliable[center] = 1;
}
// One thread per pixel of a 2D grid: the tiles keep the rays of neighbouring pixels together
// (measured faster than a work list over the WEAK pixels).
__global__ void __launch_bounds__(128, DPE_LATENCY_MIN_BLOCKS) k_gen_neighbours(const Launch lc) {
  const Blk B = resolve<kGridFull>(lc);
  const PMArgs &a = *B.a;
  int px, py;
  if (!full_pixel(a, B, &px, &py)) return;
  gen_neighbours_pixel(a, px, py);
}

__global__ void k_neighbour_update(const Launch lc) {
  const Blk B = resolve<kGridFull>(lc);
  const PMArgs &a = *B.a;
  int px, py;
  if (!full_pixel(a, B, &px, &py)) return;
  const int c = px + py * a.W;
  if (a.weak[c] == DPE_WEAK && a.reliable[c] != 1) a.weak[c] = DPE_UNKNOWN;
}

// ------------------------------------------------------------------ RandomInitialization (DPE.cu:1039-1067, 784-861)
template <int kStage>
__global__ void __launch_bounds__(128, DPE_COST_MIN_BLOCKS) k_random_init(const Launch lc) {
  const Blk B = resolve<kGridFull>(lc);
  const PMArgs &a = *B.a;
  int px, py;
  if (!full_pixel(a, B, &px, &py)) return;
  const int center = px + py * a.W;
  const dpe_camera &rc = a.cam[0];
  DPE_REF_WINDOW(rw);
  build_ref_window(a, px, py, rw, KID_RANDOM_INIT);
  const int n = a.N - 1;
  if (a.P.state == DPE_FIRST_INIT) {
    Rng rng = make_rng(a, center);
    const float depth = rng.uniform() * (a.P.depth_max - a.P.depth_min) + a.P.depth_min;
    float4 pl = random_normal(rc, px, py, rng, depth);
    pl.w = dist_to_origin(rc, px, py, depth, pl);
    a.rng_ctr[center] = rng.ctr;
    a.plane[center] = pl;
    float cv[kMaxSrc], srt[kMaxSrc];
    int valid = 0;
    ncc_all_sources<kStage, kSweepUnroll>(a, px, py, pl, rw, cv);
    for (int i = 0; i < n; ++i) {
      const float v = cv[i];
      srt[i] = v;
      if (v < 2.0f) valid++;
    }
    sort_small(srt, n);
    uint32_t views = 0;
    float cost = 2.0f;
    const int k = min(valid, a.P.top_k);
    if (k > 0) {
      float c = 0.0f;
      for (int i = 0; i < k; ++i) c += srt[i];
      const float thr = srt[k - 1];
      for (int i = 0; i < n; ++i)
        if (cv[i] <= thr) setBit(&views, i);
      cost = c / k;
    }
    a.views[center] = views;
    a.cost[center] = cost;
  } else {
    float4 pl = normal_to_ref(rc, a.plane[center]);
    const float depth = pl.w;
    pl.w = dist_to_origin(rc, px, py, depth, pl);
    a.plane[center] = pl;
    uint32_t views = a.views[center];
    int cnt = 0;
    float cost = 0.0f;
    for (int i = 1; i < a.N; ++i) {
      if (isSet(views, i - 1)) {
        const float v = ncc_strong<kStage, kSweepUnroll>(a, px, py, i, pl, rw);
        if (v < 2.0f) { cnt++; cost += v; }
        else unSetBit(&views, i - 1);
      }
    }
    a.views[center] = views;
    a.cost[center] = cnt == 0 ? 2.0f : cost / cnt;
  }
}

// ------------------------------------------------------------------ shared pieces of the propagation kernels
// Multi-hypothesis joint view selection (DPE.cu:1551-1619 / 1714-1783).
// cost_array: 8 candidate rows of per-source costs, `stride` floats apart.
__device__ __forceinline__ float sample_views(const PMArgs &a, Rng &rng, int iter, const float *cost_array, int stride,
                                              const float *priors, uint8_t *vw, uint32_t *temp_sel, float *probs) {
  const int n = a.N - 1;
  for (int i = 0; i < 32; ++i) vw[i] = 0;
  const float thr = (float)(0.8 * (double)dpe_expf((float)(iter * iter) / (-90.0f)));
  const float base = dpe_expf(thr * thr / (-0.32f));
  for (int i = 0; i < n; ++i) {
    float count = 0;
    int count_false = 0;
    float tmpw = 0;
    for (int j = 0; j < 8; ++j) {
      const float v = cost_array[j * stride + i];
      if (v < thr) { tmpw += dpe_expf(v * v / (-0.18f)); count++; }
      if (v > 1.2f) count_false++;
    }
    float p = 0.0f;
    if (count > 2 && count_false < 3) p = tmpw / count;
    else if (count_false < 3) p = base;
    probs[i] = p * priors[i];
  }
  float sum = 0.0f;
  for (int i = 0; i < n; ++i) sum += probs[i];
  const float inv = 1.0f / sum;
  float cum = 0.0f;
  for (int i = 0; i < n; ++i) { cum += probs[i] * inv; probs[i] = cum; }
  for (int s = 0; s < 15; ++s) {
    const float r = rng.uniform() - FLT_EPSILON;
    for (int id = 0; id < n; ++id)
      if (probs[id] > r) { vw[id] += 1; break; }
  }
  uint32_t sel = 0;
  float wn = 0;
  for (int i = 0; i < n; ++i)
    if (vw[i] > 0) { setBit(&sel, i); wn += vw[i]; }
  *temp_sel = sel;
  return wn;
}

__device__ __forceinline__ int find_min_cost_index(const float *c, int n) {
  float m = c[0];
  int idx = 0;
  for (int i = 1; i < n; ++i)
    if (c[i] <= m) { m = c[i]; idx = i; }
  return idx;
}

// ------------------------------------------------------------------ Gauss-Newton plane hypothesis
// The differentiation form's refinement step (no reference counterpart; dpe_options::gn_refine).
// Around the current plane (n, depth) it takes the cost of each sampled source j and its gradient
// (ncc_strong_adjoint) in the local parameters theta = (d depth, d a1, d a2), the normal tilted
// within its tangent plane (n' = normalize(n + a1 e1 + a2 e2)), and solves the damped normal
// equations  (J^T V J + lambda diag(J^T V J)) theta = -J^T V c  (V = the view weights).  The
// resulting plane is a hypothesis like the random ones: kept only when its cost is lower and its
// depth lies in range.  It draws no random numbers, so the rest of the update is unchanged.
struct GnFrame {
  float ray0, ray1, nr, d0;  // the pixel's ray (z = 1), n . ray, the current depth
  float e1x, e1y, e1z, e2x, e2y, e2z, e1r, e2r;  // tangent basis of n, e . ray
};
__device__ __forceinline__ GnFrame gn_frame(const dpe_camera &rc, int px, int py, float4 p, float d0) {
  GnFrame f;
  f.ray0 = ((float)px - rc.K[2]) / rc.K[0];
  f.ray1 = ((float)py - rc.K[5]) / rc.K[4];
  f.nr = p.x * f.ray0 + p.y * f.ray1 + p.z;
  f.d0 = d0;
  if (fabsf(p.x) < 0.9f) { f.e1x = 0.0f; f.e1y = p.z; f.e1z = -p.y; }  // n x (1, 0, 0)
  else { f.e1x = -p.z; f.e1y = 0.0f; f.e1z = p.x; }                    // n x (0, 1, 0)
  const float e1n = 1.0f / sqrtf(f.e1x * f.e1x + f.e1y * f.e1y + f.e1z * f.e1z);
  f.e1x *= e1n; f.e1y *= e1n; f.e1z *= e1n;
  f.e2x = p.y * f.e1z - p.z * f.e1y; f.e2y = p.z * f.e1x - p.x * f.e1z; f.e2z = p.x * f.e1y - p.y * f.e1x;
  f.e1r = f.e1x * f.ray0 + f.e1y * f.ray1 + f.e1z;
  f.e2r = f.e2x * f.ray0 + f.e2y * f.ray1 + f.e2z;
  return f;
}
// Adds source j's terms (view weight v) to the normal equations m = (A00 A01 A02 A11 A12 A22 b0 b1 b2).
template <class RW>
__device__ __forceinline__ void gn_accumulate(const PMArgs &a, int px, int py, const RW &rw, float4 p,
                                              const GnFrame &f, int j, float v, float m[9]) {
  float g[4];
  const float c = ncc_strong_adjoint(a, px, py, j + 1, p, rw, g, nullptr);
  if (!(c > 0.0f && c < 2.0f)) return;
  // w = -depth (n . ray): dC/ddepth = g_w (-(n . ray)); tilting n moves w by -depth (e . ray)
  const float jd = -g[3] * f.nr;
  const float j1 = g[0] * f.e1x + g[1] * f.e1y + g[2] * f.e1z - g[3] * f.d0 * f.e1r;
  const float j2 = g[0] * f.e2x + g[1] * f.e2y + g[2] * f.e2z - g[3] * f.d0 * f.e2r;
  m[0] += v * jd * jd; m[1] += v * jd * j1; m[2] += v * jd * j2;
  m[3] += v * j1 * j1; m[4] += v * j1 * j2; m[5] += v * j2 * j2;
  m[6] -= v * jd * c; m[7] -= v * j1 * c; m[8] -= v * j2 * c;
}
// Solves the damped normal equations m around plane p; false when singular, when the new plane
// does not face the camera, or when its depth is out of range.  *t receives the new plane.
__device__ __forceinline__ bool gn_solve(const PMArgs &a, int px, int py, float4 p, const GnFrame &f,
                                         const float m[9], float4 *t) {
  const float lambda = 0.1f;
  const float A00 = m[0] * (1.0f + lambda), A01 = m[1], A02 = m[2];
  const float A11 = m[3] * (1.0f + lambda), A12 = m[4], A22 = m[5] * (1.0f + lambda);
  const float b0 = m[6], b1 = m[7], b2 = m[8];
  const float c00 = A11 * A22 - A12 * A12, c01 = A02 * A12 - A01 * A22, c02 = A01 * A12 - A02 * A11;
  const float det = A00 * c00 + A01 * c01 + A02 * c02;
  if (!(fabsf(det) > 1e-30f) || !isfinite(det)) return false;
  const float c11 = A00 * A22 - A02 * A02, c12 = A01 * A02 - A00 * A12, c22 = A00 * A11 - A01 * A01;
  const float inv = 1.0f / det;
  const float td = (c00 * b0 + c01 * b1 + c02 * b2) * inv;
  const float t1 = (c01 * b0 + c11 * b1 + c12 * b2) * inv;
  const float t2 = (c02 * b0 + c12 * b1 + c22 * b2) * inv;
  float nx = p.x + t1 * f.e1x + t2 * f.e2x, ny = p.y + t1 * f.e1y + t2 * f.e2y, nz = p.z + t1 * f.e1z + t2 * f.e2z;
  const float nn = 1.0f / sqrtf(nx * nx + ny * ny + nz * nz);
  nx *= nn; ny *= nn; nz *= nn;
  if (!(nx * f.ray0 + ny * f.ray1 + nz < 0.0f)) return false;  // the plane must face the camera
  const float dn = f.d0 + td;
  if (!(dn >= a.P.depth_min && dn <= a.P.depth_max)) return false;
  *t = make_float4(nx, ny, nz, 0.0f);
  t->w = dist_to_origin(a.cam[0], px, py, dn, *t);
  return true;
}

// ------------------------------------------------------------------ strong update (DPE.cu:1218-1670, 1069-1122)
// Block-cooperative: a block holds kCoopPix pixels of one colour (consecutive x on one row of the
// half grid) and kCoopLanes threads per pixel.  The pixel's reference window and its candidate
// cost matrix live once in shared memory; the threads of a pixel evaluate its hypotheses side by
// side (lane d: candidate d; then the sampled sources of the current plane and of the five
// refinement planes), and one thread per pixel takes every decision in the reference's order, so
// the random draws and the order of each weighted sum are those of one thread doing it all.
//
// Phases, separated by block barriers:
//   0  window taps (lanes split the taps)
//   1  window sums (lane 0); candidate search (lane d: direction d)
//   2  candidate costs (lane d: candidate d)
//   3  view-selection probabilities per source and the 15 uniform draws (lanes split them)
//   4  view sampling from the draws, in order (lane 0)
//   5  candidates' weighted costs (lane d) and the current plane's costs (lanes split sources)
//   6  best candidate, acceptance, refinement planes (lane 0)
//   7  refinement costs (lanes split plane x source)
//   8  refinement decisions, outputs (lane 0)
//   9-11  with the Gauss-Newton hypothesis only: its normal equations (lanes split the sources,
//         shuffle sums), its costs (lanes split the sources), its decision and the outputs (lane 0)
constexpr int kCoopPix = 16, kCoopLanes = 8, kCoopThreads = kCoopPix * kCoopLanes;

// The strong NCC as the cooperative strong update calls it, inlined at each call site (measured:
// one shared out-of-line copy, which would ease the instruction cache, is 10 % slower).
template <int kStage>
__device__ __forceinline__ float coop_ncc(const PMArgs &a, int px, int py, int s, float4 pl, const SmemWindow &rw) {
  return ncc_strong<kStage, kStrongUnroll>(a, px, py, s, pl, rw);
}
template <int kStage>
__device__ __forceinline__ void coop_ncc_all(const PMArgs &a, int px, int py, float4 pl, const SmemWindow &rw, float *out) {
  for (int j = 0; j < a.N - 1; ++j) out[j] = coop_ncc<kStage>(a, px, py, j + 1, pl, rw);
}

// Decision state of one pixel, in shared memory.
struct CoopPixel {
  float2 win[kWinTaps];  // (w, w * (r - c)) per tap
  union {
    float rc[kWinTaps];     // phases 0-1: r - c per tap
    float probs[kMaxSrc];   // phases 3-4: view-selection probability per source
  };
  union {
    float4 hyp[5];          // phases 6-8: the refinement planes
    float u[16];            // phases 3-4: the 15 uniform draws of the view sampling
    float fc[8];            // phases 5-6: the candidates' weighted costs
  };
  float4 pl_cur, pl_now;
  float center, inv_wsum, mean_r, var_r;
  float wn, cost_now, cost_written, depth_now;
  int pos[8];
  uint8_t act[32];  // the sampled sources (source index - 1), ascending
  int na;
  uint32_t views_new, temp_sel, rng_ctr;
  uint8_t flag[8];
  uint8_t vw[32];
};
// Shared bytes of one block: the pixels' states, then per pixel 8 candidate cost rows and 6
// hypothesis cost rows of n = N - 1 floats.
__host__ __device__ inline size_t coop_smem_bytes(int n) {
  return sizeof(CoopPixel) * kCoopPix + sizeof(float) * (size_t)kCoopPix * 14 * n;
}

struct CoopCtx {
  const PMArgs *a;
  int slot, lane, px, py, center, n;
  bool live;  // a pixel of this colour inside the image, not WEAK
  CoopPixel *P;
  float *cost;  // 8 rows of n
  float *hc;    // 6 rows of n: the current plane, then the five refinement planes
  __device__ __forceinline__ SmemWindow window() const {
    return SmemWindow{P->win, P->center, P->inv_wsum, P->mean_r, P->var_r,
                      a->counters ? a->counters + 2 * KID_STRONG_UPDATE : nullptr};
  }
};

__device__ __forceinline__ CoopCtx coop_ctx(const Launch &lc, int parity, void *smem) {
  const Blk B = resolve<kGridFull>(lc);  // kGridFull's block-row width, (W + 15) / 16, is ours too
  const PMArgs &a = *B.a;
  CoopCtx c;
  c.a = B.a;
  c.slot = (int)threadIdx.x / kCoopLanes;
  c.lane = (int)threadIdx.x % kCoopLanes;
  c.n = a.N - 1;
  c.px = B.x * kCoopPix + c.slot;
  c.py = 2 * B.y + ((c.px + parity) & 1);
  c.center = c.py * a.W + c.px;
  c.live = c.px < a.W && c.py < a.H;
  if (c.live) c.live = G(a.weak, c.center, (long long)a.W * a.H, 201) != DPE_WEAK;
  CoopPixel *base = static_cast<CoopPixel *>(smem);
  c.P = base + c.slot;
  float *rows = reinterpret_cast<float *>(base + kCoopPix);
  c.cost = rows + (size_t)c.slot * 8 * c.n;
  c.hc = rows + (size_t)kCoopPix * 8 * c.n + (size_t)c.slot * 6 * c.n;
  return c;
}

// Phase 0: the window taps of build_ref_window, split over the lanes.
__device__ __forceinline__ void strong_p0(const CoopCtx &c) {
  if (!c.live) return;
  const PMArgs &a = *c.a;
  const int r = a.P.strong_radius, inc = a.P.strong_increment, side = 2 * r / inc + 1;
  const float center = texel(a, 0, c.px, c.py);
  for (int k = c.lane; k < side * side; k += kCoopLanes) {
    const int i = -r + (k / side) * inc, j = -r + (k % side) * inc;
    const float rp = texel(a, 0, c.px + i, c.py + j);
    const float w = bilateral_weight((float)i, (float)j, rp, center, a.P.sigma_spatial, a.P.sigma_color);
    const float rc = rp - center;
    G(c.P->win, k, kWinTaps, 320) = make_float2(w, w * rc);
    c.P->rc[k] = rc;
  }
  if (c.lane == 0) c.P->center = center;
}

// Candidate search of the non-edge propagation (8 slots: 0 up_near, 1 up_far, 2 down_near,
// 3 down_far, 4 left_near, 5 left_far, 6 right_near, 7 right_far), slot d only.
__device__ __forceinline__ int strong_search_plain(const PMArgs &a, int px, int py, int center, int d) {
  const int W = a.W, H = a.H;
  [[maybe_unused]] const long long L = (long long)W * H;
  const int f = d >> 1;
  if (d & 1) {  // far: every second pixel from distance 3 on
    const int starts[4] = {center - 3 * W, center + 3 * W, center - 3, center + 3};
    const int strides[4] = {-W, W, -1, 1};
    const bool oks[4] = {py > 2, py < H - 3, px > 2, px < W - 3};
    if (!oks[f]) return -1;
    float m = G(a.cost, starts[f], L, 206);
    int mp = starts[f];
    for (int i = 1; i < 11; ++i) {
      bool ok;
      switch (f) {
        case 0: ok = py > 2 + 2 * i; break;
        case 1: ok = py < H - 3 - 2 * i; break;
        case 2: ok = px > 2 + 2 * i; break;
        default: ok = px < W - 3 - 2 * i; break;
      }
      if (ok) {
        const int t = starts[f] + 2 * i * strides[f];
        const float ct = G(a.cost, t, L, 207);
        if (ct < m) { m = ct; mp = t; }
      }
    }
    return mp;
  }
  // near: base pixel one step away, then diagonal pairs at distance 1..3
  const int nbase[4] = {center - W, center + W, center - 1, center + 1};
  const bool nok[4] = {py > 0, py < H - 1, px > 0, px < W - 1};
  if (!nok[f]) return -1;
  float m = G(a.cost, nbase[f], L, 208);
  int mp = nbase[f];
  for (int i = 0; i < 3; ++i)
    for (int side = 0; side < 2; ++side) {
      bool ok;
      int t;
      const int k = 1 + i;
      switch (f) {
        case 0: t = nbase[0] - k * W + (side ? k : -k); ok = py > 1 + i && (side ? px < W - 1 - i : px > i); break;
        case 1: t = nbase[1] + k * W + (side ? k : -k); ok = py < H - 2 - i && (side ? px < W - 1 - i : px > i); break;
        case 2: t = nbase[2] - k + (side ? k * W : -k * W); ok = px > 1 + i && (side ? py < H - 1 - i : py > i); break;
        default: t = nbase[3] + k + (side ? k * W : -k * W); ok = px < W - 2 - i && (side ? py < H - 1 - i : py > i); break;
      }
      if (ok) {
        const float ct = G(a.cost, t, L, 209);
        if (ct < m) { m = ct; mp = t; }
      }
    }
  return mp;
}

// The edge-aware propagation's first search for direction d: steps along d up to the stored edge
// distance (DPE.cu:1262-1301).  Returns the position or -1.
__device__ __forceinline__ int strong_search_edge(const PMArgs &a, int px, int py, int center, int d, int iter) {
  const int W = a.W, H = a.H;
  [[maybe_unused]] const long long L = (long long)W * H;
  const float *cand_cost = a.cost_snap;
  const short2 e = G(a.edge_neigh, (long long)center * 8 + d, L * 8, 202);
  const float max_edge_dist = cvmax(H, W) / 30.0f;
  const int min_step = 2;
  const bool on_edge = G(a.edge, center, L, 203) != 0;
  const int dx = kDir[d][0], dy = kDir[d][1];
  const int sx = cvmax(1, 5 - 2 * iter) * dx, sy = cvmax(1, 5 - 2 * iter) * dy;
  const double ex = (double)(e.x - px), ey = (double)(e.y - py);
  float dist = (float)sqrt(ex * ex + ey * ey);
  if (d >= 4) dist = (float)(dist / sqrt(2.0));
  if (on_edge) dist = 11 * min_step;
  else if (e.x == -1 || e.y == -1 || dist > max_edge_dist) {
    dist = max_edge_dist;
    if (d >= 4) dist = (float)(dist / sqrt(2.0));
  }
  const int step_num = cvmin(cvmax(11, (int)(1.0f * dist / min_step)), 22);
  int step_len = cvmax((int)(1.0f * dist / step_num), min_step);
  if (d < 4 && step_len % 2 == 1) step_len -= 1;
  float mc = FLT_MAX;
  int mp = -1;
  int fx = 0, fy = 0;
  if (d > 4) { if (d % 2) fx = dx; else fy = dy; }
  for (int s = 0; s < step_num; ++s) {
    const int tx = px + sx + s * step_len * dx + fx, ty = py + sy + s * step_len * dy + fy;
    if (!(tx >= 0 && ty >= 0 && tx < W && ty < H)) continue;
    const int tc = tx + ty * W;
    const float cc = G(cand_cost, tc, L, 204);
    if (mc > cc) { mp = tc; mc = cc; }
  }
  return mc < FLT_MAX ? mp : -1;
}

// Phase 1: window sums in tap order (lane 0), as build_ref_window accumulates them; every lane
// searches its candidate direction (the non-edge form; the edge form searches in phase 2).
__device__ __forceinline__ void strong_p1(const CoopCtx &c) {
  if (!c.live) return;
  const PMArgs &a = *c.a;
  if (c.lane == 0) {
    const int r = a.P.strong_radius, inc = a.P.strong_increment, side = 2 * r / inc + 1;
    float sw = 0.f, swr = 0.f, swrr = 0.f;
    for (int k = 0; k < side * side; ++k) {
      const float2 t = c.P->win[k];
      sw += t.x; swr += t.y; swrr += t.y * c.P->rc[k];
    }
    c.P->inv_wsum = 1.0f / sw;
    c.P->mean_r = swr * c.P->inv_wsum;
    c.P->var_r = swrr * c.P->inv_wsum - c.P->mean_r * c.P->mean_r;
  }
  if (!a.P.use_edge) c.P->pos[c.lane] = strong_search_plain(a, c.px, c.py, c.center, c.lane);
}

// Phase 2: candidate d's costs against every source (lane d), with the edge form's second search
// and its replacement rule (DPE.cu:1302-1366).
template <int kStage>
__device__ __forceinline__ void strong_p2(const CoopCtx &c, int iter) {
  if (!c.live) return;
  const PMArgs &a = *c.a;
  const int n = c.n, d = c.lane;
  [[maybe_unused]] const long long L = (long long)a.W * a.H;
  float *row = c.cost + d * n;
  for (int j = 0; j < n; ++j) row[j] = 0.0f;
  if (d == 0) row[0] = 2.0f;  // `= {2.0f}` initialises only the first element (quirk Q2)
  const SmemWindow rw = c.window();
  bool flag = false;
  int pos = -1;
  if (a.P.use_edge) {
    pos = strong_search_edge(a, c.px, c.py, c.center, d, iter);
    if (pos >= 0) {
      flag = true;
      coop_ncc_all<kStage>(a, c.px, c.py, G(a.plane_snap, pos, L, 205), rw, row);
    }
    if (G(a.edge, c.center, L, 203) == 0) {
      const float good_thr = 0.8f * dpe_expf((float)(iter * iter) / (-90.0f));
      const int dx = kDir[d][0], dy = kDir[d][1], min_step = 2;
      const int sx = cvmax(1, 5 - 2 * iter) * dx, sy = cvmax(1, 5 - 2 * iter) * dy;
      const bool had = flag;
      float mc = FLT_MAX;
      int mp = -1;
      int fx = 0, fy = 0;
      if (d > 4) { if (d % 2) fx = dx; else fy = dy; }
      for (int s = 0; s < 11; ++s) {
        const int tx = c.px + sx + s * min_step * dx + fx, ty = c.py + sy + s * min_step * dy + fy;
        if (!(tx >= 0 && ty >= 0 && tx < a.W && ty < a.H)) continue;
        const int tc = tx + ty * a.W;
        const float cc = G(a.cost_snap, tc, L, 204);
        if (mc > cc) { mp = tc; mc = cc; }
      }
      if (mc < FLT_MAX) {
        flag = true;
        float tca[kMaxSrc];
        coop_ncc_all<kStage>(a, c.px, c.py, G(a.plane_snap, mp, L, 205), rw, tca);
        int g0 = 0, g1 = 0, b0 = 0, b1 = 0;
        for (int j = 0; j < n; ++j) {
          if (row[j] < good_thr) g0++;
          if (row[j] > 1.2f) b0++;
          if (tca[j] < good_thr) g1++;
          if (tca[j] > 1.2f) b1++;
        }
        if (!had || g1 > g0 || (g1 == g0 && b1 < b0)) {
          pos = mp;
          for (int j = 0; j < n; ++j) row[j] = tca[j];
        }
      }
    }
  } else {
    pos = c.P->pos[d];
    if (pos >= 0) {
      flag = true;
      coop_ncc_all<kStage>(a, c.px, c.py, G(a.plane, pos, L, 210), rw, row);
    }
  }
  c.P->flag[d] = flag ? 1 : 0;
  c.P->pos[d] = pos;
}

// Phase 3: the view-selection probability of each source (sample_views' first loop, with the
// priors of DPE.cu:1551-1563), lane j taking sources j, j + 8, ...; and the 15 uniform draws of
// the sampling (counter-based, so draw s is the pixel's counter + s), split over the lanes.
__device__ __forceinline__ void strong_p3(const CoopCtx &c, int iter) {
  if (!c.live) return;
  const PMArgs &a = *c.a;
  const int W = a.W, n = c.n, center = c.center;
  const long long L = (long long)W * a.H;
  CoopPixel &P = *c.P;
  const uint32_t ctr0 = G(a.rng_ctr, center, L, 106);
  for (int s = c.lane; s < 15; s += kCoopLanes) {
    Rng r{a.key[0], a.key[1], (uint32_t)center, ctr0 + (uint32_t)s};
    P.u[s] = r.uniform();
  }
  const long total = (long)W * a.H;
  const long nbr[4] = {(long)center - W, (long)center + W, (long)center - 1, (long)center + 1};
  uint32_t sv[4];
  for (int i = 0; i < 4; ++i)
    sv[i] = (P.flag[2 * i] && nbr[i] >= 0 && nbr[i] < total) ? G(a.views, nbr[i], L, 211) : 0u;
  const float thr = (float)(0.8 * (double)dpe_expf((float)(iter * iter) / (-90.0f)));
  const float base = dpe_expf(thr * thr / (-0.32f));
  for (int j = c.lane; j < n; j += kCoopLanes) {
    float prior = 0.0f;
    for (int i = 0; i < 4; ++i)
      if (P.flag[2 * i]) prior += isSet(sv[i], j) == 1 ? 0.9f : 0.1f;
    float count = 0;
    int count_false = 0;
    float tmpw = 0;
    for (int d = 0; d < 8; ++d) {
      const float v = c.cost[d * n + j];
      if (v < thr) { tmpw += dpe_expf(v * v / (-0.18f)); count++; }
      if (v > 1.2f) count_false++;
    }
    float p = 0.0f;
    if (count > 2 && count_false < 3) p = tmpw / count;
    else if (count_false < 3) p = base;
    P.probs[j] = p * prior;
  }
  if (c.lane == 0) {
    P.rng_ctr = ctr0 + 15;
    P.pl_cur = G(a.plane, center, L, 212);
  }
}

// Phase 4 (lane 0): the rest of sample_views (normalised cumulative probabilities, the 15
// samples, the selection mask and weight sum) and the list of sampled sources.
__device__ __forceinline__ void strong_p4(const CoopCtx &c) {
  if (!c.live || c.lane != 0) return;
  const int n = c.n;
  CoopPixel &P = *c.P;
  for (int i = 0; i < 32; ++i) P.vw[i] = 0;
  float sum = 0.0f;
  for (int i = 0; i < n; ++i) sum += P.probs[i];
  const float inv = 1.0f / sum;
  float cum = 0.0f;
  for (int i = 0; i < n; ++i) { cum += P.probs[i] * inv; P.probs[i] = cum; }
  for (int s = 0; s < 15; ++s) {
    const float r = P.u[s] - FLT_EPSILON;
    for (int id = 0; id < n; ++id)
      if (P.probs[id] > r) { P.vw[id] += 1; break; }
  }
  uint32_t sel = 0;
  float wn = 0;
  int na = 0;
  for (int i = 0; i < n; ++i)
    if (P.vw[i] > 0) { setBit(&sel, i); wn += P.vw[i]; P.act[na++] = i; }
  P.na = na;
  P.wn = wn;
  P.temp_sel = sel;
}

// Phase 5: candidate d's cost weighted by the samples (lane d), then the current plane's cost
// against each sampled source (lanes split the sources).
template <int kStage>
__device__ __forceinline__ void strong_p5(const CoopCtx &c) {
  if (!c.live) return;
  CoopPixel &P = *c.P;
  const int n = c.n, d = c.lane;
  float fc = 0.0f;
  for (int j = 0; j < n; ++j)
    if (P.vw[j] > 0) fc += P.vw[j] * c.cost[d * n + j];
  P.fc[d] = fc / P.wn;
  const SmemWindow rw = c.window();
  const int na = P.na;
  const float4 pl = P.pl_cur;
  for (int q = c.lane; q < na; q += kCoopLanes)
    c.hc[q] = coop_ncc<kStage>(*c.a, c.px, c.py, P.act[q] + 1, pl, rw);
}

// Phase 6 (lane 0): the current cost, the best candidate and its acceptance, and the five
// refinement planes of PlaneHypothesisRefinementStrong (DPE.cu:1069-1122) with their draws.
__device__ __forceinline__ void strong_p6(const CoopCtx &c) {
  if (!c.live || c.lane != 0) return;
  const PMArgs &a = *c.a;
  const dpe_camera &rc = a.cam[0];
  [[maybe_unused]] const long long L = (long long)a.W * a.H;
  CoopPixel &P = *c.P;
  const int na = P.na;
  float cost_now = 0.0f;
  for (int q = 0; q < na; ++q) cost_now += P.vw[P.act[q]] * c.hc[q];
  cost_now /= P.wn;
  P.cost_written = cost_now;
  const float4 pl_cur = P.pl_cur;
  float depth_now = depth_from_plane(rc, pl_cur, c.px, c.py);
  float4 pl_now = pl_cur;
  uint32_t views_new = G(a.views, c.center, L, 213);
  const int mi = find_min_cost_index(P.fc, 8);
  const float fcost_mi = P.fc[mi];
  if (P.flag[mi]) {
    const float4 cand = G(a.P.use_edge ? a.plane_snap : a.plane, P.pos[mi], L, 214);
    const float db = depth_from_plane(rc, cand, c.px, c.py);
    if (db >= a.P.depth_min && db <= a.P.depth_max && fcost_mi < cost_now) {
      depth_now = db; pl_now = cand; cost_now = fcost_mi;
      views_new = P.temp_sel;
    }
  }
  Rng rng{a.key[0], a.key[1], (uint32_t)c.center, P.rng_ctr};
  const float dmin = a.P.depth_min, dmax = a.P.depth_max;
  const float depth_rand = rng.uniform() * (dmax - dmin) + dmin;
  const float4 n_rand = random_normal(rc, c.px, c.py, rng, depth_now);
  const float lo = (1 - 0.02f) * depth_now, hi = (1 + 0.02f) * depth_now;
  const float depth_pert = rng.uniform() * (hi - lo) + lo;
  const float4 n_pert = perturbed_normal(rc, c.px, c.py, pl_now, rng, (float)(0.02f * 3.14159265358979323846));
  const float depths[5] = {depth_rand, depth_now, depth_rand, depth_now, depth_pert};
  const float4 normals[5] = {pl_now, n_rand, n_rand, n_pert, pl_now};
  for (int h = 0; h < 5; ++h) {
    float4 t = normals[h];
    t.w = dist_to_origin(rc, c.px, c.py, depths[h], t);
    P.hyp[h] = t;
  }
  P.pl_now = pl_now;
  P.depth_now = depth_now;
  P.cost_now = cost_now;
  P.views_new = views_new;
  P.rng_ctr = rng.ctr;
}

// Phase 7: the refinement planes' costs, (plane, sampled source) pairs split over the lanes.
template <int kStage>
__device__ __forceinline__ void strong_p7(const CoopCtx &c) {
  if (!c.live) return;
  const SmemWindow rw = c.window();
  const int na = c.P->na, n = c.n;
  for (int i = c.lane; i < 5 * na; i += kCoopLanes) {
    const int h = i / na, q = i - h * na;
    c.hc[(1 + h) * n + q] = coop_ncc<kStage>(*c.a, c.px, c.py, c.P->act[q] + 1, c.P->hyp[h], rw);
  }
}

// The pixel's outputs after its last decision.
__device__ __forceinline__ void strong_write(const CoopCtx &c, float4 pl_now, float cost_now) {
  const PMArgs &a = *c.a;
  [[maybe_unused]] const long long L = (long long)a.W * a.H;
  const int center = c.center;
  CoopPixel &P = *c.P;
  G(a.rng_ctr, center, L, 215) = P.rng_ctr;
  G(a.views, center, L, 216) = P.views_new;
  store_vweight(&G(a.vweight, center, L, 217), P.vw);
  const float cost_written = P.cost_written;
  if (a.P.state == DPE_REFINE_INIT) {
    if ((double)cost_now < (double)cost_written - 0.1) { G(a.cost, center, L, 218) = cost_now; G(a.plane, center, L, 219) = pl_now; }
    else G(a.cost, center, L, 220) = cost_written;
  } else {
    G(a.cost, center, L, 221) = cost_now;
    G(a.plane, center, L, 222) = pl_now;
  }
}

// Phase 8 (lane 0): the refinement decisions in order, then the outputs -- or, with the
// Gauss-Newton hypothesis, the state phases 9-11 continue from.
template <int kStage, bool kGN>
__device__ __forceinline__ void strong_p8(const CoopCtx &c) {
  if (!c.live || c.lane != 0) return;
  const PMArgs &a = *c.a;
  const dpe_camera &rc = a.cam[0];
  const int na = c.P->na, n = c.n;
  CoopPixel &P = *c.P;
  const float dmin = a.P.depth_min, dmax = a.P.depth_max;
  float depth_now = P.depth_now, cost_now = P.cost_now;
  float4 pl_now = P.pl_now;
  for (int h = 0; h < 5; ++h) {
    const float4 t = P.hyp[h];
    float tc = 0.0f;
    for (int q = 0; q < na; ++q) tc += P.vw[P.act[q]] * c.hc[(1 + h) * n + q];
    tc /= P.wn;
    const float db = depth_from_plane(rc, t, c.px, c.py);
    if (db >= dmin && db <= dmax && tc < cost_now) { depth_now = db; pl_now = t; cost_now = tc; }
  }
  if (kGN) {
    P.pl_now = pl_now; P.depth_now = depth_now; P.cost_now = cost_now;
    return;
  }
  strong_write(c, pl_now, cost_now);
}

#ifdef __CUDA_ARCH__
// Phases 9-11, the Gauss-Newton hypothesis split over the lanes of a pixel.
// Phase 9: lane q adds the normal equations of sampled sources q, q + 8, ...; the lanes' sums are
// added by shuffles inside each 8-lane group (a pixel's lanes are 8 consecutive threads of one
// warp, and every thread of the block takes part); lane 0 solves and keeps the plane in hyp[0].
template <int kStage>
__device__ __forceinline__ void strong_p9_gn(const CoopCtx &c) {
  static_assert(kCoopLanes == 8 && kCoopThreads % 32 == 0, "lane groups must tile whole warps");
  CoopPixel &P = *c.P;
  const bool on = c.live && P.na > 0;
  float m[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  GnFrame f{};
  if (on) {
    const PMArgs &a = *c.a;
    f = gn_frame(a.cam[0], c.px, c.py, P.pl_now, P.depth_now);
    const SmemWindow rw = c.window();
    for (int q = c.lane; q < P.na; q += kCoopLanes)
      gn_accumulate(a, c.px, c.py, rw, P.pl_now, f, P.act[q], (float)P.vw[P.act[q]], m);
  }
#pragma unroll
  for (int k = 0; k < 9; ++k)
#pragma unroll
    for (int off = 1; off < kCoopLanes; off <<= 1) m[k] += __shfl_xor_sync(0xffffffffu, m[k], off, kCoopLanes);
  if (on && c.lane == 0) {
    float4 t;
    const bool ok = gn_solve(*c.a, c.px, c.py, P.pl_now, f, m, &t);
    P.flag[0] = ok ? 1 : 0;
    if (ok) P.hyp[0] = t;
  }
}
// Phase 10: the hypothesis' cost against each sampled source, split over the lanes (hc row 0).
template <int kStage>
__device__ __forceinline__ void strong_p10_gn(const CoopCtx &c) {
  if (!c.live) return;
  const CoopPixel &P = *c.P;
  if (P.na == 0 || !P.flag[0]) return;
  const SmemWindow rw = c.window();
  for (int q = c.lane; q < P.na; q += kCoopLanes) c.hc[q] = coop_ncc<kStage>(*c.a, c.px, c.py, P.act[q] + 1, P.hyp[0], rw);
}
// Phase 11 (lane 0): the weighted cost in list order, the decision, the outputs.
__device__ __forceinline__ void strong_p11_gn(const CoopCtx &c) {
  if (!c.live || c.lane != 0) return;
  const PMArgs &a = *c.a;
  const CoopPixel &P = *c.P;
  float4 pl_now = P.pl_now;
  float cost_now = P.cost_now;
  if (P.na > 0 && P.flag[0]) {
    float tc = 0.0f;
    for (int q = 0; q < P.na; ++q) tc += P.vw[P.act[q]] * c.hc[q];
    tc /= P.wn;
    const float4 t = P.hyp[0];
    const float db = depth_from_plane(a.cam[0], t, c.px, c.py);
    if (db >= a.P.depth_min && db <= a.P.depth_max && tc < cost_now) { pl_now = t; cost_now = tc; }
  }
  strong_write(c, pl_now, cost_now);
}
#endif

// One phase for one thread (host builds of this source run the phases in lock-step over a block).
template <int kStage, bool kGN>
__device__ __forceinline__ void strong_update_phase(int phase, const Launch &lc, int iter, int parity, void *smem) {
  const CoopCtx c = coop_ctx(lc, parity, smem);
  switch (phase) {
    case 0: strong_p0(c); break;
    case 1: strong_p1(c); break;
    case 2: strong_p2<kStage>(c, iter); break;
    case 3: strong_p3(c, iter); break;
    case 4: strong_p4(c); break;
    case 5: strong_p5<kStage>(c); break;
    case 6: strong_p6(c); break;
    case 7: strong_p7<kStage>(c); break;
    default: strong_p8<kStage, kGN>(c); break;
  }
}
constexpr int kStrongPhases = 9;

// Grid: ((W + 15) / 16, (H + 1) / 2) blocks of kCoopThreads; coop_smem_bytes(N - 1) dynamic shared
// bytes (the largest N of a batch).
template <int kStage, bool kGN>
__global__ void __launch_bounds__(kCoopThreads, DPE_STRONG_MIN_BLOCKS) k_strong_update(const Launch lc, int iter, int parity) {
  extern __shared__ float4 coop_smem[];
  const CoopCtx c = coop_ctx(lc, parity, coop_smem);
  strong_p0(c);
  __syncthreads();
  strong_p1(c);
  __syncthreads();
  strong_p2<kStage>(c, iter);
  __syncthreads();
  strong_p3(c, iter);
  __syncthreads();
  strong_p4(c);
  __syncthreads();
  strong_p5<kStage>(c);
  __syncthreads();
  strong_p6(c);
  __syncthreads();
  strong_p7<kStage>(c);
  __syncthreads();
  strong_p8<kStage, kGN>(c);
#ifdef __CUDA_ARCH__
  if constexpr (kGN) {
    __syncthreads();
    strong_p9_gn<kStage>(c);
    __syncthreads();
    strong_p10_gn<kStage>(c);
    __syncthreads();
    strong_p11_gn(c);
  }
#endif
}


// ------------------------------------------------------------------ RANSACToGetFitPlane (DPE.cu:2895-3128)
__device__ __forceinline__ void ransac_fit_plane_pixel(const PMArgs &a, int px, int py) {
  const int W = a.W, center = px + py * W;
  if (a.weak[center] != DPE_WEAK) { a.fit_plane[center] = a.plane[center]; return; }
  Rng rng = make_rng(a, center);
  const dpe_camera &cam = a.cam[0];
  bool edge_limit = false;
  if (a.P.use_limit) {
    edge_limit = true;
    if (a.P.use_edge) {
      const float cv = a.complexity[center];
      const float rp = rng.uniform() - FLT_EPSILON;
      if (rp < cv) edge_limit = false;
    }
  }
  short2 sp[kNeighbours - 1];
  float3 sp3[kNeighbours - 1], spn[kNeighbours - 1];
  int sc = 0;
  float X[3];
  for (int i = 1; i < kNeighbours; ++i) {
    const short2 t = neighbour(a, center, i);
    if (t.x == -1 || t.y == -1) continue;
    sp[sc] = t;
    const int tc = t.x + t.y * W;
    const float4 tpl = a.plane[tc];
    const float d = depth_from_plane(cam, tpl, t.x, t.y);
    point3d(cam, t.x, t.y, d, X);
    sp3[sc] = make_float3(X[0], X[1], X[2]);
    spn[sc] = make_float3(tpl.x, tpl.y, tpl.z);
    sc++;
  }
  if (sc < 3) { a.fit_plane[center] = a.plane[center]; a.rng_ctr[center] = rng.ctr; return; }
  int ua = -1, ub = -1, uc = -1;
  float min_cost = FLT_MAX;
  float4 best = make_float4(0, 0, 0, 0);
  bool has_best = false, has_strong = false;
  bool must_tri = (a.P.use_label && a.label[center] > 0 && edge_limit) ? false : true;
  for (int iteration = 0; iteration < 50; ++iteration) {
    const int ia = (int)(rng.u32() % (uint32_t)sc);
    const int ib = (int)(rng.u32() % (uint32_t)sc);
    const int ic = (int)(rng.u32() % (uint32_t)sc);
    if (ia == ib || ib == ic || ia == ic) continue;
    bool is_strong = false;
    if (a.P.geom_consistency && edge_limit) {
      const float3 AN = spn[ia], BN = spn[ib], CN = spn[ic];
      is_strong = true;
      if ((double)(AN.x * BN.x + AN.y * BN.y + AN.z * BN.z) < 0.8660254 ||
          (double)(AN.x * CN.x + AN.y * CN.y + AN.z * CN.z) < 0.8660254 ||
          (double)(BN.x * CN.x + BN.y * CN.y + BN.z * CN.z) < 0.8660254)
        is_strong = false;
      if (has_strong && !is_strong) continue;
    }
    if (must_tri && !point_in_triangle(sp[ia], sp[ib], sp[ic], px, py)) continue;
    if (edge_limit) {
      if (bresenham(a, sp[ia].x, sp[ia].y, sp[ib].x, sp[ib].y) || bresenham(a, sp[ib].x, sp[ib].y, sp[ic].x, sp[ic].y) ||
          bresenham(a, sp[ic].x, sp[ic].y, sp[ia].x, sp[ia].y))
        continue;
    }
    const float3 A = sp3[ia], B = sp3[ib], C = sp3[ic];
    const float3 AC = make_float3(A.x - C.x, A.y - C.y, A.z - C.z), BC = make_float3(B.x - C.x, B.y - C.y, B.z - C.z);
    float4 cr;
    cr.x = AC.y * BC.z - BC.y * AC.z;
    cr.y = -(AC.x * BC.z - BC.x * AC.z);
    cr.z = AC.x * BC.y - BC.x * AC.y;
    if ((cr.x == 0 && cr.y == 0 && cr.z == 0) || isnan(cr.x) || isnan(cr.y) || isnan(cr.z)) continue;
    normalize3(&cr);
    cr.w = -(cr.x * A.x + cr.y * A.y + cr.z * A.z);
    if (!has_strong && is_strong) has_strong = true;
    float tc = 0.0f;
    for (int s = 0; s < sc; ++s) {
      if (s == ia || s == ib || s == ic) continue;
      const float fx = (sp[s].x - cam.K[2]) / cam.K[0];
      const float fy = (sp[s].y - cam.K[5]) / cam.K[4];
      const float fd = -cr.w / (cr.x * fx + cr.y * fy + cr.z);
      tc += fabsf(fd - sp3[s].z);
    }
    if (tc < min_cost) {
      if (!must_tri && point_in_triangle(sp[ia], sp[ib], sp[ic], px, py)) must_tri = true;
      min_cost = tc; best = cr; has_best = true; ua = ia; ub = ib; uc = ic;
    }
  }
  a.rng_ctr[center] = rng.ctr;
  if (has_best) {
    const float depth = depth_from_plane(cam, a.plane[center], px, py);
    const float4 v = view_direction(cam, px, py, depth);
    if (best.x * v.x + best.y * v.y + best.z * v.z > 0) { best.x = -best.x; best.y = -best.y; best.z = -best.z; best.w = -best.w; }
    a.fit_plane[center] = best;
    if (a.P.use_radius) {
      if (must_tri) {
        const short2 A = sp[ua], B = sp[ub], C = sp[uc];
        const float la = sqrtf((float)((A.x - B.x) * (A.x - B.x) + (A.y - B.y) * (A.y - B.y)));
        const float lb = sqrtf((float)((B.x - C.x) * (B.x - C.x) + (B.y - C.y) * (B.y - C.y)));
        const float lc = sqrtf((float)((C.x - A.x) * (C.x - A.x) + (C.y - A.y) * (C.y - A.y)));
        const float p = (float)((la + lb + lc) / 2.0);
        const float S = sqrtf(p * (p - la) * (p - lb) * (p - lc));
        int radius = (int)floor(sqrtf(S) / 2.0);
        const float ad = sqrtf((float)((A.x - px) * (A.x - px) + (A.y - py) * (A.y - py)));
        const float bd = sqrtf((float)((B.x - px) * (B.x - px) + (B.y - py) * (B.y - py)));
        const float cd = sqrtf((float)((C.x - px) * (C.x - px) + (C.y - py) * (C.y - py)));
        const float md = cvmin(cvmin(ad, bd), cd);
        if (2.5 * md < radius) radius = (int)md;
        if (edge_limit) {
          if (a.P.use_edge) {
            float med = FLT_MAX;
            const short2 *en = &a.edge_neigh[(size_t)center * 8];
            for (int d = 0; d < 8; ++d) {
              const short2 e = en[d];
              if (e.x == -1 || e.y == -1) continue;
              med = cvmin(med, sqrtf((float)((e.x - px) * (e.x - px) + (e.y - py) * (e.y - py))));
            }
            if (med < radius) radius = (int)med;
          }
          if (a.P.use_label && a.label[center] > 0) {
            float mbd = FLT_MAX;
            const short2 *lb2 = &a.lab_bound[(size_t)a.nmap[center] * 8];
            for (int d = 0; d < 8; ++d) {
              const short2 bb = lb2[d];
              if (bb.x == -1 || bb.y == -1) continue;
              const double ddx = (double)(px - bb.x), ddy = (double)(py - bb.y);
              mbd = cvmin(mbd, (float)sqrt(ddx * ddx + ddy * ddy));
            }
            if (mbd < radius) radius = (int)mbd;
          }
        }
        for (int guard = 0; (radius << 1) % 5 != 0 && guard < 5; ++guard) radius--;
        if (!edge_limit) a.radius[center] = radius > a.P.strong_radius ? 0 : a.P.strong_radius;
        else a.radius[center] = radius > a.P.strong_radius ? radius : a.P.strong_radius;
      } else {
        a.radius[center] = a.P.strong_radius;
      }
    }
  } else {
    a.fit_plane[center] = make_float4(0, 0, 0, 0);
    if (a.P.use_radius) a.radius[center] = a.P.strong_radius;
  }
}
// One thread per pixel of a 2D grid: the tiles keep the rays of neighbouring pixels together
// (measured faster than a work list over the WEAK pixels).
__global__ void __launch_bounds__(128, DPE_LATENCY_MIN_BLOCKS) k_ransac_fit_plane(const Launch lc) {
  const Blk B = resolve<kGridFull>(lc);
  const PMArgs &a = *B.a;
  int px, py;
  if (!full_pixel(a, B, &px, &py)) return;
  ransac_fit_plane_pixel(a, px, py);
}

// ------------------------------------------------------------------ weak update (DPE.cu:1672-1866, 1124-1216)
// CheckerboardPropagationWeak + PlaneHypothesisRefinementWeak for the WEAK pixels of one colour,
// split into work lists so that every lane has work:
//   k_weak_prepare      per pixel: the reference side of its nine windows (table, sums);
//   k_weak_eval<false>  per (pixel, hypothesis, source): the 8 strong-neighbour candidates, the
//                       current plane and the fitted plane;
//   k_weak_decide       per pixel: view sampling, candidate choice, fitted-plane test, and the five
//                       random refinement hypotheses (all random draws of the pixel);
//   k_weak_eval<true>   per (pixel, random hypothesis, sampled source);
//   k_weak_finish       per pixel: the random-hypothesis test, the REFINE_INIT rule, the write-back
//                       and the final strong-window re-cost.
// Each cost is the one the fused per-pixel form computes, and every sum runs in the same order.
// Pixels of one colour read only STRONG neighbours and their own state, so the order of the
// list does not matter.  Work items are strided over a grid sized for the GPU; the list lengths
// stay on the device.

__global__ void __launch_bounds__(128) k_weak_prepare(const Launch lc, int parity) {
  const Blk B = resolve<kGridList>(lc);
  const PMArgs &a = *B.a;
  const int count = a.wcount[parity];
  const int *list = a.wlist[parity];
  for (int slot = B.x * blockDim.x + threadIdx.x; slot < count; slot += B.gx * blockDim.x) {
    const int center = list[slot];
    const int px = center % a.W, py = center / a.W;
    const float ref_center = texel(a, 0, px, py);
    float2 *tab = a.wtab + (size_t)slot * a.wtab_stride;
    for (int k = 0; k < kNeighbours; ++k) {
      const short2 nb = neighbour(a, center, k);
      float4 win = make_float4(0, 0, 0, 0);
      if (nb.x != -1 && nb.y != -1) {
        int radius, inc;
        weak_window_shape(a, center, k, &radius, &inc);
        int t = weak_window_base(a, k);
        float s_r = 0, s_rr = 0, s_w = 0;
        for (int i = -radius; i <= radius; i += inc) {
          float r_r = 0, r_rr = 0, r_w = 0;
          for (int j = -radius; j <= radius; j += inc) {
            const float rp = texel(a, 0, nb.x + i, nb.y + j);
            const float w = bilateral_weight((float)i, (float)j, rp, ref_center, a.P.sigma_spatial, a.P.sigma_color);
            const float rc = rp - ref_center;
            tab[t++] = make_float2(w, w * rc);
            r_r += w * rc; r_rr += w * rc * rc; r_w += w;
          }
          s_r += r_r; s_rr += r_rr; s_w += r_w;
        }
        win = make_float4(s_w, s_r, s_rr, 0.0f);
      }
      a.wwin[(size_t)slot * kNeighbours + k] = win;
    }
  }
}

// kRandom = false: hypotheses 0..7 are the candidates (the planes of the strong neighbours 1..8),
// 8 the current plane, 9 the fitted plane.  kRandom = true: the five random hypotheses, for the
// sources the pixel sampled.  Unevaluated candidates keep the fused form's initial costs (0, and 2
// for the first candidate's first source: quirk Q2).
template <bool kRandom, int kStage>
// Resident blocks requested for the deformable evaluation (__launch_bounds__): measured on the
// 10-view 1600x1200 schedule, 8 blocks (64 registers, a few spills) make it 21 % faster than the
// unbounded 96 registers and 5 blocks: it waits on its gathers, and more warps hide them.
#ifndef DPE_WEAK_MIN_BLOCKS
#define DPE_WEAK_MIN_BLOCKS 8
#endif
__global__ void __launch_bounds__(128, DPE_WEAK_MIN_BLOCKS) k_weak_eval(const Launch lc, int parity) {
  const Blk B = resolve<kGridList>(lc);
  const PMArgs &a = *B.a;
  const int n = a.N - 1;
  const int hyps = kRandom ? 5 : 10;
  const long long per = (long long)hyps * n;
  const long long total = (long long)a.wcount[parity] * per;
  const int *list = a.wlist[parity];
  const bool geom = a.P.geom_consistency != 0;
  float *costs = kRandom ? a.wcost_r : a.wcost;
  float *geoms = kRandom ? a.wgeom_r : a.wgeom;
  for (long long t = (long long)B.x * blockDim.x + threadIdx.x; t < total; t += (long long)B.gx * blockDim.x) {
    const int slot = (int)(t / per);
    const int r = (int)(t - (long long)slot * per);
    const int h = r / n, j = r - h * n;
    const int center = list[slot];
    const int px = center % a.W, py = center / a.W;
    float4 pl;
    if (kRandom) {
      const float4 fp = a.fit_plane[center];
      if (fp.x == 0 && fp.y == 0 && fp.z == 0) continue;  // no random refinement for this pixel
      if (vweight_at(a.vweight[center], j) == 0) continue;
      pl = a.whyp[(size_t)slot * 5 + h];
    } else if (h < 8) {
      const short2 nb = neighbour(a, center, h + 1);
      if (nb.x == -1 || nb.y == -1 || a.weak[nb.x + nb.y * a.W] != DPE_STRONG) {
        costs[t] = (h == 0 && j == 0) ? 2.0f : 0.0f;
        geoms[t] = 0.0f;
        continue;
      }
      pl = a.plane[nb.x + nb.y * a.W];
    } else if (h == 8) {
      pl = a.plane[center];
    } else {
      pl = a.fit_plane[center];
      if (pl.x == 0 && pl.y == 0 && pl.z == 0) continue;  // unused: refinement skipped
    }
    costs[t] = ncc_weak_tab<kStage>(a, slot, center, px, py, j + 1, pl, KID_WEAK_EVAL);
    geoms[t] = geom ? geom_cost(a, px, py, j + 1, pl) : 0.0f;
  }
}

__global__ void __launch_bounds__(128) k_weak_decide(const Launch lc, int iter, int parity) {
  const Blk B = resolve<kGridList>(lc);
  const PMArgs &a = *B.a;
  const int n = a.N - 1, W = a.W;
  const int count = a.wcount[parity];
  const int *list = a.wlist[parity];
  const dpe_camera &rc = a.cam[0];
  const bool geom = a.P.geom_consistency != 0;
  const float gf = a.P.geom_factor;
  const float dmin = a.P.depth_min, dmax = a.P.depth_max;
  float priors[kMaxSrc], probs[kMaxSrc];
  uint8_t vw[32];
  float final_costs[8];
  bool flag[8];
  float4 cand[8];
  for (int slot = B.x * blockDim.x + threadIdx.x; slot < count; slot += B.gx * blockDim.x) {
    const int center = list[slot];
    const int px = center % W, py = center / W;
    const float *ca = a.wcost + (size_t)slot * 10 * n;
    const float *ga = a.wgeom + (size_t)slot * 10 * n;
    for (int i = 0; i < 8; ++i) {
      const short2 nb = neighbour(a, center, i + 1);
      flag[i] = !(nb.x == -1 || nb.y == -1 || a.weak[nb.x + nb.y * W] != DPE_STRONG);
      cand[i] = flag[i] ? a.plane[nb.x + nb.y * W] : make_float4(0, 0, 0, 0);
    }
    for (int j = 0; j < n; ++j) priors[j] = 0.0f;
    for (int i = 0; i < 8; ++i) {
      const short2 nb = neighbour(a, center, i + 1);
      if (nb.x == -1 || nb.y == -1) continue;
      const uint32_t sv = a.views[nb.x + nb.y * W];
      for (int j = 0; j < n; ++j) priors[j] += isSet(sv, j) == 1 ? 0.9f : 0.1f;
    }
    Rng rng = make_rng(a, center);
    uint32_t temp_sel = 0;
    const float wn = sample_views(a, rng, iter, ca, n, priors, vw, &temp_sel, probs);
    for (int i = 0; i < 8; ++i) {
      float fc = 0.0f;
      for (int j = 0; j < n; ++j)
        if (vw[j] > 0) {
          if (geom) fc += vw[j] * (ca[i * n + j] + gf * (flag[i] ? ga[i * n + j] : 3.0f));
          else fc += vw[j] * ca[i * n + j];
        }
      final_costs[i] = fc / wn;
    }
    const int mi = find_min_cost_index(final_costs, 8);
    const float4 pl_cur = a.plane[center];
    float cost_now = 0.0f;
    for (int i = 0; i < n; ++i) {
      if (vw[i] == 0) continue;  // 0 * (finite cost) contributes nothing
      const float c = ca[8 * n + i];
      if (geom) cost_now += vw[i] * (c + gf * ga[8 * n + i]);
      else cost_now += vw[i] * c;
    }
    cost_now /= wn;
    const float cost_written = cost_now;
    float depth_now = depth_from_plane(rc, pl_cur, px, py);
    float4 pl_now = pl_cur;
    uint32_t views_new = a.views[center];
    if (flag[mi]) {
      const float db = depth_from_plane(rc, cand[mi], px, py);
      if (db >= dmin && db <= dmax && final_costs[mi] < cost_now) {
        depth_now = db; pl_now = cand[mi]; cost_now = final_costs[mi];
        views_new = temp_sel;
      }
    }
    // PlaneHypothesisRefinementWeak: the fitted plane, then five random hypotheses.  A zero fitted
    // plane ends the refinement before the random hypotheses (DPE.cu:1146-1148).
    const float4 fp = a.fit_plane[center];
    if (!(fp.x == 0 && fp.y == 0 && fp.z == 0)) {
      float tc = 0.0f;
      for (int j = 0; j < n; ++j)
        if (vw[j] > 0) {
          const float c = ca[9 * n + j];
          if (geom) tc += vw[j] * (c + gf * ga[9 * n + j]);
          else tc += vw[j] * c;
        }
      tc /= wn;
      const float db = depth_from_plane(rc, fp, px, py);
      if (db >= dmin && db <= dmax && tc < cost_now) { depth_now = db; pl_now = fp; cost_now = tc; }
      const float depth_rand = rng.uniform() * (dmax - dmin) + dmin;
      const float4 n_rand = random_normal(rc, px, py, rng, depth_now);
      const float lo = (1 - 0.02f) * depth_now, hi = (1 + 0.02f) * depth_now;
      const float depth_pert = rng.uniform() * (hi - lo) + lo;
      const float4 n_pert = perturbed_normal(rc, px, py, pl_now, rng, (float)(0.02f * 3.14159265358979323846));
      const float depths[5] = {depth_rand, depth_now, depth_rand, depth_now, depth_pert};
      const float4 normals[5] = {pl_now, n_rand, n_rand, n_pert, pl_now};
      for (int h = 0; h < 5; ++h) {
        float4 t = normals[h];
        t.w = dist_to_origin(rc, px, py, depths[h], t);
        a.whyp[(size_t)slot * 5 + h] = t;
      }
    }
    a.rng_ctr[center] = rng.ctr;
    a.views[center] = views_new;
    store_vweight(&a.vweight[center], vw);
    a.wstate[(size_t)slot * 2] = pl_now;
    a.wstate[(size_t)slot * 2 + 1] = make_float4(depth_now, cost_now, cost_written, wn);
  }
}

template <int kStage>
__global__ void __launch_bounds__(128) k_weak_finish(const Launch lc, int parity) {
  const Blk B = resolve<kGridList>(lc);
  const PMArgs &a = *B.a;
  const int n = a.N - 1, W = a.W;
  const int count = a.wcount[parity];
  const int *list = a.wlist[parity];
  const dpe_camera &rc = a.cam[0];
  const bool geom = a.P.geom_consistency != 0;
  const float gf = a.P.geom_factor;
  const float dmin = a.P.depth_min, dmax = a.P.depth_max;
  for (int slot = B.x * blockDim.x + threadIdx.x; slot < count; slot += B.gx * blockDim.x) {
    const int center = list[slot];
    const int px = center % W, py = center / W;
    float4 pl_now = a.wstate[(size_t)slot * 2];
    const float4 st = a.wstate[(size_t)slot * 2 + 1];
    float cost_now = st.y;
    const float cost_written = st.z, wn = st.w;
    const uint4 vwp = a.vweight[center];
    const float4 fp = a.fit_plane[center];
    if (!(fp.x == 0 && fp.y == 0 && fp.z == 0)) {
      const float *cr = a.wcost_r + (size_t)slot * 5 * n;
      const float *gr = a.wgeom_r + (size_t)slot * 5 * n;
      for (int h = 0; h < 5; ++h) {
        const float4 t = a.whyp[(size_t)slot * 5 + h];
        float tc = 0.0f;
        for (int j = 0; j < n; ++j) {
          const int v = vweight_at(vwp, j);
          if (v > 0) {
            const float c = cr[h * n + j];
            if (geom) tc += v * (c + gf * gr[h * n + j]);
            else tc += v * c;
          }
        }
        tc /= wn;
        const float db = depth_from_plane(rc, t, px, py);
        if (db >= dmin && db <= dmax && tc < cost_now) { pl_now = t; cost_now = tc; }
      }
    }
    float4 pl_final = a.plane[center];
    if (a.P.state == DPE_REFINE_INIT) {
      if ((double)cost_now < (double)cost_written - 0.1) pl_final = pl_now;
    } else {
      pl_final = pl_now;
    }
    a.plane[center] = pl_final;
    // final re-cost with the strong window (DPE.cu:1849-1865); the radius swap there has no effect
    DPE_REF_WINDOW(rw);
    build_ref_window(a, px, py, rw, KID_WEAK_FINISH);
    uint8_t vw[32];
    int act[kMaxSrc];
    int na = 0;
    for (int i = 0; i < n; ++i) {
      vw[i] = (uint8_t)vweight_at(vwp, i);
      if (vw[i] > 0) act[na++] = i;
    }
    a.cost[center] = weighted_ncc<kStage>(a, px, py, pl_final, rw, act, na, vw) / wn;
  }
}

// ------------------------------------------------------------------ post passes
__global__ void k_get_depth_normal(const Launch lc) {
  const Blk B = resolve<kGridFull>(lc);
  const PMArgs &a = *B.a;
  int px, py;
  if (!full_pixel(a, B, &px, &py)) return;
  const int c = py * a.W + px;
  float4 pl = a.plane[c];
  pl.w = depth_from_plane(a.cam[0], pl, px, py);
  a.plane[c] = normal_to_world(a.cam[0], pl);
}

// CheckerboardFilterStrong (DPE.cu:1961-2071)
__global__ void k_filter_strong(const Launch lc, int parity) {
  const Blk B = resolve<kGridHalf>(lc);
  const PMArgs &a = *B.a;
  int px, py;
  if (!colour_pixel(a, B, parity, &px, &py)) return;
  const int W = a.W, H = a.H, center = py * W + px;
  if (a.weak[center] == DPE_WEAK) return;
  if (a.cost[center] < 0.001f) return;
  float f[21];
  int k = 0;
  f[k++] = a.plane[center].w;
  const int up = center - W, upup = center - 3 * W, dn = center + W, dndn = center + 3 * W;
  const int lf = center - 1, lflf = center - 3, rt = center + 1, rtrt = center + 3;
  const int idx[20] = {up, upup, upup - 2 * W, dn, dndn, dndn + 2 * W, lf, lflf, lflf - 2, rt, rtrt, rtrt + 2,
                       up + 2, dn + 2, up - 2, dn - 2, lf - 2 * W, rt - 2 * W, lf + 2 * W, rt + 2 * W};
  const bool ok[20] = {py > 0, py > 2, py > 4, py < H - 1, py < H - 3, py < H - 5, px > 0, px > 2, px > 4,
                       px < W - 1, px < W - 3, px < W - 5, py > 0 && px < W - 2, py < H - 1 && px < W - 2,
                       py > 0 && px > 1, py < H - 1 && px > 1, px > 0 && py > 2, px < W - 1 && py > 2,
                       px > 0 && py < H - 2, px < W - 1 && py < H - 2};
  for (int i = 0; i < 20; ++i)
    if (ok[i] && a.weak[idx[i]] == DPE_STRONG) f[k++] = a.plane[idx[i]].w;
  sort_small(f, k);
  const int m = k / 2;
  a.plane[center].w = (k % 2 == 0) ? (f[m - 1] + f[m]) / 2 : f[m];
}

// ------------------------------------------------------------------ DepthToWeak / LocalRefine
// Block-cooperative like the strong update: a block holds kCoopPix consecutive pixels of one row
// and kCoopLanes threads per pixel.  The pixel's reference window and its per-sample costs live
// in shared memory; the lanes split the depth samples (each sample's sum over the selected
// sources stays on one lane, in source order), and one lane per pixel takes the decision.
//   phase 0  window taps (lanes split the taps)
//   phase 1  window sums and the sweep prologue (DPE.cu:2619-2660, 2767-2806) (lane 0)
//   phase 2  sample costs (lanes split the samples; LocalRefine also the current plane's sources)
//   phase 3  the decision (lane 0)
struct SweepPixel {
  float2 win[kWinTaps];
  float rc[kWinTaps];
  float4 pl;
  uint4 vw;
  float center, inv_wsum, mean_r, var_r;
  float depth, base_line, weight_normal, disp;
  int act[kMaxSrc];
  int na, ok;           // ok: the sweep runs for this pixel
  float pc[64];         // DepthToWeak: the 61 sample costs
};
constexpr int kSweepPhases = 4;
// LocalRefine's shared bytes: the pixels, then per pixel 12 planes (the current one, then the 11
// samples) x n = N - 1 sources of (NCC, geometric cost).
__host__ __device__ inline size_t local_refine_smem_bytes(int n) {
  return sizeof(SweepPixel) * kCoopPix + sizeof(float2) * (size_t)kCoopPix * 12 * n;
}

struct SweepCtx {
  const PMArgs *a;
  int slot, lane, px, py, center;
  bool live;  // inside the image
  SweepPixel *P;
  float2 *items;  // LocalRefine: [12][n] (NCC, geometric cost) of this pixel
  int kid;
  __device__ __forceinline__ SmemWindow window() const {
    return SmemWindow{P->win, P->center, P->inv_wsum, P->mean_r, P->var_r, a->counters ? a->counters + 2 * kid : nullptr};
  }
};
__device__ __forceinline__ SweepCtx sweep_ctx(const Launch &lc, void *smem, int kid) {
  const Blk B = resolve<kGridFull>(lc);
  SweepCtx c;
  c.a = B.a;
  c.slot = (int)threadIdx.x / kCoopLanes;
  c.lane = (int)threadIdx.x % kCoopLanes;
  c.px = B.x * kCoopPix + c.slot;
  c.py = B.y;
  c.center = c.py * B.a->W + c.px;
  c.live = c.px < B.a->W && c.py < B.a->H;
  c.P = static_cast<SweepPixel *>(smem) + c.slot;
  c.items = reinterpret_cast<float2 *>(static_cast<SweepPixel *>(smem) + kCoopPix) + (size_t)c.slot * 12 * (B.a->N - 1);
  c.kid = kid;
  return c;
}

// Phase 0: the window taps, split over the lanes (as strong_p0).
__device__ __forceinline__ void sweep_p0(const SweepCtx &c) {
  if (!c.live) return;
  const PMArgs &a = *c.a;
  const int r = a.P.strong_radius, inc = a.P.strong_increment, side = 2 * r / inc + 1;
  const float center = texel(a, 0, c.px, c.py);
  for (int k = c.lane; k < side * side; k += kCoopLanes) {
    const int i = -r + (k / side) * inc, j = -r + (k % side) * inc;
    const float rp = texel(a, 0, c.px + i, c.py + j);
    const float w = bilateral_weight((float)i, (float)j, rp, center, a.P.sigma_spatial, a.P.sigma_color);
    const float rcv = rp - center;
    G(c.P->win, k, kWinTaps, 320) = make_float2(w, w * rcv);
    c.P->rc[k] = rcv;
  }
  if (c.lane == 0) c.P->center = center;
}

// Phase 1 (lane 0): window sums; the prologue's plane, baseline, weights and selected sources.
// (The reference's DepthToWeak also costs the current plane here and never reads the result; it
// is not computed.  LocalRefine's current cost is computed by the lanes in phase 2.)
__device__ __forceinline__ void sweep_p1(const SweepCtx &c) {
  if (!c.live || c.lane != 0) return;
  const PMArgs &a = *c.a;
  SweepPixel &P = *c.P;
  const int r = a.P.strong_radius, inc = a.P.strong_increment, side = 2 * r / inc + 1;
  float sw = 0.f, swr = 0.f, swrr = 0.f;
  for (int k = 0; k < side * side; ++k) {
    const float2 t = P.win[k];
    sw += t.x; swr += t.y; swrr += t.y * P.rc[k];
  }
  P.inv_wsum = 1.0f / sw;
  P.mean_r = swr * P.inv_wsum;
  P.var_r = swrr * P.inv_wsum - P.mean_r * P.mean_r;
  P.pl = normal_to_ref(a.cam[0], a.plane[c.center]);
  P.depth = P.pl.w;
  const uint32_t views = a.views[c.center];
  P.vw = a.vweight[c.center];
  float base_line = 0.0f, weight_normal = 0.0f;
  int valid = 0, na = 0;
  for (int si = 1; si < a.N; ++si) {
    const int vi = si - 1;
    if (!isSet(views, vi)) continue;
    weight_normal += vweight_at(P.vw, vi);
    const float d0 = a.cam[0].c[0] - a.cam[si].c[0], d1 = a.cam[0].c[1] - a.cam[si].c[1], d2 = a.cam[0].c[2] - a.cam[si].c[2];
    const double tv = d0 * d0 + d1 * d1 + d2 * d2;
    base_line += sqrtf((float)tv);
    valid++;
    P.act[na++] = vi;
  }
  P.na = na;
  P.ok = P.depth != 0 && valid != 0;
  P.weight_normal = weight_normal;
  if (P.ok) {
    P.base_line = base_line / valid;
    P.disp = a.cam[0].K[0] * P.base_line / P.depth;
  }
}

// Cost of the plane of depth pdep: the weighted sum over the selected sources (DPE.cu:2676-2700,
// 2815-2828), summed in source order.  kLocal: LocalRefine's association (each term weighted).
template <int kStage, bool kLocal>
__device__ __forceinline__ float sweep_sample(const SweepCtx &c, const SmemWindow &rw, float pdep) {
  const PMArgs &a = *c.a;
  const SweepPixel &P = *c.P;
  float4 t = P.pl;
  t.w = dist_to_origin(a.cam[0], c.px, c.py, pdep, t);
  float cost = 0.0f;
  for (int q = 0; q < P.na; ++q) {
    const int vi = P.act[q];
    const int w = vweight_at(P.vw, vi);
    if (kLocal) {
      cost += ncc_strong<kStage, kSweepUnroll>(a, c.px, c.py, vi + 1, t, rw) * w;
      if (a.P.geom_consistency) cost += a.P.geom_factor * geom_cost(a, c.px, c.py, vi + 1, t) * w;
    } else {
      float tc = ncc_strong<kStage, kSweepUnroll>(a, c.px, c.py, vi + 1, t, rw);
      if (a.P.geom_consistency) tc += a.P.geom_factor * geom_cost(a, c.px, c.py, vi + 1, t);
      cost += tc * w;
    }
  }
  return cost;
}

// DepthToWeak (DPE.cu:2597-2751), phases 2 and 3.
template <int kStage>
__device__ __forceinline__ void d2w_p2(const SweepCtx &c) {
  if (!c.live || !c.P->ok) return;
  const PMArgs &a = *c.a;
  const SmemWindow rw = c.window();
  constexpr int R = 30, NS = 61;
  for (int s = c.lane; s < NS; s += kCoopLanes) {
    const int pd = s - R;
    const float pdep = a.cam[0].K[0] * c.P->base_line / (c.P->disp + pd);
    float v = 2.0f;
    if (!(pdep < a.P.depth_min || pdep > a.P.depth_max))
      v = cvmin(2.0f, sweep_sample<kStage, false>(c, rw, pdep) / c.P->weight_normal);
    c.P->pc[s] = v;
  }
}
__device__ __forceinline__ void d2w_p3(const SweepCtx &c) {
  if (!c.live || c.lane != 0) return;
  const PMArgs &a = *c.a;
  const int W = a.W, H = a.H, margin = 6;
  const float *pc = c.P->pc;
  if (c.px < margin || c.py < margin || c.px >= W - margin || c.py >= H - margin || !c.P->ok) {
    a.weak[c.center] = DPE_UNKNOWN;
    return;
  }
  constexpr int R = 30, NS = 61;
  int peaks = 0, min_peak = 0;
  float min_cost = 2.0f;
  uint64_t peak_mask = 0;
  for (int i = 2; i < NS - 2; ++i)
    if (pc[i - 1] > pc[i] && pc[i + 1] > pc[i]) {
      peak_mask |= 1ull << i; peaks++;
      if (pc[i] < min_cost) { min_peak = i; min_cost = pc[i]; }
    }
  uint8_t res;
  if (abs(min_peak - R) > a.P.weak_peak_radius || pc[min_peak] > 0.5f) res = DPE_WEAK;
  else if (peaks == 1) res = pc[min_peak] <= 0.15f ? DPE_STRONG : DPE_WEAK;
  else {
    float var = 0.0f;
    for (int i = 2; i < NS - 2; ++i)
      if (((peak_mask >> i) & 1ull) && i != min_peak) { const float d = pc[i] - min_cost; var += d * d; }
    var = sqrtf(var);
    var /= (peaks - 1);
    res = var > 0.2f ? DPE_STRONG : DPE_WEAK;
  }
  a.weak[c.center] = res;
}
// The margin pixels take no window or sweep: phase 0 and 1 skip them through `live` as well.
__device__ __forceinline__ SweepCtx d2w_ctx(const Launch &lc, void *smem) {
  SweepCtx c = sweep_ctx(lc, smem, KID_DEPTH_TO_WEAK);
  const int margin = 6;
  if (c.live && (c.px < margin || c.py < margin || c.px >= c.a->W - margin || c.py >= c.a->H - margin)) {
    if (c.lane == 0) c.a->weak[c.center] = DPE_UNKNOWN;
    c.live = false;
  }
  return c;
}

// LocalRefine (DPE.cu:2753-2839), phases 2 and 3.  Phase 2 evaluates every (plane, selected
// source) pair as one item, split over the lanes: plane 0 is the current one (the prologue's
// cost), planes 1..11 the disparity samples -5..5; items of samples out of the depth range are
// not evaluated.  Phase 3 sums them in the reference's order.
__device__ __forceinline__ float lr_sample_depth(const PMArgs &a, const SweepPixel &P, int pd) {
  return a.cam[0].K[0] * P.base_line / (P.disp + pd);
}
template <int kStage>
__device__ __forceinline__ void lr_p2(const SweepCtx &c) {
  if (!c.live || !c.P->ok) return;
  const PMArgs &a = *c.a;
  const SweepPixel &P = *c.P;
  const SmemWindow rw = c.window();
  const int na = P.na, n = a.N - 1;
  const bool geom = a.P.geom_consistency != 0;
  for (int i = c.lane; i < 12 * na; i += kCoopLanes) {
    const int h = i / na, q = i - h * na;
    float pdep = P.depth;
    if (h > 0) {
      pdep = lr_sample_depth(a, P, h - 6);
      if (pdep < a.P.depth_min || pdep > a.P.depth_max) continue;
    }
    float4 t = P.pl;
    t.w = dist_to_origin(a.cam[0], c.px, c.py, pdep, t);
    const int si = P.act[q] + 1;
    const float ncc = ncc_strong<kStage, kSweepUnroll>(a, c.px, c.py, si, t, rw);
    c.items[h * n + q] = make_float2(ncc, geom ? geom_cost(a, c.px, c.py, si, t) : 0.0f);
  }
}
__device__ __forceinline__ void lr_p3(const SweepCtx &c) {
  if (!c.live || c.lane != 0 || !c.P->ok) return;
  const PMArgs &a = *c.a;
  const SweepPixel &P = *c.P;
  if (P.weight_normal == 0) return;
  const int na = P.na, n = a.N - 1;
  const bool geom = a.P.geom_consistency != 0;
  float cost_now = 0.0f;
  for (int q = 0; q < na; ++q) {
    const float2 e = c.items[q];
    float tc = e.x;
    if (geom) tc += a.P.geom_factor * e.y;
    cost_now += tc * vweight_at(P.vw, P.act[q]);
  }
  cost_now /= P.weight_normal;
  float min_cost = 2.0f, best = P.depth;
  for (int pd = -5; pd <= 5; ++pd) {
    const float pdep = lr_sample_depth(a, P, pd);
    if (pdep < a.P.depth_min || pdep > a.P.depth_max) continue;
    const float2 *row = c.items + (pd + 6) * n;
    float tc = 0.0f;
    for (int q = 0; q < na; ++q) {
      const int w = vweight_at(P.vw, P.act[q]);
      tc += row[q].x * w;
      if (geom) tc += a.P.geom_factor * row[q].y * w;
    }
    tc /= P.weight_normal;
    if (tc < min_cost) { min_cost = tc; best = pdep; }
  }
  if ((double)(cost_now - min_cost) > 0.1) a.plane[c.center].w = best;
}

// One phase for one thread (host builds run the phases in lock-step over a block).
template <int kStage>
__device__ __forceinline__ void depth_to_weak_phase(int phase, const Launch &lc, void *smem) {
  const SweepCtx c = d2w_ctx(lc, smem);
  switch (phase) {
    case 0: sweep_p0(c); break;
    case 1: sweep_p1(c); break;
    case 2: d2w_p2<kStage>(c); break;
    default: d2w_p3(c); break;
  }
}
template <int kStage>
__device__ __forceinline__ void local_refine_phase(int phase, const Launch &lc, void *smem) {
  const SweepCtx c = sweep_ctx(lc, smem, KID_LOCAL_REFINE);
  switch (phase) {
    case 0: sweep_p0(c); break;
    case 1: sweep_p1(c); break;
    case 2: lr_p2<kStage>(c); break;
    default: lr_p3(c); break;
  }
}

// Grid: ((W + 15) / 16, H) blocks of kCoopThreads.
template <int kStage>
__global__ void __launch_bounds__(kCoopThreads, DPE_SWEEP_MIN_BLOCKS) k_depth_to_weak(const Launch lc) {
  __shared__ SweepPixel sp[kCoopPix];
  const SweepCtx c = d2w_ctx(lc, sp);
  sweep_p0(c);
  __syncthreads();
  sweep_p1(c);
  __syncthreads();
  d2w_p2<kStage>(c);
  __syncthreads();
  d2w_p3(c);
}
// LocalRefine: the same grid, local_refine_smem_bytes(N - 1) dynamic shared bytes.
template <int kStage>
__global__ void __launch_bounds__(kCoopThreads, DPE_COST_MIN_BLOCKS) k_local_refine(const Launch lc) {
  extern __shared__ float4 lr_smem[];
  const SweepCtx c = sweep_ctx(lc, lr_smem, KID_LOCAL_REFINE);
  sweep_p0(c);
  __syncthreads();
  sweep_p1(c);
  __syncthreads();
  lr_p2<kStage>(c);
  __syncthreads();
  lr_p3(c);
}

}  // namespace dpe

