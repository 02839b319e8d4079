// edges.cu -- the edge map of EdgeSegment (DPE.cpp:136-250, mode 0 with use_canny) on the GPU.
//
// GetProblemEdges (main.cpp:166-197) makes the edge map of a pyramid level from the level image
// converted to 8 bits: EdgeSegment takes the median of its histogram (DPE.cpp:193-216), runs
// cv::Canny with thresholds (1 - 0.67) * median and median, a 3x3 aperture and the L2 gradient
// norm (DPE.cpp:217-221), leaves the map at its size (the resize to the same size and the
// threshold at 4 change nothing on a 0 / 255 map) and clears border pixels whose inner neighbour
// is clear (DPE.cpp:239-250).
//
// Canny follows the published algorithm as OpenCV (4.x) implements it:
//   - Sobel derivatives with a replicated border; squared L2 magnitude dx^2 + dy^2 in integers,
//     compared with squared integer thresholds;
//   - non-maximum suppression along the gradient sector, chosen by the fixed-point tangent of
//     22.5 degrees (round(tan(pi/8) * 2^15)); the magnitude must exceed the neighbour before the
//     pixel and be >= the one after it (> both on the diagonals); outside the image the magnitude
//     is 0;
//   - hysteresis: a pixel that survives suppression with magnitude above the low threshold is an
//     edge when its 8-connected component of such pixels holds one above the high threshold.
// The hysteresis is a connected-components pass: union-find over the candidate pixels with
// atomicMin on the roots (the lock-free union of Playne and Hawick, "A new algorithm for
// parallel connected-component labelling on GPUs", IEEE TPDS 2018), then one flag per root.
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "ctx.h"

namespace {

constexpr int kTg22 = 13573;  // round(tan(22.5 deg) * 2^15)

// EdgeSegment's thresholds from the 8-bit histogram (DPE.cpp:193-219), as cv::Canny turns them
// into squared integer bounds for the L2 norm.
struct CannyBounds {
  int low, high;
};

__global__ void k_level_to_u8(const float *__restrict__ src, uint8_t *__restrict__ dst, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  // convertTo(CV_8UC1): round half to even, saturate
  const int v = __float2int_rn(src[i]);
  dst[i] = (uint8_t)(v < 0 ? 0 : v > 255 ? 255 : v);
}

__global__ void k_histogram(const uint8_t *__restrict__ img, int n, unsigned *__restrict__ hist) {
  __shared__ unsigned h[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) atomicAdd(&h[img[i]], 1u);
  __syncthreads();
  for (int i = threadIdx.x; i < 256; i += blockDim.x)
    if (h[i]) atomicAdd(&hist[i], h[i]);
}

__global__ void k_canny_bounds(const unsigned *__restrict__ hist, int n, CannyBounds *b) {
  // the first value whose cumulative count exceeds half the pixels, over 0..254; -1 if none
  const int half = n / 2;
  int median = -1, sum = 0;
  for (int i = 0; i < 255; ++i) {
    sum += (int)hist[i];
    if (sum > half) { median = i; break; }
  }
  const int t1 = (int)((1.0f - 0.67f) * (float)median);  // (1 - sigma) * median_val in float
  const int t2 = median;
  // L2 gradient: thresholds clamped to 32767 and squared when positive; the smaller is low
  int lo = t1 > 0 ? t1 * t1 : t1;
  int hi = t2 > 0 ? t2 * t2 : t2;
  if (lo > hi) { const int t = lo; lo = hi; hi = t; }
  b->low = lo;
  b->high = hi;
}

__device__ __forceinline__ int px_clamped(const uint8_t *img, int w, int h, int x, int y) {
  x = x < 0 ? 0 : x >= w ? w - 1 : x;
  y = y < 0 ? 0 : y >= h ? h - 1 : y;
  return img[y * w + x];
}

// 3x3 Sobel with a replicated border; dx, dy packed as two int16 and the squared magnitude.
__global__ void k_canny_gradient(const uint8_t *__restrict__ img, int w, int h, short2 *__restrict__ grad,
                                 int *__restrict__ mag) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  const int a = px_clamped(img, w, h, x - 1, y - 1), b = px_clamped(img, w, h, x, y - 1),
            c = px_clamped(img, w, h, x + 1, y - 1);
  const int d = px_clamped(img, w, h, x - 1, y), f = px_clamped(img, w, h, x + 1, y);
  const int g = px_clamped(img, w, h, x - 1, y + 1), k = px_clamped(img, w, h, x, y + 1),
            l = px_clamped(img, w, h, x + 1, y + 1);
  const int dx = (c + 2 * f + l) - (a + 2 * d + g);
  const int dy = (g + 2 * k + l) - (a + 2 * b + c);
  grad[y * w + x] = make_short2((short)dx, (short)dy);
  mag[y * w + x] = dx * dx + dy * dy;
}

__device__ __forceinline__ int mag_at(const int *mag, int w, int h, int x, int y) {
  return (x < 0 || x >= w || y < 0 || y >= h) ? 0 : mag[y * w + x];
}

// Non-maximum suppression.  state: 0 not a candidate, 1 candidate, 2 candidate above high.
__global__ void k_canny_suppress(const short2 *__restrict__ grad, const int *__restrict__ mag, int w, int h,
                                 const CannyBounds *__restrict__ bounds, uint8_t *__restrict__ state) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  const int p = y * w + x;
  const int m = mag[p];
  const CannyBounds b = *bounds;
  uint8_t st = 0;
  if (m > b.low) {
    const int xs = grad[p].x, ys = grad[p].y;
    const long long ax = xs < 0 ? -xs : xs;
    const long long ay = (long long)(ys < 0 ? -ys : ys) << 15;
    const long long tg22x = ax * kTg22;
    bool keep;
    if (ay < tg22x) {  // near horizontal gradient: compare left and right
      keep = m > mag_at(mag, w, h, x - 1, y) && m >= mag_at(mag, w, h, x + 1, y);
    } else {
      const long long tg67x = tg22x + (ax << 16);
      if (ay > tg67x) {  // near vertical: above and below
        keep = m > mag_at(mag, w, h, x, y - 1) && m >= mag_at(mag, w, h, x, y + 1);
      } else {  // diagonal: the sign of dx * dy picks the diagonal
        const int s = (xs ^ ys) < 0 ? -1 : 1;
        keep = m > mag_at(mag, w, h, x - s, y - 1) && m > mag_at(mag, w, h, x + s, y + 1);
      }
    }
    if (keep) st = m > b.high ? 2 : 1;
  }
  state[p] = st;
}

__device__ __forceinline__ int uf_find(const int *parent, int i) {
  int p = parent[i];
  while (p != i) {  // indices strictly decrease along the chain
    i = p;
    p = parent[i];
  }
  return i;
}

// Merge the two sets: the larger root is pointed at the smaller by atomicMin; a failed attempt
// (the root moved meanwhile) retries from the new value.  Every retry lowers a root index, so the
// loop ends; the bound below only guards the impossible case.
__device__ __forceinline__ void uf_union(int *parent, int a, int b, int *error) {
  for (int it = 0; it < (1 << 26); ++it) {
    a = uf_find(parent, a);
    b = uf_find(parent, b);
    if (a == b) return;
    if (a < b) { const int t = a; a = b; b = t; }  // a > b: link a under b
    const int old = atomicMin(&parent[a], b);
    if (old == a) return;
    a = old;
  }
  atomicExch(error, 1);
}

__global__ void k_cc_init(const uint8_t *__restrict__ state, int n, int *__restrict__ parent) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) parent[p] = state[p] ? p : -1;
}

// 8-connectivity: each candidate joins its candidate neighbours before it in raster order.
__global__ void k_cc_union(const uint8_t *__restrict__ state, int w, int h, int *parent, int *error) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  const int p = y * w + x;
  if (!state[p]) return;
  if (x > 0 && state[p - 1]) uf_union(parent, p, p - 1, error);
  if (y > 0) {
    if (x > 0 && state[p - w - 1]) uf_union(parent, p, p - w - 1, error);
    if (state[p - w]) uf_union(parent, p, p - w, error);
    if (x + 1 < w && state[p - w + 1]) uf_union(parent, p, p - w + 1, error);
  }
}

__global__ void k_cc_mark(const uint8_t *__restrict__ state, int n, const int *parent, uint8_t *__restrict__ strong) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n && state[p] == 2) strong[uf_find(parent, p)] = 1;
}

__global__ void k_cc_output(const uint8_t *__restrict__ state, int n, const int *parent,
                            const uint8_t *__restrict__ strong, uint8_t *__restrict__ edge) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  edge[p] = (state[p] && strong[uf_find(parent, p)]) ? 255 : 0;
}

// DPE.cpp:239-250: rows first (left and right columns), then columns (top and bottom rows), each
// in the reference's statement order.
__global__ void k_border_rows(uint8_t *d, int w, int h) {
  const int y = blockIdx.x * blockDim.x + threadIdx.x;
  if (y >= h || w < 2) return;
  uint8_t *r = d + (size_t)y * w;
  if (r[1] == 0) r[0] = 0;
  if (r[w - 2] == 0) r[w - 1] = 0;
}
__global__ void k_border_cols(uint8_t *d, int w, int h) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= w || h < 2) return;
  if (d[(size_t)w + x] == 0) d[x] = 0;
  if (d[(size_t)(h - 2) * w + x] == 0) d[(size_t)(h - 1) * w + x] = 0;
}


// =============================================================================================
// The label map of EdgeSegment (DPE.cpp:136-291, mode 1 without Canny), as GetProblemEdges asks
// for it (main.cpp:199-214): from the full-resolution 8-bit image, halved (high_res_img) and
// halved again, a Roberts gradient thresholded at robthr, Connect's labelling, Hough segments
// drawn across every large weak region's outer border, the map resized to the level, thresholded
// and border-ruled, labelled again, and regions up to weak_tex_num pixels marked -1.
// OpenCV's resize, HoughLinesP and line are restated in OpenCV's integer forms (the CPU
// restatement in the test oracle states each rule), so the map is OpenCV's bit for bit.
// =============================================================================================

// cv::resize INTER_LINEAR, 8-bit: source coordinate (d + 0.5) * scale - 0.5 in double rounded to
// float, 11-bit weights rounded half to even; horizontal weights and columns clamped at the
// borders, vertical weights kept and only the rows clamped; the vertical pass in OpenCV's 16-bit
// form.  Explicit roundings keep the compiler from contracting any step.
__device__ __forceinline__ void lin_coeff(int d, double scale, int ssize, bool clamp_weight, int &s0, int &s1,
                                          int &w0, int &w1) {
  float f = __double2float_rn(__dsub_rn(__dmul_rn((double)d + 0.5, scale), 0.5));
  int si = (int)floorf(f);
  f = __fsub_rn(f, (float)si);
  if (clamp_weight) {
    if (si < 0) { f = 0.f; si = 0; }
    if (si >= ssize - 1) { f = 0.f; si = ssize - 1; }
    s0 = si;
    s1 = si + 1 < ssize ? si + 1 : ssize - 1;
  } else {
    s0 = si < 0 ? 0 : si > ssize - 1 ? ssize - 1 : si;
    s1 = si + 1 < 0 ? 0 : si + 1 > ssize - 1 ? ssize - 1 : si + 1;
  }
  w0 = __float2int_rn(__fmul_rn(__fsub_rn(1.f, f), 2048.f));
  w1 = __float2int_rn(__fmul_rn(f, 2048.f));
}

__global__ void k_resize_u8(const uint8_t *__restrict__ src, int sw, int sh, uint8_t *__restrict__ dst, int dw,
                            int dh, double xscale, double yscale) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= dw || y >= dh) return;
  int xa, xb, a0, a1, ya, yb, b0, b1;
  lin_coeff(x, xscale, sw, true, xa, xb, a0, a1);
  lin_coeff(y, yscale, sh, false, ya, yb, b0, b1);
  const uint8_t *r0 = src + (size_t)ya * sw, *r1 = src + (size_t)yb * sw;
  const int h0 = r0[xa] * a0 + r0[xb] * a1, h1 = r1[xa] * a0 + r1[xb] * a1;
  const int v = (((b0 * (h0 >> 4)) >> 16) + ((b1 * (h1 >> 4)) >> 16) + 2) >> 2;
  dst[(size_t)y * dw + x] = (uint8_t)(v < 0 ? 0 : v > 255 ? 255 : v);
}

// Roberts (DPE.cpp:9-25) then cv::threshold(robthr, 255, BINARY): the magnitude is the low byte of
// the truncated root, border pixels use t1 = t2 = 50.
__global__ void k_roberts_threshold(const uint8_t *__restrict__ s, int cols, int rows, int thr, uint8_t *__restrict__ d) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= cols || i >= rows) return;
  int t1 = 50, t2 = 50;
  if (i > 0 && i < rows - 1 && j > 0 && j < cols - 1) {
    t1 = s[(size_t)i * cols + j] - s[(size_t)(i + 1) * cols + j + 1];
    t2 = s[(size_t)(i + 1) * cols + j] - s[(size_t)i * cols + j + 1];
  }
  const uint8_t m = (uint8_t)(int)sqrt((double)(t1 * t1 + t2 * t2));
  d[(size_t)i * cols + j] = m > thr ? 255 : 0;
}

__global__ void k_threshold(uint8_t *d, int n, int thr) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) d[p] = d[p] > thr ? 255 : 0;
}

// ---- Connect (DPE.cpp:27-134) -------------------------------------------------------------
// One CTA walks the rows in order (each row's provisional labels need the previous row's).  In a
// row a pixel opens a new label when it joins neither its left nor its upper neighbour; new labels
// are numbered by a block prefix count.  Along a run of left-joined pixels the provisional label
// is the running minimum of the opening label and the upper labels where the pixel joins upwards:
// a segmented inclusive min-scan, restarted at each pixel without a left join.  A pixel joined to
// both neighbours with different labels records the join connection[larger] = smaller; the
// reference overwrites earlier joins of the same label, so only the last in raster order counts,
// kept as atomicMax of (pixel index << 32 | smaller label).
constexpr int kConnectThreads = 512;

struct SegMin {
  int start;  // a run starts within the scanned prefix
  int v;
};
struct SegMinOp {
  __device__ __forceinline__ SegMin operator()(const SegMin &a, const SegMin &b) const {
    return SegMin{a.start | b.start, b.start ? b.v : min(a.v, b.v)};
  }
};

__global__ void __launch_bounds__(kConnectThreads) k_connect_rows(const uint8_t *__restrict__ img, int cols, int rows,
                                                                 int *__restrict__ lab,
                                                                 unsigned long long *__restrict__ join, int *nlab) {
  typedef cub::BlockScan<int, kConnectThreads> ScanI;
  typedef cub::BlockScan<SegMin, kConnectThreads> ScanS;
  __shared__ typename ScanI::TempStorage ts_i;
  __shared__ typename ScanS::TempStorage ts_s;
  __shared__ int s_next, s_carry;
  const int tid = threadIdx.x;
  if (tid == 0) s_next = 1;
  __syncthreads();
  for (int y = 0; y < rows; ++y) {
    for (int base = 0; base < cols; base += kConnectThreads) {
      const int x = base + tid;
      const bool in = x < cols;
      const size_t p = (size_t)y * cols + x;
      const int v = in ? img[p] : 255;
      const bool labelled = in && v != 255, zero = in && v == 0;
      const bool leftj = zero && x > 0 && img[p - 1] == 0;
      const bool upj = zero && y > 0 && img[p - cols] == 0;
      const bool opens = labelled && !leftj && !upj;
      int pre, total;
      ScanI(ts_i).ExclusiveSum(opens ? 1 : 0, pre, total);
      const int up = upj ? lab[p - cols] : 0;
      const int val = upj ? up : (opens ? s_next + pre : INT_MAX);
      SegMin o;
      ScanS(ts_s).InclusiveScan(SegMin{leftj ? 0 : 1, val}, o, SegMinOp());
      const int run = (o.start || base == 0) ? o.v : min(s_carry, o.v);
      if (in) lab[p] = labelled ? run : 0;
      __syncthreads();  // this chunk's labels are written; s_next and s_carry are read
      if (in && leftj && upj) {
        const int left = lab[p - 1];
        if (left != up) {
          const int big = left > up ? left : up, small = left > up ? up : left;
          atomicMax(&join[big], ((unsigned long long)p << 32) | (unsigned)small);
        }
      }
      if (x == min(base + kConnectThreads, cols) - 1) s_carry = run;
      if (tid == 0) s_next += total;
      __syncthreads();
    }
  }
  if (tid == 0) *nlab = s_next;
}

__global__ void k_connect_links(const unsigned long long *__restrict__ join, const int *nlab, int cap, int *conn) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cap) return;
  conn[i] = (i < *nlab && i > 0 && join[i]) ? (int)(join[i] & 0xffffffffu) : i;
}

// chain ends by pointer doubling (every link points to a smaller label)
__global__ void k_connect_jump(const int *__restrict__ a, int *__restrict__ b, int cap) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < cap) b[i] = a[a[i]];
}

__global__ void k_connect_roots(const int *__restrict__ conn, const int *nlab, int cap, int *__restrict__ is_root) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < cap) is_root[i] = (i > 0 && i < *nlab && conn[i] == i) ? 1 : 0;
}

// final label per pixel (roots renumbered in increasing order) and the count per label
__global__ void k_connect_final(const int *__restrict__ lab, int n, const int *__restrict__ conn,
                                const int *__restrict__ rank, int *__restrict__ out, int *__restrict__ counts) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int l = lab[p];
  const int f = l == 0 ? 0 : rank[conn[l]] + 1;
  out[p] = f;
  atomicAdd(&counts[f], 1);
}

__global__ void k_mark_small(int *labels, int n, const int *__restrict__ counts, int weak_tex_num) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int l = labels[p];
  if (l != 0 && counts[l] <= weak_tex_num) labels[p] = -1;
}

__global__ void k_list_large(const int *__restrict__ counts, int cap, int weak_tex_num, int *list, int *nlist) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 1 && k < cap && counts[k] > 0 && counts[k] >= weak_tex_num) list[atomicAdd(nlist, 1)] = k;
}

// ---- HoughLinesP on one weak region's outer border, and its segments drawn --------------------
// cv::HoughLinesP(img_weak, 1, CV_PI / 180, thr, thr, thr) (DPE.cpp:185-188): OpenCV's progressive
// probabilistic Hough transform.  One CTA per region runs the reference's sequential loop; the
// votes of a point over the angles are spread over the threads, the rest (the generator, the
// segment walks) runs on thread 0.  The walks are bounded by the image, a guard counts steps.
struct HoughArgs {
  const int *labels;  // first labelling, w x h
  const int *regions; // region labels, one per CTA
  int w, h, threshold, line_length, line_gap, numangle, numrho;
  const float2 *tab;  // (cos, sin) / rho in float, from the host's libm as OpenCV computes it
  uint8_t *mask;      // per CTA: w*h
  int2 *points;       // per CTA: w*h
  int *accum;         // per CTA: numangle*numrho
  int4 *lines;        // per CTA: line_cap
  int line_cap;
  uint8_t *dst;       // the thresholded Roberts map the segments are drawn on
  int *error;
};

__device__ __forceinline__ int hough_bin(const HoughArgs &a, float2 t, int x, int y) {
  return __float2int_rn(__fadd_rn(__fmul_rn((float)x, t.x), __fmul_rn((float)y, t.y))) + (a.numrho - 1) / 2;
}

__device__ void draw_line8(uint8_t *img, int width, int x1, int y1, int x2, int y2) {
  int dx = x2 - x1, dy = y2 - y1;
  if (dx < 0) { int t = x1; x1 = x2; x2 = t; t = y1; y1 = y2; y2 = t; dx = -dx; dy = -dy; }
  long long step_y = width, step_x = 1;
  if (dy < 0) { dy = -dy; step_y = -step_y; }
  if (dy > dx) { int t = dx; dx = dy; dy = t; const long long u = step_x; step_x = step_y; step_y = u; }
  int err = dx - (dy + dy);
  const int plus_delta = dx + dx, minus_delta = -(dy + dy);
  long long p = (long long)y1 * width + x1;
  for (int c = 0; c <= dx; ++c) {
    img[p] = 255;
    const bool m = err < 0;
    err += minus_delta + (m ? plus_delta : 0);
    p += step_x + (m ? step_y : 0);
  }
}

constexpr int kHoughThreads = 256;

__global__ void __launch_bounds__(kHoughThreads) k_hough_region(const __grid_constant__ HoughArgs a) {
  extern __shared__ int2 walk[];  // pixels withdrawn by one segment, both directions
  typedef cub::BlockScan<int, kHoughThreads> ScanI;
  typedef cub::BlockReduce<unsigned long long, kHoughThreads> RedU;
  __shared__ typename ScanI::TempStorage ts_i;
  __shared__ typename RedU::TempStorage ts_r;
  __shared__ int s_count, s_idx_x, s_idx_y, s_skip, s_nwalk, s_good, s_nlines, s_best_n, s_best_v;
  const int tid = threadIdx.x;
  const int region = a.regions[blockIdx.x];
  const int w = a.w, h = a.h, n = w * h;
  uint8_t *mask = a.mask + (size_t)blockIdx.x * n;
  int2 *pts = a.points + (size_t)blockIdx.x * n;
  int *acc = a.accum + (size_t)blockIdx.x * a.numangle * a.numrho;
  int4 *lines = a.lines + (size_t)blockIdx.x * a.line_cap;
  const int walk_cap = 2 * (max(w, h) + 2);
  // the region's outer border in raster order (DPE.cpp:168-182): not the region, 4-adjacent to it
  if (tid == 0) s_count = 0;
  __syncthreads();
  for (int base = 0; base < n; base += kHoughThreads) {
    const int p = base + tid;
    bool on = false;
    if (p < n && a.labels[p] != region) {
      const int x = p % w, y = p / w;
      on = (x > 0 && a.labels[p - 1] == region) || (x < w - 1 && a.labels[p + 1] == region) ||
           (y > 0 && a.labels[p - w] == region) || (y < h - 1 && a.labels[p + w] == region);
    }
    int pre, total;
    ScanI(ts_i).ExclusiveSum(on ? 1 : 0, pre, total);
    if (p < n) mask[p] = on ? 1 : 0;
    if (on) pts[s_count + pre] = make_int2(p % w, p / w);
    __syncthreads();
    if (tid == 0) s_count += total;
    __syncthreads();
  }
  for (int i = tid; i < a.numangle * a.numrho; i += kHoughThreads) acc[i] = 0;
  if (tid == 0) s_nlines = 0;
  __syncthreads();
  uint64_t state = ~0ull;  // cv::RNG((uint64)-1), thread 0 only
  const int shift = 16;
  for (int count = s_count; count > 0; --count) {
    // Every thread has read the previous point's shared values (s_skip, s_idx_*, s_best_*) before
    // thread 0 overwrites them: the `continue`s below leave an iteration without a later barrier.
    __syncthreads();
    if (tid == 0) {
      state = (uint64_t)(unsigned)state * 4164903690u + (unsigned)(state >> 32);
      const int idx = (int)((unsigned)state % (unsigned)count);
      const int2 pt = pts[idx];
      pts[idx] = pts[count - 1];
      s_idx_x = pt.x;
      s_idx_y = pt.y;
      s_skip = mask[pt.y * w + pt.x] ? 0 : 1;
    }
    __syncthreads();
    if (s_skip) continue;  // uniform: already withdrawn by an earlier segment
    const int j = s_idx_x, i = s_idx_y;
    // vote, and the first angle with the largest count.  Counts can be negative: a segment
    // withdraws the votes of every mask pixel on it, also of pixels that have not voted yet (as
    // OpenCV does).  The key's high word is the count with its sign bit flipped, so unsigned
    // order is the counts' signed order; the low word prefers the smaller angle on ties.
    unsigned long long best = 0;
    for (int nn = tid; nn < a.numangle; nn += kHoughThreads) {
      const int r = hough_bin(a, a.tab[nn], j, i);
      const int val = ++acc[(size_t)nn * a.numrho + r];
      const unsigned long long key =
          ((unsigned long long)((unsigned)val ^ 0x80000000u) << 32) | (unsigned)(0x7fffffff - nn);
      best = key > best ? key : best;
    }
    best = RedU(ts_r).Reduce(best, cub::Max());
    if (tid == 0) {
      s_best_v = (int)((unsigned)(best >> 32) ^ 0x80000000u);
      s_best_n = 0x7fffffff - (int)(best & 0xffffffffu);
    }
    __syncthreads();
    if (s_best_v < a.threshold) continue;  // uniform
    if (tid == 0) {
      const float2 t = a.tab[s_best_n];
      const float fa = -t.y, fb = t.x;
      int x0 = j, y0 = i, dx0, dy0;
      bool xflag;
      if (fabsf(fa) > fabsf(fb)) {
        xflag = true;
        dx0 = fa > 0 ? 1 : -1;
        dy0 = __float2int_rn(__fdiv_rn(__fmul_rn(fb, (float)(1 << shift)), fabsf(fa)));
        y0 = (y0 << shift) + (1 << (shift - 1));
      } else {
        xflag = false;
        dy0 = fb > 0 ? 1 : -1;
        dx0 = __float2int_rn(__fdiv_rn(__fmul_rn(fa, (float)(1 << shift)), fabsf(fb)));
        x0 = (x0 << shift) + (1 << (shift - 1));
      }
      int ex[2] = {j, j}, ey[2] = {i, i};
      for (int k = 0; k < 2; ++k) {
        int gap = 0, x = x0, y = y0;
        const int dx = k ? -dx0 : dx0, dy = k ? -dy0 : dy0;
        for (int step = 0;; x += dx, y += dy, ++step) {
          const int j1 = xflag ? x : x >> shift, i1 = xflag ? y >> shift : y;
          if (j1 < 0 || j1 >= w || i1 < 0 || i1 >= h) break;
          if (mask[i1 * w + j1]) {
            gap = 0;
            ex[k] = j1;
            ey[k] = i1;
          } else if (++gap > a.line_gap) {
            break;
          }
          if (step > w + h + 4) { atomicExch(a.error, 1); break; }
        }
      }
      const bool good = abs(ex[1] - ex[0]) >= a.line_length || abs(ey[1] - ey[0]) >= a.line_length;
      int nw = 0;
      for (int k = 0; k < 2; ++k) {
        int x = x0, y = y0;
        const int dx = k ? -dx0 : dx0, dy = k ? -dy0 : dy0;
        for (int step = 0;; x += dx, y += dy, ++step) {
          const int j1 = xflag ? x : x >> shift, i1 = xflag ? y >> shift : y;
          if (j1 < 0 || j1 >= w || i1 < 0 || i1 >= h || step > w + h + 4) { atomicExch(a.error, 1); break; }
          uint8_t &m = mask[i1 * w + j1];
          if (m) {
            if (good && nw < walk_cap) walk[nw++] = make_int2(j1, i1);
            m = 0;
          }
          if (i1 == ey[k] && j1 == ex[k]) break;
        }
      }
      s_nwalk = good ? nw : 0;
      s_good = good ? 1 : 0;
      if (good && s_nlines < a.line_cap) lines[s_nlines] = make_int4(ex[0], ey[0], ex[1], ey[1]);
      if (good) s_nlines++;
    }
    __syncthreads();
    // withdraw the segment's votes: each thread owns whole angle rows, so no two threads meet
    for (int q = 0; q < s_nwalk; ++q) {
      const int2 pq = walk[q];
      for (int nn = tid; nn < a.numangle; nn += kHoughThreads)
        --acc[(size_t)nn * a.numrho + hough_bin(a, a.tab[nn], pq.x, pq.y)];
    }
    __syncthreads();
  }
  __syncthreads();
  if (s_nlines > a.line_cap && tid == 0) atomicExch(a.error, 2);
  const int nl = min(s_nlines, a.line_cap);
  for (int q = tid; q < nl; q += kHoughThreads) draw_line8(a.dst, w, lines[q].x, lines[q].y, lines[q].z, lines[q].w);
}
}  // namespace

int dpe_edge_reserve(dpe_ctx *ctx, size_t pixels) {
  Arena &A = ctx->arena;
  A.get<uint8_t>("eg_u8", pixels);
  A.get<short2>("eg_grad", pixels);
  A.get<int>("eg_mag", pixels);
  A.get<uint8_t>("eg_state", pixels);
  A.get<int>("eg_parent", pixels);
  A.get<uint8_t>("eg_strong", pixels);
  A.get<unsigned>("eg_hist", 256);
  A.get<CannyBounds>("eg_bounds", 1);
  A.get<int>("eg_error", 1);
  return A.ok() ? DPE_OK : DPE_ERR_OUT_OF_MEMORY;
}

int dpe_edge_map_device(dpe_ctx *ctx, const float *level, const uint8_t *image, int w, int h, uint8_t *edge) {
  const int n = w * h;
  cudaStream_t s = ctx->stream;
  Arena &A = ctx->arena;
  uint8_t *u8 = A.get<uint8_t>("eg_u8", n);
  short2 *grad = A.get<short2>("eg_grad", n);
  int *mag = A.get<int>("eg_mag", n);
  uint8_t *state = A.get<uint8_t>("eg_state", n);
  int *parent = A.get<int>("eg_parent", n);
  uint8_t *strong = A.get<uint8_t>("eg_strong", n);
  unsigned *hist = A.get<unsigned>("eg_hist", 256);
  CannyBounds *bounds = A.get<CannyBounds>("eg_bounds", 1);
  int *error = A.get<int>("eg_error", 1);
  if (!A.ok()) return DPE_ERR_OUT_OF_MEMORY;
  const unsigned b1 = (unsigned)((n + 255) / 256);
  const dim3 bl(32, 8), g2((w + 31) / 32, (h + 7) / 8);
  if (level) {
    k_level_to_u8<<<b1, 256, 0, s>>>(level, u8, n);
    DPE_LAUNCHED("k_level_to_u8", s);
    image = u8;
  }
  DPE_TRY(cudaMemsetAsync(hist, 0, 256 * sizeof(unsigned), s));
  DPE_TRY(cudaMemsetAsync(strong, 0, (size_t)n, s));
  DPE_TRY(cudaMemsetAsync(error, 0, sizeof(int), s));
  DPE_TIMED(ctx, KID_EDGE_MAP, s, k_histogram<<<(unsigned)std::min(b1, 2u * (unsigned)ctx->sms), 256, 0, s>>>(image, n, hist));
  DPE_LAUNCHED("k_histogram", s);
  k_canny_bounds<<<1, 1, 0, s>>>(hist, n, bounds);
  DPE_LAUNCHED("k_canny_bounds", s);
  DPE_TIMED(ctx, KID_EDGE_MAP, s, k_canny_gradient<<<g2, bl, 0, s>>>(image, w, h, grad, mag));
  DPE_LAUNCHED("k_canny_gradient", s);
  DPE_TIMED(ctx, KID_EDGE_MAP, s, k_canny_suppress<<<g2, bl, 0, s>>>(grad, mag, w, h, bounds, state));
  DPE_LAUNCHED("k_canny_suppress", s);
  k_cc_init<<<b1, 256, 0, s>>>(state, n, parent);
  DPE_LAUNCHED("k_cc_init", s);
  DPE_TIMED(ctx, KID_EDGE_MAP, s, k_cc_union<<<g2, bl, 0, s>>>(state, w, h, parent, error));
  DPE_LAUNCHED("k_cc_union", s);
  k_cc_mark<<<b1, 256, 0, s>>>(state, n, parent, strong);
  DPE_LAUNCHED("k_cc_mark", s);
  DPE_TIMED(ctx, KID_EDGE_MAP, s, k_cc_output<<<b1, 256, 0, s>>>(state, n, parent, strong, edge));
  DPE_LAUNCHED("k_cc_output", s);
  k_border_rows<<<(unsigned)((h + 255) / 256), 256, 0, s>>>(edge, w, h);
  DPE_LAUNCHED("k_border_rows", s);
  k_border_cols<<<(unsigned)((w + 255) / 256), 256, 0, s>>>(edge, w, h);
  DPE_LAUNCHED("k_border_cols", s);
  return DPE_OK;
}

// The union loop's guard (never expected to trip): read after the caller has synchronised.
int dpe_edge_check(dpe_ctx *ctx) {
  int *error = ctx->arena.get<int>("eg_error", 1);
  int e = 0;
  DPE_TRY(cudaMemcpy(&e, error, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    dpe_set_last_error("k_cc_union", cudaErrorUnknown, __FILE__, __LINE__);
    return DPE_ERR_CUDA;
  }
  return DPE_OK;
}

extern "C" int dpe_edge_map(dpe_ctx *ctx, const uint8_t *image, int width, int height, int memory, uint8_t *edge_out) {
  if (!ctx || !image || !edge_out || width < 1 || height < 1) return DPE_ERR_INVALID_ARGUMENT;
  if (memory != DPE_MEM_HOST && memory != DPE_MEM_DEVICE) return DPE_ERR_INVALID_ARGUMENT;
  if ((size_t)width * height > (size_t)INT_MAX / 2) return DPE_ERR_INVALID_ARGUMENT;
  DPE_TRY(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  const size_t n = (size_t)width * height;
  const uint8_t *img = image;
  uint8_t *out = edge_out;
  if (memory == DPE_MEM_HOST) {
    uint8_t *in_d = ctx->arena.get<uint8_t>("eg_in", n);
    uint8_t *out_d = ctx->arena.get<uint8_t>("eg_out", n);
    if (!ctx->arena.ok()) return DPE_ERR_OUT_OF_MEMORY;
    DPE_TRY(cudaMemcpyAsync(in_d, image, n, cudaMemcpyHostToDevice, s));
    img = in_d;
    out = out_d;
  }
  DPE_TRY(cudaEventRecord(ctx->ev0, s));
  int st = dpe_edge_map_device(ctx, nullptr, img, width, height, out);
  if (st != DPE_OK) return st;
  DPE_TRY(cudaEventRecord(ctx->ev1, s));
  if (memory == DPE_MEM_HOST) DPE_TRY(cudaMemcpyAsync(edge_out, out, n, cudaMemcpyDeviceToHost, s));
  DPE_TRY(cudaStreamSynchronize(s));
  ctx->collect();
  return dpe_edge_check(ctx);
}

// ---------------------------------------------------------------------------------------------
// Label maps on the device.
// ---------------------------------------------------------------------------------------------
namespace {

struct ConnectScratch {
  int *lab, *conn_a, *conn_b, *is_root, *rank, *nlab;
  unsigned long long *join;
  void *scan_tmp;
  size_t scan_bytes;
};

int connect_scratch(dpe_ctx *ctx, size_t pixels, ConnectScratch &c) {
  Arena &A = ctx->arena;
  const size_t cap = pixels + 1;
  c.lab = A.get<int>("lb_lab", pixels);
  c.conn_a = A.get<int>("lb_conn_a", cap);
  c.conn_b = A.get<int>("lb_conn_b", cap);
  c.is_root = A.get<int>("lb_is_root", cap);
  c.rank = A.get<int>("lb_rank", cap);
  c.nlab = A.get<int>("lb_nlab", 1);
  c.join = A.get<unsigned long long>("lb_join", cap);
  c.scan_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, c.scan_bytes, c.is_root, c.rank, (int)cap, ctx->stream);
  c.scan_tmp = A.get<uint8_t>("lb_scan_tmp", c.scan_bytes + 16);
  return A.ok() ? DPE_OK : DPE_ERR_OUT_OF_MEMORY;
}

// Connect (DPE.cpp:27-134) of a w x h map: final labels into `out`, pixels per label into
// `counts` (w*h + 1 entries, label 0 = the 255 pixels).
int connect_device(dpe_ctx *ctx, const uint8_t *img, int w, int h, ConnectScratch &c, int *out, int *counts) {
  cudaStream_t s = ctx->stream;
  const int n = w * h, cap = n + 1;
  const unsigned bn = (unsigned)((n + 255) / 256), bc = (unsigned)((cap + 255) / 256);
  DPE_TRY(cudaMemsetAsync(c.join, 0, (size_t)cap * sizeof(unsigned long long), s));
  DPE_TIMED(ctx, KID_EDGE_LABELS, s, k_connect_rows<<<1, kConnectThreads, 0, s>>>(img, w, h, c.lab, c.join, c.nlab));
  DPE_LAUNCHED("k_connect_rows", s);
  k_connect_links<<<bc, 256, 0, s>>>(c.join, c.nlab, cap, c.conn_a);
  DPE_LAUNCHED("k_connect_links", s);
  int *a = c.conn_a, *b = c.conn_b;
  for (int span = 1; span < 2 * cap; span *= 2) {  // ceil(log2(cap)) + 1 doublings
    k_connect_jump<<<bc, 256, 0, s>>>(a, b, cap);
    DPE_LAUNCHED("k_connect_jump", s);
    std::swap(a, b);
  }
  k_connect_roots<<<bc, 256, 0, s>>>(a, c.nlab, cap, c.is_root);
  DPE_LAUNCHED("k_connect_roots", s);
  size_t nb = c.scan_bytes;
  DPE_TRY(cub::DeviceScan::ExclusiveSum(c.scan_tmp, nb, c.is_root, c.rank, cap, s));
  DPE_TRY(cudaMemsetAsync(counts, 0, (size_t)cap * sizeof(int), s));
  k_connect_final<<<bn, 256, 0, s>>>(c.lab, n, a, c.rank, out, counts);
  DPE_LAUNCHED("k_connect_final", s);
  return DPE_OK;
}

void resize_u8_launch(cudaStream_t s, const uint8_t *src, int sw, int sh, uint8_t *dst, int dw, int dh) {
  const dim3 bl(32, 8), g((dw + 31) / 32, (dh + 7) / 8);
  k_resize_u8<<<g, bl, 0, s>>>(src, sw, sh, dst, dw, dh, 1.0 / ((double)dw / sw), 1.0 / ((double)dh / sh));
}

}  // namespace

int dpe_edge_labels_device(dpe_ctx *ctx, const uint8_t *gray, int W, int H, int scale, int high_res_img, int32_t *out,
                           int ow, int oh) {
  cudaStream_t s = ctx->stream;
  Arena &A = ctx->arena;
  const int robthr = high_res_img ? 4 : 6;
  const int weak_tex_num = (int)(1.0 * H * W / (1024 << scale << scale));
  const int c1 = high_res_img ? W / 2 : W, r1 = high_res_img ? H / 2 : H;
  const int c2 = c1 / 2, r2 = r1 / 2;
  const float factor = 1.0f / (float)(1 << scale);
  if ((int)std::round(W * factor) != ow || (int)std::round(H * factor) != oh) return DPE_ERR_INVALID_ARGUMENT;
  if (c2 < 1 || r2 < 1 || ow < 3 || oh < 3) return DPE_ERR_INVALID_ARGUMENT;
  const size_t n_full = (size_t)W * H, n2 = (size_t)c2 * r2, n_out = (size_t)ow * oh;
  uint8_t *half = high_res_img ? A.get<uint8_t>("lb_half", (size_t)c1 * r1) : nullptr;
  uint8_t *down = A.get<uint8_t>("lb_down", n2);
  uint8_t *dst = A.get<uint8_t>("lb_dst", n2);
  uint8_t *up = A.get<uint8_t>("lb_up", n_out);
  int *lab0 = A.get<int>("lb_lab0", n2);
  int *counts = A.get<int>("lb_counts", std::max(n2, n_out) + 1);
  int *regions = A.get<int>("lb_regions", n2 + 1);
  int *nregions = A.get<int>("lb_nregions", 1);
  int *error = A.get<int>("lb_error", 1);
  if (!A.ok()) return DPE_ERR_OUT_OF_MEMORY;
  ConnectScratch cs;
  int st = connect_scratch(ctx, std::max(n2, n_out), cs);
  if (st != DPE_OK) return st;
  (void)n_full;

  // halve (high_res_img), halve again, Roberts > robthr (DPE.cpp:141-160)
  const uint8_t *s1 = gray;
  if (high_res_img) {
    resize_u8_launch(s, gray, W, H, half, c1, r1);
    DPE_LAUNCHED("k_resize_u8", s);
    s1 = half;
  }
  resize_u8_launch(s, s1, c1, r1, down, c2, r2);
  DPE_LAUNCHED("k_resize_u8", s);
  {
    const dim3 bl(32, 8), g((c2 + 31) / 32, (r2 + 7) / 8);
    k_roberts_threshold<<<g, bl, 0, s>>>(down, c2, r2, robthr, dst);
    DPE_LAUNCHED("k_roberts_threshold", s);
  }
  // first labelling and the large weak regions (DPE.cpp:162-166)
  if ((st = connect_device(ctx, dst, c2, r2, cs, lab0, counts)) != DPE_OK) return st;
  DPE_TRY(cudaMemsetAsync(nregions, 0, sizeof(int), s));
  DPE_TRY(cudaMemsetAsync(error, 0, sizeof(int), s));
  k_list_large<<<(unsigned)((n2 + 1 + 255) / 256), 256, 0, s>>>(counts, (int)n2 + 1, weak_tex_num, regions, nregions);
  DPE_LAUNCHED("k_list_large", s);
  int nreg = 0;
  DPE_TRY(cudaMemcpyAsync(&nreg, nregions, sizeof(int), cudaMemcpyDeviceToHost, s));
  DPE_TRY(cudaStreamSynchronize(s));
  if (nreg > 0) {
    // Hough segments across each region's border, drawn on the Roberts map (DPE.cpp:164-190)
    const int thr = (int)(std::min(c2, r2) / 30.0);
    const float theta = (float)(3.14159265358979323846 / 180.0);
    int numangle = (int)std::floor(3.14159265358979323846 / theta) + 1;
    if (numangle > 1 && std::fabs(3.14159265358979323846 - (numangle - 1) * (double)theta) < theta / 2) --numangle;
    const int numrho = (int)std::nearbyint((double)((c2 + r2) * 2 + 1));
    std::vector<float2> tab(numangle);
    for (int k = 0; k < numangle; ++k)
      tab[k] = make_float2((float)(std::cos((double)k * theta) * 1.0f), (float)(std::sin((double)k * theta) * 1.0f));
    float2 *tab_d = A.get<float2>("lb_tab", numangle);
    const int line_cap = (int)(n2 / (size_t)std::max(1, thr)) + 16;
    HoughArgs ha;
    ha.labels = lab0;
    ha.regions = regions;
    ha.w = c2; ha.h = r2; ha.threshold = thr; ha.line_length = thr; ha.line_gap = thr;
    ha.numangle = numangle; ha.numrho = numrho;
    ha.tab = tab_d;
    ha.mask = A.get<uint8_t>("lb_mask", n2 * nreg);
    ha.points = A.get<int2>("lb_points", n2 * nreg);
    ha.accum = A.get<int>("lb_accum", (size_t)numangle * numrho * nreg);
    ha.lines = A.get<int4>("lb_lines", (size_t)line_cap * nreg);
    ha.line_cap = line_cap;
    ha.dst = dst;
    ha.error = error;
    if (!A.ok()) return DPE_ERR_OUT_OF_MEMORY;
    DPE_TRY(cudaMemcpyAsync(tab_d, tab.data(), numangle * sizeof(float2), cudaMemcpyHostToDevice, s));
    const size_t walk_bytes = (size_t)2 * (std::max(c2, r2) + 2) * sizeof(int2);
    if (walk_bytes > 48 * 1024)
      DPE_TRY(cudaFuncSetAttribute(k_hough_region, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)walk_bytes));
    DPE_TIMED(ctx, KID_EDGE_LABELS, s, k_hough_region<<<nreg, kHoughThreads, walk_bytes, s>>>(ha));
    DPE_LAUNCHED("k_hough_region", s);
  }
  // to the level, threshold, border rule, second labelling, small regions -1 (DPE.cpp:224-285)
  resize_u8_launch(s, dst, c2, r2, up, ow, oh);
  DPE_LAUNCHED("k_resize_u8", s);
  k_threshold<<<(unsigned)((n_out + 255) / 256), 256, 0, s>>>(up, (int)n_out, robthr);
  DPE_LAUNCHED("k_threshold", s);
  k_border_rows<<<(unsigned)((oh + 255) / 256), 256, 0, s>>>(up, ow, oh);
  DPE_LAUNCHED("k_border_rows", s);
  k_border_cols<<<(unsigned)((ow + 255) / 256), 256, 0, s>>>(up, ow, oh);
  DPE_LAUNCHED("k_border_cols", s);
  if ((st = connect_device(ctx, up, ow, oh, cs, out, counts)) != DPE_OK) return st;
  k_mark_small<<<(unsigned)((n_out + 255) / 256), 256, 0, s>>>(out, (int)n_out, counts, weak_tex_num);
  DPE_LAUNCHED("k_mark_small", s);
  return DPE_OK;
}

// The Hough guards (never expected to trip): read after the caller has synchronised.
int dpe_edge_labels_check(dpe_ctx *ctx) {
  int *error = ctx->arena.get<int>("lb_error", 1);
  int e = 0;
  DPE_TRY(cudaMemcpy(&e, error, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    dpe_set_last_error("k_hough_region", cudaErrorUnknown, __FILE__, __LINE__);
    return DPE_ERR_CUDA;
  }
  return DPE_OK;
}

extern "C" int dpe_edge_labels(dpe_ctx *ctx, const uint8_t *gray, int width, int height, int scale, int high_res_img,
                               int memory, int32_t *labels_out) {
  if (!ctx || !gray || !labels_out || width < 4 || height < 4 || scale < 0 || scale > 8) return DPE_ERR_INVALID_ARGUMENT;
  if (memory != DPE_MEM_HOST && memory != DPE_MEM_DEVICE) return DPE_ERR_INVALID_ARGUMENT;
  if ((size_t)width * height > (size_t)INT_MAX / 4) return DPE_ERR_INVALID_ARGUMENT;
  const float factor = 1.0f / (float)(1 << scale);
  const int ow = (int)std::round(width * factor), oh = (int)std::round(height * factor);
  DPE_TRY(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  const size_t n = (size_t)width * height, no = (size_t)ow * oh;
  const uint8_t *img = gray;
  int32_t *out = labels_out;
  if (memory == DPE_MEM_HOST) {
    uint8_t *in_d = ctx->arena.get<uint8_t>("lb_in", n);
    int32_t *out_d = ctx->arena.get<int32_t>("lb_out", no);
    if (!ctx->arena.ok()) return DPE_ERR_OUT_OF_MEMORY;
    DPE_TRY(cudaMemcpyAsync(in_d, gray, n, cudaMemcpyHostToDevice, s));
    img = in_d;
    out = out_d;
  }
  int st = dpe_edge_labels_device(ctx, img, width, height, scale, high_res_img ? 1 : 0, out, ow, oh);
  if (st != DPE_OK) return st;
  if (memory == DPE_MEM_HOST) DPE_TRY(cudaMemcpyAsync(labels_out, out, no * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  DPE_TRY(cudaStreamSynchronize(s));
  ctx->collect();
  return dpe_edge_labels_check(ctx);
}
