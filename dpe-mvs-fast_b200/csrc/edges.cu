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
#include <algorithm>
#include <climits>
#include <cstring>

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
