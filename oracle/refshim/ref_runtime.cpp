// ref_runtime.cpp -- HOST STAND-IN (TEST INFRASTRUCTURE: the reference-pinned oracle under
// oracle/_ref): host meanings of the CUDA runtime, cuRAND and OpenCV names declared in this
// directory's headers, for the CPU build of the reference's own DPE.cu and DPE.cpp.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "cuda_runtime.h"
#include "curand_kernel.h"
#include "opencv2/opencv.hpp"
#include "../oracle_common.h"

thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
thread_local dim3 blockDim;
thread_local dim3 gridDim;
long long clock64() { return 0; }

// ------------------------------------------------------------------ launches, textures, RNG
static int g_launch_threads = 1;
int g_ref_tex_8bit = 0;
static int g_rng_width = 0;
static uint32_t g_rng_key[2] = {0, 0};
static std::vector<const void *> g_serial_kernels;
int ref_launch_threads() { return g_launch_threads; }
bool ref_launch_serial(const void *kernel) {
  for (const void *k : g_serial_kernels)
    if (k == kernel) return true;
  return false;
}
// Kernels whose threads read what other threads of the same launch write (the reference's
// same-colour race in the edge-aware strong update) run one thread at a time, in block order.
void ref_set_serial_kernels(const std::vector<const void *> &kernels) { g_serial_kernels = kernels; }

extern "C" void ref_set_launch_threads(int n) { g_launch_threads = n > 0 ? n : 1; }
extern "C" void ref_set_texture_8bit_weights(int on) { g_ref_tex_8bit = on != 0; }

void ref_rng_configure(int width, unsigned long long seed) {
  g_rng_width = width;
  g_rng_key[0] = (uint32_t)seed;
  g_rng_key[1] = (uint32_t)(seed >> 32);
}
// curand_init(clock64(), p.y, p.x, &state) (DPE.cu:1036): subsequence = row, offset = column.
void curand_init(unsigned long long, unsigned long long subsequence, unsigned long long offset, curandState *state) {
  state->pixel = (unsigned)(subsequence * (unsigned long long)g_rng_width + offset);
  state->counter = 0;
}
unsigned int curand(curandState *state) {
  const uint32_t ctr[4] = {state->counter, state->pixel, 0x5EEDu, 0u};
  uint32_t out[4];
  oracle::philox4x32_10(ctr, g_rng_key, out);
  ++state->counter;
  return out[0];
}
float curand_uniform(curandState *state) { return (float)((curand(state) >> 8) + 1u) * (1.0f / 16777216.0f); }

// ------------------------------------------------------------------ device memory
// Every allocation sits between two zero-filled guard zones as large as itself (at least 4 KiB),
// so reads a little outside a buffer read 0.  Writes there are recorded by ref_guard_violations.
namespace {
struct Block {
  unsigned char *base;
  size_t bytes, guard;
};
std::mutex g_mem_mu;
std::map<void *, Block> g_blocks;
}  // namespace

cudaError_t cudaMalloc(void **ptr, size_t bytes) {
  const size_t guard = std::max<size_t>(4096, (bytes + 15) & ~size_t(15));
  unsigned char *base = static_cast<unsigned char *>(std::calloc(bytes + 2 * guard, 1));
  if (!base) return cudaErrorMemoryAllocation;
  *ptr = base + guard;
  std::lock_guard<std::mutex> lock(g_mem_mu);
  g_blocks[*ptr] = Block{base, bytes, guard};
  return cudaSuccess;
}
cudaError_t cudaFree(void *ptr) {
  if (!ptr) return cudaSuccess;
  std::lock_guard<std::mutex> lock(g_mem_mu);
  auto it = g_blocks.find(ptr);
  if (it == g_blocks.end()) return cudaErrorInvalidValue;
  std::free(it->second.base);
  g_blocks.erase(it);
  return cudaSuccess;
}
// Bytes written into any live buffer's guard zones since it was allocated.
extern "C" long long ref_guard_violations() {
  std::lock_guard<std::mutex> lock(g_mem_mu);
  long long n = 0;
  for (const auto &kv : g_blocks) {
    const Block &b = kv.second;
    for (size_t i = 0; i < b.guard; ++i) n += b.base[i] != 0;
    for (size_t i = 0; i < b.guard; ++i) n += b.base[b.guard + b.bytes + i] != 0;
  }
  return n;
}
cudaError_t cudaMemcpy(void *dst, const void *src, size_t bytes, enum cudaMemcpyKind) {
  if (bytes) std::memmove(dst, src, bytes);
  return cudaSuccess;
}
cudaError_t cudaMemset(void *dst, int value, size_t bytes) {
  std::memset(dst, value, bytes);
  return cudaSuccess;
}

// ------------------------------------------------------------------ arrays and textures
cudaChannelFormatDesc cudaCreateChannelDesc(int x, int y, int z, int w, enum cudaChannelFormatKind f) {
  cudaChannelFormatDesc d;
  d.x = x; d.y = y; d.z = z; d.w = w; d.f = f;
  return d;
}
cudaError_t cudaMallocArray(cudaArray_t *array, const cudaChannelFormatDesc *desc, size_t width, size_t height,
                            unsigned int) {
  if (!desc || desc->x != 32 || desc->y || desc->z || desc->w || desc->f != cudaChannelFormatKindFloat)
    return cudaErrorInvalidValue;
  cudaArray *a = new cudaArray;
  a->w = (int)width;
  a->h = (int)(height ? height : 1);
  a->data = new float[(size_t)a->w * a->h]();
  *array = a;
  return cudaSuccess;
}
cudaError_t cudaFreeArray(cudaArray_t array) {
  if (array) delete[] array->data;
  delete array;
  return cudaSuccess;
}
cudaError_t cudaMemcpy2DToArray(cudaArray_t dst, size_t w_offset, size_t h_offset, const void *src, size_t spitch,
                                size_t width_bytes, size_t height, enum cudaMemcpyKind) {
  if (w_offset || h_offset || width_bytes % 4 || (int)(width_bytes / 4) > dst->w || (int)height > dst->h)
    return cudaErrorInvalidValue;
  for (size_t r = 0; r < height; ++r)
    std::memcpy(&dst->data[r * dst->w], static_cast<const unsigned char *>(src) + r * spitch, width_bytes);
  return cudaSuccess;
}
cudaError_t cudaCreateTextureObject(cudaTextureObject_t *tex, const cudaResourceDesc *res, const cudaTextureDesc *desc,
                                    const cudaResourceViewDesc *) {
  if (res->resType != cudaResourceTypeArray) return cudaErrorInvalidValue;
  RefTexture *t = new RefTexture{res->res.array.array, desc->filterMode, desc->normalizedCoords};
  *tex = (cudaTextureObject_t)(uintptr_t)t;
  return cudaSuccess;
}
cudaError_t cudaDestroyTextureObject(cudaTextureObject_t tex) {
  delete reinterpret_cast<RefTexture *>((uintptr_t)tex);
  return cudaSuccess;
}

// ------------------------------------------------------------------ events, errors
struct CUevent_st { int unused; };
cudaError_t cudaEventCreate(cudaEvent_t *ev) { *ev = new CUevent_st{0}; return cudaSuccess; }
cudaError_t cudaEventDestroy(cudaEvent_t ev) { delete ev; return cudaSuccess; }
cudaError_t cudaEventRecord(cudaEvent_t, void *) { return cudaSuccess; }
cudaError_t cudaEventSynchronize(cudaEvent_t) { return cudaSuccess; }
cudaError_t cudaEventElapsedTime(float *ms, cudaEvent_t, cudaEvent_t) { *ms = 0.0f; return cudaSuccess; }
cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }
cudaError_t cudaPeekAtLastError() { return cudaSuccess; }
cudaError_t cudaGetLastError() { return cudaSuccess; }
const char *cudaGetErrorString(cudaError_t e) { return e == cudaSuccess ? "no error" : "host stand-in error"; }

// ------------------------------------------------------------------ OpenCV subset
namespace cv {

int ref_depth_bytes(int depth) {
  static const int b[8] = {1, 1, 2, 2, 4, 4, 8, 2};
  return b[depth & 7];
}

void Mat::create(int r, int c, int type) {
  rows = r;
  cols = c;
  type_ = type;
  step.p[1] = elemSize();
  step.p[0] = (size_t)c * step.p[1];
  buf_ = std::make_shared<std::vector<uchar>>((size_t)r * step.p[0], (uchar)0);
  data = buf_->empty() ? nullptr : buf_->data();
}

template <class T> static void fill_as(uchar *p, size_t n, int cn, const Scalar &s) {
  T *q = reinterpret_cast<T *>(p);
  for (size_t i = 0; i < n; ++i)
    for (int k = 0; k < cn; ++k) q[i * cn + k] = (T)s.val[k < 4 ? k : 3];
}
void Mat::setTo(const Scalar &s) {
  const size_t n = total();
  switch (depth()) {
    case CV_8U: fill_as<uint8_t>(data, n, channels(), s); break;
    case CV_8S: fill_as<int8_t>(data, n, channels(), s); break;
    case CV_16U: fill_as<uint16_t>(data, n, channels(), s); break;
    case CV_16S: fill_as<int16_t>(data, n, channels(), s); break;
    case CV_32S: fill_as<int32_t>(data, n, channels(), s); break;
    case CV_32F: fill_as<float>(data, n, channels(), s); break;
    default: fill_as<double>(data, n, channels(), s); break;
  }
}

Mat Mat::clone() const {
  Mat m(rows, cols, type_);
  if (data && m.data) std::memcpy(m.data, data, (size_t)rows * step.p[0]);
  return m;
}

static double read_elem(const uchar *p, int depth) {
  switch (depth) {
    case CV_8U: return *p;
    case CV_8S: return *reinterpret_cast<const int8_t *>(p);
    case CV_16U: return *reinterpret_cast<const uint16_t *>(p);
    case CV_16S: return *reinterpret_cast<const int16_t *>(p);
    case CV_32S: return *reinterpret_cast<const int32_t *>(p);
    case CV_32F: return *reinterpret_cast<const float *>(p);
    default: return *reinterpret_cast<const double *>(p);
  }
}
template <class T> static T saturate_int(double v, double lo, double hi) {
  v = std::nearbyint(v);
  return (T)(v < lo ? lo : (v > hi ? hi : v));
}
static void write_elem(uchar *p, int depth, double v) {
  switch (depth) {
    case CV_8U: *p = saturate_int<uint8_t>(v, 0, 255); break;
    case CV_8S: *reinterpret_cast<int8_t *>(p) = saturate_int<int8_t>(v, -128, 127); break;
    case CV_16U: *reinterpret_cast<uint16_t *>(p) = saturate_int<uint16_t>(v, 0, 65535); break;
    case CV_16S: *reinterpret_cast<int16_t *>(p) = saturate_int<int16_t>(v, -32768, 32767); break;
    case CV_32S: *reinterpret_cast<int32_t *>(p) = saturate_int<int32_t>(v, -2147483648.0, 2147483647.0); break;
    case CV_32F: *reinterpret_cast<float *>(p) = (float)v; break;
    default: *reinterpret_cast<double *>(p) = v; break;
  }
}
void Mat::convertTo(Mat &dst, int rtype, double alpha, double beta) const {
  const int ddepth = rtype < 0 ? depth() : (rtype & 7);
  Mat out(rows, cols, CV_MAKETYPE(ddepth, channels()));
  const int sb = ref_depth_bytes(depth()), db = ref_depth_bytes(ddepth);
  const size_t n = total() * channels();
  for (size_t i = 0; i < n; ++i) {
    const double v = read_elem(data + i * sb, depth());
    write_elem(out.data + i * db, ddepth, (alpha == 1.0 && beta == 0.0) ? v : v * alpha + beta);
  }
  dst = out;
}

// Binary PGM (P5, gray) / PPM (P6, stored RGB, returned BGR), 8 bits per sample; a gray read
// needs a PGM.
Mat imread(const std::string &filename, int flags) {
  std::ifstream in(filename, std::ios::binary);
  if (!in) return Mat();
  std::string magic;
  int w = 0, h = 0, maxv = 0;
  in >> magic >> w >> h >> maxv;
  in.get();
  if ((magic != "P5" && magic != "P6") || w <= 0 || h <= 0 || maxv != 255) return Mat();
  const int cn = magic == "P6" ? 3 : 1;
  std::vector<uchar> raw((size_t)w * h * cn);
  in.read(reinterpret_cast<char *>(raw.data()), (std::streamsize)raw.size());
  if (!in) return Mat();
  if (flags == IMREAD_GRAYSCALE) {
    if (cn != 1) return Mat();  // the harness stores gray images as PGM
    Mat m(h, w, CV_8UC1);
    std::memcpy(m.data, raw.data(), raw.size());
    return m;
  }
  Mat m(h, w, CV_8UC3);
  for (size_t i = 0; i < (size_t)w * h; ++i) {
    const uchar r = cn == 3 ? raw[3 * i] : raw[i], g = cn == 3 ? raw[3 * i + 1] : raw[i], b = cn == 3 ? raw[3 * i + 2] : raw[i];
    m.data[3 * i] = b; m.data[3 * i + 1] = g; m.data[3 * i + 2] = r;
  }
  return m;
}

[[noreturn]] static void unavailable(const char *what) {
  std::fprintf(stderr, "host build of the reference: cv::%s is not available (never called on the PatchMatch and "
               "fusion paths)\n", what);
  std::abort();
}
bool imwrite(const std::string &, const Mat &, const std::vector<int> &) { unavailable("imwrite"); }
void resize(const Mat &src, Mat &dst, Size dsize, double, double, int) {
  if (dsize.width == src.cols && dsize.height == src.rows) { dst = src.clone(); return; }
  unavailable("resize");
}
double threshold(const Mat &, Mat &, double, double, int) { unavailable("threshold"); }
void Canny(const Mat &, Mat &, double, double, int, bool) { unavailable("Canny"); }
void HoughLinesP(const Mat &, std::vector<Vec4i> &, double, double, int, double, double) { unavailable("HoughLinesP"); }
void line(Mat &, Point, Point, const Scalar &, int) { unavailable("line"); }

}  // namespace cv
