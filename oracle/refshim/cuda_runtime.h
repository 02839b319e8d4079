// cuda_runtime.h -- HOST STAND-IN used only to compile the reference's own DPE.cu / DPE.cpp for the
// CPU (TEST INFRASTRUCTURE: the reference-pinned oracle under oracle/_ref).  It declares the names
// and signatures of the small part of the CUDA runtime those files use; ref_runtime.cpp gives
// them host meanings:
//   * device memory is host memory with zero-filled guard zones on both sides, so the reference's
//     documented reads just outside its buffers read 0 instead of faulting;
//   * a 2D float array plus a texture object is a clamp-to-edge, linearly filtered image whose
//     bilinear weights are exact floats (or, selectable, quantised to 8 fractional bits like the
//     texture unit), sampled by tex2D<float>;
//   * a kernel launch runs every thread of every block on the host, blocks in parallel when the
//     harness allows it (the reference's kernels use no shared memory and no block barriers).
// Nothing here is CUDA's code: these are the documented interfaces, written for the host.
#ifndef REFSHIM_CUDA_RUNTIME_H_
#define REFSHIM_CUDA_RUNTIME_H_

#include <cfloat>  // CUDA's headers make FLT_MAX / FLT_EPSILON visible
#include <climits>
#include <cstddef>
#include <cstdint>
#include <cstring>

#define __host__
#define __device__
#define __global__
#define __forceinline__ inline
#define __constant__

// ---- vector types (CUDA's sizes and alignments)
struct alignas(8) float2 { float x, y; };
struct float3 { float x, y, z; };
struct alignas(16) float4 { float x, y, z, w; };
struct alignas(8) int2 { int x, y; };
struct alignas(4) short2 { short x, y; };
struct uint3 { unsigned int x, y, z; };
struct dim3 {
  unsigned int x, y, z;
  dim3(unsigned int a = 1, unsigned int b = 1, unsigned int c = 1) : x(a), y(b), z(c) {}
};
inline float2 make_float2(float x, float y) { return float2{x, y}; }
inline float3 make_float3(float x, float y, float z) { return float3{x, y, z}; }
inline float4 make_float4(float x, float y, float z, float w) { return float4{x, y, z, w}; }
inline int2 make_int2(int x, int y) { return int2{x, y}; }
inline short2 make_short2(short x, short y) { return short2{x, y}; }

// ---- built-in thread coordinates: set per simulated thread by the launcher
extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;
extern thread_local dim3 blockDim;
extern thread_local dim3 gridDim;
long long clock64();

// ---- runtime API subset
enum cudaError { cudaSuccess = 0, cudaErrorInvalidValue = 1, cudaErrorMemoryAllocation = 2 };
typedef enum cudaError cudaError_t;
enum cudaMemcpyKind {
  cudaMemcpyHostToHost = 0,
  cudaMemcpyHostToDevice = 1,
  cudaMemcpyDeviceToHost = 2,
  cudaMemcpyDeviceToDevice = 3,
  cudaMemcpyDefault = 4
};
enum cudaChannelFormatKind { cudaChannelFormatKindSigned = 0, cudaChannelFormatKindUnsigned = 1, cudaChannelFormatKindFloat = 2 };
struct cudaChannelFormatDesc { int x, y, z, w; enum cudaChannelFormatKind f; };
struct cudaArray {  // a W x H float image
  int w, h;
  float *data;
};
typedef struct cudaArray *cudaArray_t;
enum cudaResourceType { cudaResourceTypeArray = 0, cudaResourceTypeMipmappedArray = 1, cudaResourceTypeLinear = 2, cudaResourceTypePitch2D = 3 };
struct cudaResourceDesc {
  enum cudaResourceType resType;
  union {
    struct { cudaArray_t array; } array;
    struct { void *devPtr; size_t sizeInBytes; } linear;
  } res;
};
enum cudaTextureAddressMode { cudaAddressModeWrap = 0, cudaAddressModeClamp = 1, cudaAddressModeMirror = 2, cudaAddressModeBorder = 3 };
enum cudaTextureFilterMode { cudaFilterModePoint = 0, cudaFilterModeLinear = 1 };
enum cudaTextureReadMode { cudaReadModeElementType = 0, cudaReadModeNormalizedFloat = 1 };
struct cudaTextureDesc {
  enum cudaTextureAddressMode addressMode[3];
  enum cudaTextureFilterMode filterMode;
  enum cudaTextureReadMode readMode;
  int sRGB;
  float borderColor[4];
  int normalizedCoords;
  unsigned int maxAnisotropy;
  int mipmapFilterMode;
  float mipmapLevelBias, minMipmapLevelClamp, maxMipmapLevelClamp;
  int disableTrilinearOptimization;
  int seamlessCubemap;
};
struct cudaResourceViewDesc;
typedef unsigned long long cudaTextureObject_t;
typedef struct CUevent_st *cudaEvent_t;

cudaChannelFormatDesc cudaCreateChannelDesc(int x, int y, int z, int w, enum cudaChannelFormatKind f);
cudaError_t cudaMalloc(void **ptr, size_t bytes);
cudaError_t cudaFree(void *ptr);
cudaError_t cudaMemcpy(void *dst, const void *src, size_t bytes, enum cudaMemcpyKind kind);
cudaError_t cudaMemset(void *dst, int value, size_t bytes);
cudaError_t cudaMallocArray(cudaArray_t *array, const cudaChannelFormatDesc *desc, size_t width, size_t height = 0,
                            unsigned int flags = 0);
cudaError_t cudaFreeArray(cudaArray_t array);
cudaError_t cudaMemcpy2DToArray(cudaArray_t dst, size_t w_offset, size_t h_offset, const void *src, size_t spitch,
                                size_t width_bytes, size_t height, enum cudaMemcpyKind kind);
cudaError_t cudaCreateTextureObject(cudaTextureObject_t *tex, const cudaResourceDesc *res, const cudaTextureDesc *desc,
                                    const cudaResourceViewDesc *view);
cudaError_t cudaDestroyTextureObject(cudaTextureObject_t tex);
cudaError_t cudaEventCreate(cudaEvent_t *ev);
cudaError_t cudaEventDestroy(cudaEvent_t ev);
cudaError_t cudaEventRecord(cudaEvent_t ev, void *stream = nullptr);
cudaError_t cudaEventSynchronize(cudaEvent_t ev);
cudaError_t cudaEventElapsedTime(float *ms, cudaEvent_t start, cudaEvent_t stop);
cudaError_t cudaDeviceSynchronize();
cudaError_t cudaPeekAtLastError();
cudaError_t cudaGetLastError();
const char *cudaGetErrorString(cudaError_t e);

// A texture object: the array, its filter mode and whether coordinates are normalised.
struct RefTexture {
  const cudaArray *arr;
  enum cudaTextureFilterMode filter;
  int normalized;
};
extern int g_ref_tex_8bit;  // 1: bilinear weights rounded to 8 fractional bits (the texture unit's)

// Sampling with unnormalised coordinates (the reference's textures, DPE.cpp:1078-1097): the
// sample at (u, v) blends the texels around (u - 0.5, v - 0.5); addresses beyond the image take
// the edge texel (unnormalised coordinates do not wrap), which for linear filtering is the clamp
// of the coordinate to [-1, size - 1] before the blend.  Weights are exact floats unless
// g_ref_tex_8bit.
inline float ref_texel(const cudaArray *a, int x, int y) {
  x = x < 0 ? 0 : (x >= a->w ? a->w - 1 : x);
  y = y < 0 ? 0 : (y >= a->h ? a->h - 1 : y);
  return a->data[(size_t)y * a->w + x];
}
inline float ref_floorf(float v) { return __builtin_floorf(v); }
inline float ref_tex2D_float(cudaTextureObject_t tex, float u, float v) {
  const RefTexture *t = reinterpret_cast<const RefTexture *>((uintptr_t)tex);
  const cudaArray *a = t->arr;
  if (t->normalized) { u *= (float)a->w; v *= (float)a->h; }
  if (t->filter == cudaFilterModePoint) return ref_texel(a, (int)ref_floorf(u), (int)ref_floorf(v));
  const float x = u - 0.5f, y = v - 0.5f;
  const float xc = __builtin_fminf(__builtin_fmaxf(x, -1.0f), (float)(a->w - 1));
  const float yc = __builtin_fminf(__builtin_fmaxf(y, -1.0f), (float)(a->h - 1));
  const float fx = ref_floorf(xc), fy = ref_floorf(yc);
  const int x0 = (int)fx, y0 = (int)fy;
  float ax = xc - fx, ay = yc - fy;
  if (g_ref_tex_8bit) { ax = ref_floorf(ax * 256.0f + 0.5f) / 256.0f; ay = ref_floorf(ay * 256.0f + 0.5f) / 256.0f; }
  const float v00 = ref_texel(a, x0, y0), v10 = ref_texel(a, x0 + 1, y0);
  const float v01 = ref_texel(a, x0, y0 + 1), v11 = ref_texel(a, x0 + 1, y0 + 1);
  const float top = (1.0f - ax) * v00 + ax * v10;
  const float bot = (1.0f - ax) * v01 + ax * v11;
  return (1.0f - ay) * top + ay * bot;
}
template <class T> T tex2D(cudaTextureObject_t tex, float x, float y);
template <> inline float tex2D<float>(cudaTextureObject_t tex, float x, float y) { return ref_tex2D_float(tex, x, y); }

// ---- kernel launch: `kernel<<<grid, block>>>(args)` is rewritten by the build recipe into
// `ref_launcher(grid, block, kernel)(args)`.
int ref_launch_threads();  // 1: blocks one after another; > 1: blocks in parallel (OpenMP)
bool ref_launch_serial(const void *kernel);  // kernels the harness runs one thread at a time
template <class K> struct RefLaunch {
  dim3 grid, block;
  K kernel;
  template <class... A> void operator()(A... args) const {
    const long long nb = (long long)grid.x * grid.y * grid.z;
    const int threads = ref_launch_serial((const void *)kernel) ? 1 : ref_launch_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads) if (threads > 1)
    for (long long b = 0; b < nb; ++b) {
      blockDim = block;
      gridDim = grid;
      blockIdx = uint3{(unsigned)(b % grid.x), (unsigned)((b / grid.x) % grid.y), (unsigned)(b / ((long long)grid.x * grid.y))};
      for (unsigned tz = 0; tz < block.z; ++tz)
        for (unsigned ty = 0; ty < block.y; ++ty)
          for (unsigned tx = 0; tx < block.x; ++tx) {
            threadIdx = uint3{tx, ty, tz};
            kernel(args...);
          }
    }
  }
};
template <class K> RefLaunch<K> ref_launcher(dim3 grid, dim3 block, K kernel) { return RefLaunch<K>{grid, block, kernel}; }

#endif
