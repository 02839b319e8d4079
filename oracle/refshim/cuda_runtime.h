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
struct cudaArray;  // a W x H float image (ref_runtime.cpp)
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

// Linear filtering of a 32-bit float texture with unnormalised coordinates: texel centres at
// i + 0.5; coordinates outside the image address the edge texel (unnormalised coordinates do not
// wrap).  Implemented in ref_runtime.cpp.
float ref_tex2D_float(cudaTextureObject_t tex, float x, float y);
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
