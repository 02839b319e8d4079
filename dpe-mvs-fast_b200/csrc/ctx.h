// ctx.h -- the dpe_ctx object behind the C ABI: device, stream, events and a device arena.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "../../include/dpe_b200.h"

// Text of the last failure on this host thread (read through dpe_last_error()).
void dpe_set_last_error(const char *what, cudaError_t err, const char *file, int line);

// Return DPE_ERR_CUDA (or DPE_ERR_OUT_OF_MEMORY) from the enclosing ABI function when a CUDA call
// fails; the reference exits the process instead (CudaSafeCall, DPE.cpp:646-679).
#define DPE_TRY(call)                                                              \
  do {                                                                             \
    cudaError_t dpe_err_ = (call);                                                 \
    if (dpe_err_ != cudaSuccess) {                                                 \
      cudaGetLastError();                                                          \
      dpe_set_last_error(#call, dpe_err_, __FILE__, __LINE__);                     \
      return dpe_err_ == cudaErrorMemoryAllocation ? DPE_ERR_OUT_OF_MEMORY : DPE_ERR_CUDA; \
    }                                                                              \
  } while (0)

// After a kernel launch: report launch-configuration errors with the kernel's name; with
// DPE_DEBUG_SYNC=1 in the environment also synchronise, so an execution error names its kernel
// (the reference's DPE_POST_KERNEL, DPE.cu:3-7).
bool dpe_debug_sync();
void dpe_count_launch();
#define DPE_LAUNCHED(name, stream)                                                 \
  do {                                                                             \
    dpe_count_launch();                                                            \
    cudaError_t dpe_err_ = cudaPeekAtLastError();                                  \
    if (dpe_err_ == cudaSuccess && dpe_debug_sync()) dpe_err_ = cudaStreamSynchronize(stream); \
    if (dpe_err_ != cudaSuccess) {                                                 \
      cudaGetLastError();                                                          \
      dpe_set_last_error(name, dpe_err_, __FILE__, __LINE__);                      \
      return DPE_ERR_CUDA;                                                         \
    }                                                                              \
  } while (0)

// Named grow-only device buffers, reused across calls (the reference's GpuWorkspace pools
// best-fit blocks per call; here each role keeps one buffer that only grows).
class Arena {
 public:
  template <class T> T *get(const char *name, size_t count) {
    const size_t bytes = count * sizeof(T) + 256;
    Slot &s = slots_[name];
    if (s.bytes < bytes) {
      if (s.ptr) cudaFree(s.ptr);
      s.ptr = nullptr;
      s.bytes = 0;
      if (cudaMalloc(&s.ptr, bytes) != cudaSuccess) {
        cudaGetLastError();
        s.ptr = nullptr;
        failed_ = true;
        return nullptr;
      }
      s.bytes = bytes;
      reserved_ += bytes;
    }
    return static_cast<T *>(s.ptr);
  }
  bool ok() {
    const bool r = !failed_;
    failed_ = false;
    return r;
  }
  void release() {
    for (auto &kv : slots_)
      if (kv.second.ptr) cudaFree(kv.second.ptr);
    slots_.clear();
  }
  size_t reserved() const { return reserved_; }

 private:
  struct Slot {
    void *ptr = nullptr;
    size_t bytes = 0;
  };
  std::map<std::string, Slot> slots_;
  bool failed_ = false;
  size_t reserved_ = 0;
};

#include "kernel_ids.h"

// ------------------------------------------------------------------ launch tuner
// Online choice of launch settings that change no result: the block shape of the
// one-thread-per-pixel kernels and the shared-memory carveout of the cooperative ones.  Per
// (kernel, size class) the first launches cycle through the candidates, each timed by an event
// pair on its stream; the times are read without synchronising, once the events have completed.
// When every candidate has kRounds samples, the lowest mean is kept for every later launch.
struct TuneEntry {
  static constexpr int kMaxCand = 8;
  int ncand = 0, trial = 0, chosen = -1;
  double sum[kMaxCand] = {};
  int count[kMaxCand] = {};
  struct Pend {
    int cand;
    cudaEvent_t t0, t1;
  };
  std::vector<Pend> pending;
};
struct LaunchTuner {
  static constexpr int kRounds = 2;
  bool enabled = true;
  std::map<long long, TuneEntry> table;  // key: kernel id * 64 + size class (log2 of the pixels)
  std::vector<cudaEvent_t> events;       // completed event pairs, for reuse
  static long long key(int kid, int cls) { return (long long)kid * 64 + cls; }
};

struct dpe_ctx {
  LaunchTuner tuner;
  int device = 0;
  int sms = 148;  // multiprocessors of the device: grid size of the work-list kernels
  dpe_options opt = {DPE_STAGE_FP32, 0};
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool count_evals = false;
  bool profile = false;
  Arena arena;
  // per-kernel statistics since the last reset
  double kms[KID_COUNT] = {};
  long long klaunch[KID_COUNT] = {};
  unsigned long long kevals[KID_COUNT][2] = {};
  struct Pending { int kid; cudaEvent_t a, b; };
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> pool;
  cudaEvent_t event() {
    if (pool.empty()) {
      cudaEvent_t e = nullptr;
      cudaEventCreate(&e);
      return e;
    }
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
  }
  // after the stream has been synchronised: fold the recorded launch times into kms/klaunch
  void collect() {
    for (const Pending &p : pending) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
        kms[p.kid] += ms;
        klaunch[p.kid] += 1;
      } else {
        cudaGetLastError();
      }
      pool.push_back(p.a);
      pool.push_back(p.b);
    }
    pending.clear();
  }
};

// Launch with per-kernel timing when ctx->profile is on (event pair around the launch).
#define DPE_TIMED(ctx, kid, stream, ...)                            \
  do {                                                              \
    cudaEvent_t t0_ = nullptr, t1_ = nullptr;                       \
    if ((ctx)->profile) {                                           \
      t0_ = (ctx)->event();                                         \
      t1_ = (ctx)->event();                                         \
      cudaEventRecord(t0_, stream);                                 \
    }                                                               \
    __VA_ARGS__;                                                    \
    if ((ctx)->profile) {                                           \
      cudaEventRecord(t1_, stream);                                 \
      (ctx)->pending.push_back(dpe_ctx::Pending{kid, t0_, t1_});    \
    }                                                               \
  } while (0)

// Edge maps of EdgeSegment mode 0 on the device (edges.cu).  dpe_edge_reserve sizes the scratch
// for images of up to `pixels`; dpe_edge_map_device enqueues the pipeline on ctx->stream for an
// 8-bit image, or for a float level image (converted like convertTo(CV_8UC1)) when `level` is
// given; dpe_edge_check reports the union-find guard after the stream has been synchronised.
int dpe_edge_reserve(dpe_ctx *ctx, size_t pixels);
int dpe_edge_map_device(dpe_ctx *ctx, const float *level, const uint8_t *image, int w, int h, uint8_t *edge);
int dpe_edge_check(dpe_ctx *ctx);
// Label maps of EdgeSegment mode 1 on the device (edges.cu): from the full-resolution 8-bit image
// `gray` (W x H, device memory) the int32 map at the level size ow x oh of `scale`; the stream is
// synchronised once inside (the number of large weak regions sizes the Hough launch).
int dpe_edge_labels_device(dpe_ctx *ctx, const uint8_t *gray, int W, int H, int scale, int high_res_img, int32_t *out,
                           int ow, int oh);
int dpe_edge_labels_check(dpe_ctx *ctx);
