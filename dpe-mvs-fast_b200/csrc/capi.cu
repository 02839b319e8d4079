// capi.cu -- C ABI: context, per-view PatchMatch call, NCC queries.
//
// dpe_pm_run replaces DPE::CudaSpaceInitialization + SetDataPassHelperInCuda + RunPatchMatch
// (DPE.cpp:1071-1252, DPE.cu:3130-3262).  The context owns a grow-only device arena (replacing
// the process-wide GpuWorkspace, DPE.cpp:775-837), one stream and timing events.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "ctx.h"
#include "pm_kernels.cuh"

using namespace dpe;

// ------------------------------------------------------------------ host helpers
namespace {

int check_problem(const dpe_problem *p) {
  if (!p) return DPE_ERR_INVALID_ARGUMENT;
  if (p->width < 16 || p->height < 16 || p->width > 32767 || p->height > 32767) return DPE_ERR_INVALID_ARGUMENT;
  if (p->num_images < 2 || p->num_images > DPE_MAX_IMAGES) return DPE_ERR_INVALID_ARGUMENT;
  if (p->memory != DPE_MEM_HOST && p->memory != DPE_MEM_DEVICE) return DPE_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < p->num_images; ++i) {
    if (!p->images[i]) return DPE_ERR_INVALID_ARGUMENT;
    if (p->params.geom_consistency && !p->depths[i]) return DPE_ERR_INVALID_ARGUMENT;
  }
  const dpe_params &P = p->params;
  if (P.state < DPE_FIRST_INIT || P.state > DPE_REFINE_ITER) return DPE_ERR_INVALID_ARGUMENT;
  if (P.state != DPE_FIRST_INIT && !p->plane_in) return DPE_ERR_INVALID_ARGUMENT;
  if (P.use_APD && !p->weak_in) return DPE_ERR_INVALID_ARGUMENT;
  if ((P.use_edge || P.use_limit) && (!p->edge || !p->edge_low_res || p->low_width <= 0 || p->low_height <= 0))
    return DPE_ERR_INVALID_ARGUMENT;
  if (P.use_label && !p->label) return DPE_ERR_INVALID_ARGUMENT;
  if (P.strong_radius < 0 || P.strong_increment <= 0 || P.weak_increment <= 0 || P.weak_radius < 0)
    return DPE_ERR_INVALID_ARGUMENT;
  if ((2 * P.strong_radius) / P.strong_increment + 1 > kMaxWin) return DPE_ERR_INVALID_ARGUMENT;
  if (P.use_APD && (2 * P.weak_radius) / P.weak_increment + 1 > kMaxWin) return DPE_ERR_INVALID_ARGUMENT;
  if (P.rotate_time < 1 || P.rotate_time > 4 || P.top_k < 0 || P.max_iterations < 0) return DPE_ERR_INVALID_ARGUMENT;
  return DPE_OK;
}

}  // namespace

// ------------------------------------------------------------------ error reporting
namespace {
thread_local std::string g_last_error;
}

void dpe_set_last_error(const char *what, cudaError_t err, const char *file, int line) {
  char buf[512];
  std::snprintf(buf, sizeof(buf), "%s failed: %s (%s) at %s:%d", what, cudaGetErrorName(err), cudaGetErrorString(err),
                file, line);
  g_last_error = buf;
}

bool dpe_debug_sync() {
  static const bool on = [] {
    const char *v = std::getenv("DPE_DEBUG_SYNC");
    return v && v[0] && v[0] != '0';
  }();
  return on;
}

extern "C" const char *dpe_last_error(void) { return g_last_error.c_str(); }

namespace {
std::atomic<unsigned long long> g_launches{0};
}
void dpe_count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
extern "C" uint64_t dpe_launch_count(void) { return g_launches.load(); }

// In checked builds (-DDPE_CHECKED) every kernel is followed by a read of the out-of-range record.
#ifdef DPE_CHECKED
static int dpe_check_oob(const char *name, cudaStream_t s) {
  long long o[4] = {0, 0, 0, 0};
  if (cudaStreamSynchronize(s) != cudaSuccess || cudaMemcpyFromSymbol(o, dpe::g_oob, sizeof(o)) != cudaSuccess) {
    cudaGetLastError();
    return DPE_ERR_CUDA;
  }
  if (o[3] == 0) return DPE_OK;
  char buf[256];
  std::snprintf(buf, sizeof(buf), "%s: %lld out-of-range accesses, first at tag %lld index %lld bound %lld", name, o[3],
                o[0], o[1], o[2]);
  g_last_error = buf;
  const long long z[4] = {0, 0, 0, 0};
  cudaMemcpyToSymbol(dpe::g_oob, z, sizeof(z));
  return DPE_ERR_CUDA;
}
#define PM_LAUNCHED(name, stream)                  \
  do {                                             \
    DPE_LAUNCHED(name, stream);                    \
    if (dpe_check_oob(name, stream)) return DPE_ERR_CUDA; \
  } while (0)
#else
#define PM_LAUNCHED(name, stream) DPE_LAUNCHED(name, stream)
#endif

// ------------------------------------------------------------------ context
extern "C" const char *dpe_status_string(int s) {
  switch (s) {
    case DPE_OK: return "ok";
    case DPE_ERR_INVALID_ARGUMENT: return "invalid argument";
    case DPE_ERR_CUDA: return "CUDA runtime error";
    case DPE_ERR_OUT_OF_MEMORY: return "device out of memory";
    case DPE_ERR_CAPACITY: return "output capacity too small";
    case DPE_ERR_NO_DEVICE: return "no usable CUDA device";
    case DPE_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
    default: return "unknown status";
  }
}

extern "C" void dpe_params_default(dpe_params *p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->max_iterations = 3;
  p->num_images = 5;
  p->sigma_spatial = 5.0f;
  p->sigma_color = 3.0f;
  p->top_k = 4;
  p->depth_min = 0.0f;
  p->depth_max = 1.0f;
  p->geom_consistency = 0;
  p->strong_radius = 5;
  p->strong_increment = 2;
  p->weak_radius = 5;
  p->weak_increment = 5;
  p->use_APD = 1;
  p->use_edge = 1;
  p->use_limit = 1;
  p->use_label = 1;
  p->use_radius = 1;
  p->high_res_img = 1;
  p->max_scale_size = 1;
  p->scale_size = 1;
  p->weak_peak_radius = 2;
  p->rotate_time = 4;
  p->ransac_threshold = 0.005f;
  p->geom_factor = 0.2f;
  p->state = DPE_FIRST_INIT;
}

extern "C" int dpe_ctx_create(int device, const dpe_limits *limits, dpe_ctx **out) {
  if (!out) return DPE_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
    cudaGetLastError();
    return DPE_ERR_NO_DEVICE;
  }
  dpe_ctx *c = new dpe_ctx();
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
    cudaGetLastError();
    delete c;
    return DPE_ERR_CUDA;
  }
  (void)limits;
  if (cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
    cudaGetLastError();
    dpe_ctx_destroy(c);
    return DPE_ERR_CUDA;
  }
  if (const char *v = std::getenv("DPE_STACK_LIMIT")) {
    const long long bytes = std::atoll(v);
    if (bytes > 0 && cudaDeviceSetLimit(cudaLimitStackSize, (size_t)bytes) != cudaSuccess) {
      cudaGetLastError();
      dpe_ctx_destroy(c);
      return DPE_ERR_CUDA;
    }
  }
  *out = c;
  return DPE_OK;
}

extern "C" int dpe_ctx_destroy(dpe_ctx *c) {
  if (!c) return DPE_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  c->arena.release();
  for (auto &kv : c->tuner.table)
    for (const TuneEntry::Pend &p : kv.second.pending) {
      cudaEventDestroy(p.t0);
      cudaEventDestroy(p.t1);
    }
  for (cudaEvent_t e : c->tuner.events) cudaEventDestroy(e);
  cudaEventDestroy(c->ev0);
  cudaEventDestroy(c->ev1);
  cudaStreamDestroy(c->stream);
  delete c;
  return DPE_OK;
}

// ------------------------------------------------------------------ dpe_pm_run
namespace {

dim3 full_grid(int W, int H) { return dim3((W + 15) / 16, (H + 7) / 8); }
const dim3 kFullBlock(16, 8);
dim3 half_grid(int W, int H) { return dim3((W + 31) / 32, ((H + 1) / 2 + 3) / 4); }
const dim3 kHalfBlock(32, 4);
// the cooperative strong update: 16 pixels of one colour per block (kCoopPix), one half-grid row
dim3 coop_grid(int W, int H) { return dim3((W + kCoopPix - 1) / kCoopPix, (H + 1) / 2); }
// the cooperative sweeps (DepthToWeak, LocalRefine): 16 pixels of one row per block
dim3 sweep_grid(int W, int H) { return dim3((W + kCoopPix - 1) / kCoopPix, H); }

// Blocks of 128 threads for a strided work list of up to `items` entries: enough to fill every
// multiprocessor, no more than the list needs.
unsigned list_grid(const dpe_ctx *ctx, long long items) {
  const long long need = (items + 127) / 128;
  const long long fill = (long long)ctx->sms * 16;
  return (unsigned)std::max(1LL, std::min(need, fill));
}

// Calls f(std::integral_constant<int, staging>) so that f can launch the instance of a cost kernel
// built for the call's staging (DPE_STAGE_*).
template <class F> void with_stage(int staging, F &&f) {
  if (staging == DPE_STAGE_FP16) f(std::integral_constant<int, DPE_STAGE_FP16>{});
  else if (staging == DPE_STAGE_BF16) f(std::integral_constant<int, DPE_STAGE_BF16>{});
  else f(std::integral_constant<int, DPE_STAGE_FP32>{});
}

// ------------------------------------------------------------------ launch tuner (ctx.h)
// Block shapes tried for the one-thread-per-pixel kernels of one problem (each thread reads and
// writes only its own pixel, so the shape changes nothing but speed; all fit __launch_bounds__(128)).
const dim3 kShapeCands[] = {dim3(16, 8), dim3(32, 4), dim3(8, 16), dim3(64, 2), dim3(8, 8)};
constexpr int kNumShapes = 5;
// Shared-memory carveouts (percent; -1 the driver's choice) tried for the cooperative kernels.
const int kCarveCands[] = {-1, 100, 75, 50};
constexpr int kNumCarves = 4;

int size_class(long long pixels) {
  int c = 0;
  while (c < 63 && (2LL << c) <= pixels) ++c;
  return c;
}
// Folds the completed measurements of e into its sums; keeps the others pending.
void tune_harvest(dpe_ctx *ctx, TuneEntry &e) {
  size_t keep = 0;
  for (size_t i = 0; i < e.pending.size(); ++i) {
    TuneEntry::Pend &p = e.pending[i];
    const cudaError_t q = cudaEventQuery(p.t1);
    if (q == cudaErrorNotReady) {
      e.pending[keep++] = p;
      continue;
    }
    float ms = 0.f;
    if (q == cudaSuccess && cudaEventElapsedTime(&ms, p.t0, p.t1) == cudaSuccess) {
      e.sum[p.cand] += ms;
      e.count[p.cand] += 1;
    } else {
      cudaGetLastError();
    }
    ctx->tuner.events.push_back(p.t0);
    ctx->tuner.events.push_back(p.t1);
  }
  e.pending.resize(keep);
}
cudaEvent_t tune_event(dpe_ctx *ctx) {
  if (!ctx->tuner.events.empty()) {
    cudaEvent_t e = ctx->tuner.events.back();
    ctx->tuner.events.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return e;
}
// One launch under the tuner: `cand` is the candidate to launch with; call finish() right after
// the launch.  With the tuner off, or once an entry has chosen, no events are recorded.
struct TunedLaunch {
  dpe_ctx *ctx;
  TuneEntry *e = nullptr;
  cudaStream_t s;
  int cand = 0;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  TunedLaunch(dpe_ctx *c, int kid, long long pixels, int ncand, cudaStream_t st) : ctx(c), s(st) {
    if (!ctx->tuner.enabled) return;
    e = &ctx->tuner.table[LaunchTuner::key(kid, size_class(pixels))];
    e->ncand = ncand;
    if (e->chosen >= 0) {
      cand = e->chosen;
      return;
    }
    tune_harvest(ctx, *e);
    bool done = e->pending.empty();
    for (int i = 0; i < ncand && done; ++i) done = e->count[i] >= LaunchTuner::kRounds;
    if (done) {
      int best = 0;
      for (int i = 1; i < ncand; ++i)
        if (e->sum[i] / e->count[i] < e->sum[best] / e->count[best]) best = i;
      e->chosen = cand = best;
      return;
    }
    cand = e->trial++ % ncand;
    if (e->trial > 4 * LaunchTuner::kRounds * ncand) {  // samples still in flight: no more events
      cand = 0;
      return;
    }
    t0 = tune_event(ctx);
    t1 = tune_event(ctx);
    if (t0 && t1) {
      cudaEventRecord(t0, s);
      return;
    }
    if (t0) ctx->tuner.events.push_back(t0);  // no pair: this launch goes unmeasured
    if (t1) ctx->tuner.events.push_back(t1);
    t0 = t1 = nullptr;
  }
  void finish() {
    if (!t0 || !t1) return;
    cudaEventRecord(t1, s);
    e->pending.push_back(TuneEntry::Pend{cand, t0, t1});
  }
};
// The preferred carveout of a kernel function, set only when it changes (the attribute belongs
// to the function, process-wide).
void set_carveout(const void *func, int percent) {
  static std::mutex mu;
  static std::map<const void *, int> current;
  std::lock_guard<std::mutex> lock(mu);
  auto it = current.find(func);
  if (it != current.end() && it->second == percent) return;
  if (cudaFuncSetAttribute(func, cudaFuncAttributePreferredSharedMemoryCarveout, percent) == cudaSuccess)
    current[func] = percent;
  else
    cudaGetLastError();
}
dim3 shape_grid(int W, int H, dim3 b) { return dim3((W + b.x - 1) / b.x, (H + b.y - 1) / b.y); }

void launch_strong_update(int staging, bool gn, dim3 grid, size_t smem, cudaStream_t s, const Launch args, int it,
                          int parity, int carveout) {
  with_stage(staging, [&](auto st) {
    if (gn) {
      set_carveout((const void *)k_strong_update<decltype(st)::value, true>, carveout);
      k_strong_update<decltype(st)::value, true><<<grid, kCoopThreads, smem, s>>>(args, it, parity);
    } else {
      set_carveout((const void *)k_strong_update<decltype(st)::value, false>, carveout);
      k_strong_update<decltype(st)::value, false><<<grid, kCoopThreads, smem, s>>>(args, it, parity);
    }
  });
}

// WEAK pixels of one red/black colour, (x + y) & 1 == parity.
struct WeakOfColour {
  const uint8_t *weak;
  int W, parity;
  __host__ __device__ __forceinline__ bool operator()(const int &p) const {
    return weak[p] == DPE_WEAK && (((p % W) + (p / W)) & 1) == parity;
  }
};

}  // namespace

namespace {

// One problem of a call: its host-side argument block (copied to the device before the kernels)
// and the inputs the first kernel reads.  Problem i of a batch keeps its buffers under arena
// names suffixed with its index, so problems never share state.
struct ProblemState {
  PMArgs a;
  int staging = DPE_STAGE_FP32;  // the storage the cost kernels sample this problem's sources from
  const float4 *plane_in = nullptr;
  const uint32_t *views_in = nullptr;
  const uint8_t *weak_in = nullptr;
  int *weak_flag = nullptr;
  size_t L = 0, wcap = 0;
};

std::string slot_name(const char *base, int index) {
  return index == 0 ? std::string(base) : std::string(base) + "#" + std::to_string(index);
}

// Buffers, uploads and the padded / staged source images of problem `index`.
int setup_problem(dpe_ctx *ctx, const dpe_problem *p, int index, ProblemState *ps) {
  cudaStream_t s = ctx->stream;
  const int W = p->width, H = p->height, N = p->num_images;
  const size_t L = (size_t)W * H;
  const size_t PL = (size_t)(W + 2) * (H + 2);
  const bool host = p->memory == DPE_MEM_HOST;
  const cudaMemcpyKind h2d = host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  Arena &A = ctx->arena;
  auto get = [&](auto *tag, const char *name, size_t count) {
    using T = std::remove_pointer_t<decltype(tag)>;
    return A.get<T>(slot_name(name, index).c_str(), count);
  };
  PMArgs &a = ps->a;
  std::memset(&a, 0, sizeof(a));
  a.W = W; a.H = H; a.N = N; a.pad_w = W + 2;
  a.P = p->params;
  a.P.num_images = N;
  for (int i = 0; i < N; ++i) a.cam[i] = p->cameras[i];
  set_homography_bases(a);
  a.key[0] = (uint32_t)p->seed;
  a.key[1] = (uint32_t)(p->seed >> 32);
  a.gn = ctx->opt.gn_refine;
  ps->L = L;
  ps->wcap = (L + 1) / 2;  // pixels of one colour

  // ---- device buffers
  float *img_pad = get((float *)0, "img_pad", PL * N);
  float *stage = host ? get((float *)0, "img_stage", L * N) : nullptr;
  a.plane = get((float4 *)0, "plane", L);
  a.plane_snap = get((float4 *)0, "plane_snap", L);
  a.fit_plane = get((float4 *)0, "fit_plane", L);
  a.cost = get((float *)0, "cost", L);
  a.cost_snap = get((float *)0, "cost_snap", L);
  a.complexity = get((float *)0, "complexity", L);
  a.views = get((uint32_t *)0, "views", L);
  a.rng_ctr = get((uint32_t *)0, "rng_ctr", L);
  a.vweight = get((uint4 *)0, "vweight", L);
  a.weak = get((uint8_t *)0, "weak", L);
  a.reliable = get((uint8_t *)0, "reliable", L);
  a.nmap = get((int32_t *)0, "nmap", L);
  a.radius = get((int32_t *)0, "radius", L);
  ps->weak_flag = get((int32_t *)0, "weak_flag", L);
  a.neigh = get((short2 *)0, "neigh", L * kNeighbours);
  a.lab_bound = get((short2 *)0, "lab_bound", L * 8);
  a.edge_neigh = get((short2 *)0, "edge_neigh", L * 8);
  a.nearest = get((short2 *)0, "nearest", L);
  const size_t wcap = ps->wcap;
  if (a.P.use_APD) {
    const int n = N - 1;
    const int side = (2 * a.P.weak_radius) / a.P.weak_increment + 1;
    a.wtaps = side * side;
    a.wtab_stride = kMaxWin * kMaxWin + 8 * a.wtaps;
    int *wl = get((int *)0, "weak_list", 2 * wcap);
    a.wlist[0] = wl;
    a.wlist[1] = wl ? wl + wcap : nullptr;
    a.wcount = get((int *)0, "weak_count", 2);
    a.wtab = get((float2 *)0, "weak_tab", wcap * a.wtab_stride);
    a.wwin = get((float4 *)0, "weak_win", wcap * kNeighbours);
    a.wcost = get((float *)0, "weak_cost", wcap * 10 * n);
    a.wgeom = get((float *)0, "weak_geom", wcap * 10 * n);
    a.whyp = get((float4 *)0, "weak_hyp", wcap * 5);
    a.wcost_r = get((float *)0, "weak_cost_r", wcap * 5 * n);
    a.wgeom_r = get((float *)0, "weak_geom_r", wcap * 5 * n);
    a.wstate = get((float4 *)0, "weak_state", wcap * 2);
  }
  if (!A.ok()) return DPE_ERR_OUT_OF_MEMORY;

  if (host) {
    if (a.P.state != DPE_FIRST_INIT) {
      float4 *d = get((float4 *)0, "plane_in", L);
      if (!d) return DPE_ERR_OUT_OF_MEMORY;
      DPE_TRY(cudaMemcpyAsync(d, p->plane_in, L * sizeof(float4), h2d, s));
      ps->plane_in = d;
      if (p->selected_views_in) {
        uint32_t *dv = get((uint32_t *)0, "views_in", L);
        if (!dv) return DPE_ERR_OUT_OF_MEMORY;
        DPE_TRY(cudaMemcpyAsync(dv, p->selected_views_in, L * 4, h2d, s));
        ps->views_in = dv;
      }
    }
    if (a.P.use_APD) {
      uint8_t *dw = get((uint8_t *)0, "weak_in", L);
      if (!dw) return DPE_ERR_OUT_OF_MEMORY;
      DPE_TRY(cudaMemcpyAsync(dw, p->weak_in, L, h2d, s));
      ps->weak_in = dw;
    }
  } else {
    ps->plane_in = reinterpret_cast<const float4 *>(p->plane_in);
    ps->views_in = p->selected_views_in;
    ps->weak_in = p->weak_in;
  }
  if (a.P.use_edge || a.P.use_limit) {
    const size_t LL = (size_t)p->low_width * p->low_height;
    a.lowW = p->low_width; a.lowH = p->low_height;
    if (host) {
      uint8_t *de = get((uint8_t *)0, "edge", L), *dl = get((uint8_t *)0, "edge_low", LL);
      if (!de || !dl) return DPE_ERR_OUT_OF_MEMORY;
      DPE_TRY(cudaMemcpyAsync(de, p->edge, L, h2d, s));
      DPE_TRY(cudaMemcpyAsync(dl, p->edge_low_res, LL, h2d, s));
      a.edge = de; a.edge_low = dl;
    } else {
      a.edge = p->edge; a.edge_low = p->edge_low_res;
    }
  }
  if (a.P.use_label) {
    if (host) {
      int32_t *dl = get((int32_t *)0, "label", L);
      if (!dl) return DPE_ERR_OUT_OF_MEMORY;
      DPE_TRY(cudaMemcpyAsync(dl, p->label, L * 4, h2d, s));
      a.label = dl;
    } else {
      a.label = p->label;
    }
  }
  if (a.P.geom_consistency) {
    float *dd = host ? get((float *)0, "depths", L * N) : nullptr;
    if (host && !dd) return DPE_ERR_OUT_OF_MEMORY;
    for (int i = 0; i < N; ++i) {
      if (host) {
        DPE_TRY(cudaMemcpyAsync(dd + L * i, p->depths[i], L * 4, h2d, s));
        a.dep[i] = dd + L * i;
      } else {
        a.dep[i] = p->depths[i];
      }
    }
  }
  for (int i = 0; i < N; ++i) {
    const float *src = p->images[i];
    if (host) {
      DPE_TRY(cudaMemcpyAsync(stage + L * i, p->images[i], L * 4, h2d, s));
      src = stage + L * i;
    }
    a.img[i] = img_pad + PL * i;
    k_pad_image<<<dim3((W + 2 + 31) / 32, (H + 2 + 7) / 8), dim3(32, 8), 0, s>>>(src, img_pad + PL * i, W, H);
    PM_LAUNCHED("k_pad_image", s);
  }
  // FP32 staging: when every source texel is exact in BF16 (8-bit images, the finest pyramid
  // level), the cost kernels sample BF16 pairs instead: the same values, half the gather bytes.
  int staging = ctx->opt.staging;
  if (staging == DPE_STAGE_FP32 && N > 1) {
    unsigned *flag = get((unsigned *)0, "bf16_flag", 1);
    if (!flag) return DPE_ERR_OUT_OF_MEMORY;
    DPE_TRY(cudaMemsetAsync(flag, 0, sizeof(unsigned), s));
    const long long n = (long long)PL * (N - 1);
    const unsigned blocks = (unsigned)std::max(1LL, std::min((n + 255) / 256, (long long)ctx->sms * 8));
    k_bf16_exact<<<blocks, 256, 0, s>>>(img_pad + PL, n, flag);
    PM_LAUNCHED("k_bf16_exact", s);
    unsigned inexact = 1;
    DPE_TRY(cudaMemcpyAsync(&inexact, flag, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    DPE_TRY(cudaStreamSynchronize(s));
    if (!inexact) staging = DPE_STAGE_BF16;
  }
  ps->staging = staging;
  a.stage = staging;
  uint32_t *img_pairs = staging != DPE_STAGE_FP32 ? get((uint32_t *)0, "img_pairs", PL * N) : nullptr;
  if (staging != DPE_STAGE_FP32 && !img_pairs) return DPE_ERR_OUT_OF_MEMORY;
  for (int i = 1; i < N; ++i) {
    if (staging != DPE_STAGE_FP32) {
      a.pair[i] = img_pairs + PL * i;
      if (staging == DPE_STAGE_BF16)
        k_stage_pairs<true><<<(unsigned)((PL + 255) / 256), 256, 0, s>>>(img_pad + PL * i, img_pairs + PL * i, (long long)PL);
      else
        k_stage_pairs<false><<<(unsigned)((PL + 255) / 256), 256, 0, s>>>(img_pad + PL * i, img_pairs + PL * i, (long long)PL);
      PM_LAUNCHED("k_stage_pairs", s);
    }
  }
  return DPE_OK;
}

// Grids of one kernel sequence: for one problem the 2D pixel grids; for a batch one 1D grid per
// kind over all problems, with the prefix tables the kernels resolve their problem from.
struct SequenceGrids {
  Launch full, half, prep, eval, coop, sweep;
  dim3 fg, hg, cg, sg;
  size_t coop_smem = 0;  // dynamic shared bytes of the strong update (largest source count)
  size_t lr_smem = 0;    // dynamic shared bytes of LocalRefine (largest source count)
  unsigned gp = 0, ge = 0;
  const dim3 fb = kFullBlock, hb = kHalfBlock;
};

// The kernel sequence of DPE::RunPatchMatch (DPE.cu:3157-3234) for n problems that share the
// schedule flags (state, APD, edges, geometric term, iteration count).
int run_sequence(dpe_ctx *ctx, ProblemState *ps, int n, const PMArgs *d_args, const SequenceGrids &g) {
  cudaStream_t s = ctx->stream;
  Arena &A = ctx->arena;
  const dpe_params &P = ps[0].a.P;
  // one staging for the sequence: BF16 pairs only when every problem has them
  int staging = ps[0].staging;
  for (int b = 1; b < n; ++b)
    if (ps[b].staging != staging) staging = ctx->opt.staging;
  const bool gn = ctx->opt.gn_refine != 0;
  DPE_TIMED(ctx, KID_INIT_STATE, s, for (int b = 0; b < n; ++b) {
    // k_init_state takes per-problem inputs: one launch per problem
    const Launch one{d_args + b, nullptr, 1};
    k_init_state<<<full_grid(ps[b].a.W, ps[b].a.H), kFullBlock, 0, s>>>(one, ps[b].plane_in, ps[b].views_in,
                                                                         ps[b].weak_in, ps[b].weak_flag);
  });
  PM_LAUNCHED("k_init_state", s);
  for (int b = 0; b < n; ++b) {
    const PMArgs &a = ps[b].a;
    const int L = (int)ps[b].L;
    if (P.use_APD) {
      size_t tmp_bytes = 0;
      cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, ps[b].weak_flag, a.nmap, L, s);
      void *tmp = A.get<uint8_t>("scan_tmp", tmp_bytes + 16);
      if (!tmp) return DPE_ERR_OUT_OF_MEMORY;
      DPE_TRY(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, ps[b].weak_flag, a.nmap, L, s));
    } else {
      DPE_TRY(cudaMemsetAsync(a.nmap, 0, (size_t)L * 4, s));
    }
  }
  // Launch settings the tuner picks (results do not depend on them): the block shape of the random
  // initialisation for one problem (a batch keeps the 16 x 8 layout its block table is built for)
  // and the shared-memory carveout of the strong update.  These two do the same work in every
  // launch of a size class, so launches with different settings compare; the kernels whose work
  // follows a view's weak pixels (GenNeighbours, the nearest-strong search, the plane fit,
  // DepthToWeak, LocalRefine) keep hand-measured settings, since their samples would compare views.
  long long pix_all = 0;
  for (int b = 0; b < n; ++b) pix_all += (long long)ps[b].L;
  auto shaped = [&](int kid, auto launch) {
    if (n != 1 || kid != KID_RANDOM_INIT) {
      launch(g.fg, g.fb);
      return;
    }
    TunedLaunch t(ctx, kid, pix_all, kNumShapes, s);
    const dim3 bl = kShapeCands[t.cand];
    launch(shape_grid(ps[0].a.W, ps[0].a.H, bl), bl);
    t.finish();
  };
  auto carved = [&](int kid, auto launch) {
    if (kid != KID_STRONG_UPDATE) {
      launch(-1);
      return;
    }
    TunedLaunch t(ctx, kid, pix_all, kNumCarves, s);
    launch(kCarveCands[t.cand]);
    t.finish();
  };
  DPE_TIMED(ctx, KID_GEN_EDGE_INFORM, s,
            shaped(KID_GEN_EDGE_INFORM, [&](dim3 gr, dim3 bl) { k_gen_edge_inform<<<gr, bl, 0, s>>>(g.full); }));
  PM_LAUNCHED("k_gen_edge_inform", s);
  DPE_TIMED(ctx, KID_FIND_NEAREST, s,
            shaped(KID_FIND_NEAREST, [&](dim3 gr, dim3 bl) { k_find_nearest_strong<<<gr, bl, 0, s>>>(g.full); }));
  PM_LAUNCHED("k_find_nearest_strong", s);
  DPE_TIMED(ctx, KID_GEN_NEIGHBOURS, s,
            shaped(KID_GEN_NEIGHBOURS, [&](dim3 gr, dim3 bl) { k_gen_neighbours<<<gr, bl, 0, s>>>(g.full); }));
  PM_LAUNCHED("k_gen_neighbours", s);
  DPE_TIMED(ctx, KID_NEIGHBOUR_UPDATE, s, k_neighbour_update<<<g.fg, g.fb, 0, s>>>(g.full));
  PM_LAUNCHED("k_neighbour_update", s);
  if (P.use_APD) {
    // WEAK pixels per colour, in raster order; the states are final for the iterations
    for (int b = 0; b < n; ++b) {
      const PMArgs &a = ps[b].a;
      const int L = (int)ps[b].L;
      size_t sel_bytes = 0;
      thrust::counting_iterator<int> first(0);
      cub::DeviceSelect::If(nullptr, sel_bytes, first, const_cast<int *>(a.wlist[0]), const_cast<int *>(a.wcount), L,
                            WeakOfColour{a.weak, a.W, 0}, s);
      void *sel_tmp = A.get<uint8_t>("select_tmp", sel_bytes + 16);
      if (!sel_tmp) return DPE_ERR_OUT_OF_MEMORY;
      for (int parity = 0; parity < 2; ++parity)
        DPE_TRY(cub::DeviceSelect::If(sel_tmp, sel_bytes, first, const_cast<int *>(a.wlist[parity]),
                                      const_cast<int *>(a.wcount) + parity, L, WeakOfColour{a.weak, a.W, parity}, s));
    }
  }
  DPE_TIMED(ctx, KID_RANDOM_INIT, s, shaped(KID_RANDOM_INIT, [&](dim3 gr, dim3 bl) {
              with_stage(staging, [&](auto st) { k_random_init<decltype(st)::value><<<gr, bl, 0, s>>>(g.full); });
            }));
  PM_LAUNCHED("k_random_init", s);
  for (int it = 0; it < P.max_iterations; ++it) {
    for (int parity = 0; parity < 2; ++parity) {
      if (P.use_edge)
        for (int b = 0; b < n; ++b) {
          const PMArgs &a = ps[b].a;
          DPE_TRY(cudaMemcpyAsync(a.plane_snap, a.plane, ps[b].L * sizeof(float4), cudaMemcpyDeviceToDevice, s));
          DPE_TRY(cudaMemcpyAsync(a.cost_snap, a.cost, ps[b].L * 4, cudaMemcpyDeviceToDevice, s));
        }
      DPE_TIMED(ctx, KID_STRONG_UPDATE, s, carved(KID_STRONG_UPDATE, [&](int cv) {
                  launch_strong_update(staging, gn, g.cg, g.coop_smem, s, g.coop, it, parity, cv);
                }));
      PM_LAUNCHED("k_strong_update", s);
    }
    DPE_TIMED(ctx, KID_RANSAC, s,
              shaped(KID_RANSAC, [&](dim3 gr, dim3 bl) { k_ransac_fit_plane<<<gr, bl, 0, s>>>(g.full); }));
    PM_LAUNCHED("k_ransac_fit_plane", s);
    if (P.use_APD)
      for (int parity = 0; parity < 2; ++parity) {
        DPE_TIMED(ctx, KID_WEAK_PREPARE, s, k_weak_prepare<<<g.gp, 128, 0, s>>>(g.prep, parity));
        PM_LAUNCHED("k_weak_prepare", s);
        DPE_TIMED(ctx, KID_WEAK_EVAL, s, with_stage(staging, [&](auto st) { k_weak_eval<false, decltype(st)::value><<<g.ge, 128, 0, s>>>(g.eval, parity); }));
        PM_LAUNCHED("k_weak_eval", s);
        DPE_TIMED(ctx, KID_WEAK_DECIDE, s, k_weak_decide<<<g.gp, 128, 0, s>>>(g.prep, it, parity));
        PM_LAUNCHED("k_weak_decide", s);
        DPE_TIMED(ctx, KID_WEAK_EVAL, s, with_stage(staging, [&](auto st) { k_weak_eval<true, decltype(st)::value><<<g.ge, 128, 0, s>>>(g.eval, parity); }));
        PM_LAUNCHED("k_weak_eval", s);
        DPE_TIMED(ctx, KID_WEAK_FINISH, s, with_stage(staging, [&](auto st) { k_weak_finish<decltype(st)::value><<<g.gp, 128, 0, s>>>(g.prep, parity); }));
        PM_LAUNCHED("k_weak_finish", s);
      }
  }
  DPE_TIMED(ctx, KID_DEPTH_NORMAL, s, k_get_depth_normal<<<g.fg, g.fb, 0, s>>>(g.full));
  PM_LAUNCHED("k_get_depth_normal", s);
  for (int parity = 0; parity < 2; ++parity) {
    DPE_TIMED(ctx, KID_FILTER, s, k_filter_strong<<<g.hg, g.hb, 0, s>>>(g.half, parity));
    PM_LAUNCHED("k_filter_strong", s);
  }
  DPE_TIMED(ctx, KID_DEPTH_TO_WEAK, s, carved(KID_DEPTH_TO_WEAK, [&](int cv) {
              with_stage(staging, [&](auto st) {
                set_carveout((const void *)k_depth_to_weak<decltype(st)::value>, cv);
                k_depth_to_weak<decltype(st)::value><<<g.sg, kCoopThreads, 0, s>>>(g.sweep);
              });
            }));
  PM_LAUNCHED("k_depth_to_weak", s);
  {
    cudaError_t attr = cudaSuccess;
    with_stage(staging, [&](auto st) {
      if (g.lr_smem > 48 * 1024)
        attr = cudaFuncSetAttribute(k_local_refine<decltype(st)::value>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)g.lr_smem);
    });
    DPE_TRY(attr);
  }
  DPE_TIMED(ctx, KID_LOCAL_REFINE, s, carved(KID_LOCAL_REFINE, [&](int cv) {
              with_stage(staging, [&](auto st) {
                set_carveout((const void *)k_local_refine<decltype(st)::value>, cv);
                k_local_refine<decltype(st)::value><<<g.sg, kCoopThreads, g.lr_smem, s>>>(g.sweep);
              });
            }));
  PM_LAUNCHED("k_local_refine", s);
  return DPE_OK;
}

int copy_outputs(dpe_ctx *ctx, const ProblemState &ps, const dpe_problem *p, dpe_pm_out *out) {
  cudaStream_t s = ctx->stream;
  const PMArgs &a = ps.a;
  const size_t L = ps.L;
  const cudaMemcpyKind d2o = p->memory == DPE_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  DPE_TRY(cudaMemcpyAsync(out->plane, a.plane, L * sizeof(float4), d2o, s));
  DPE_TRY(cudaMemcpyAsync(out->weak, a.weak, L, d2o, s));
  DPE_TRY(cudaMemcpyAsync(out->selected_views, a.views, L * 4, d2o, s));
  if (out->costs) DPE_TRY(cudaMemcpyAsync(out->costs, a.cost, L * 4, d2o, s));
  return DPE_OK;
}

// Runs problems ps[0..n) through one kernel sequence and fills outs[0..n).
int pm_run_problems(dpe_ctx *ctx, const dpe_problem *const *problems, int n, dpe_pm_out *const *outs) {
  DPE_TRY(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  Arena &A = ctx->arena;
  std::vector<ProblemState> ps(n);
  unsigned long long *counters = A.get<unsigned long long>("counters", 2 * KID_COUNT);
  PMArgs *d_args = A.get<PMArgs>("pm_args", n);
  int *d_start = n > 1 ? A.get<int>("batch_start", 6 * (n + 1)) : nullptr;
  if (!counters || !d_args || (n > 1 && !d_start)) return DPE_ERR_OUT_OF_MEMORY;
  if (ctx->count_evals) DPE_TRY(cudaMemsetAsync(counters, 0, 16 * KID_COUNT, s));
  for (int b = 0; b < n; ++b) {
    int st = setup_problem(ctx, problems[b], b, &ps[b]);
    if (st) return st;
    ps[b].a.counters = ctx->count_evals ? counters : nullptr;
  }
  std::vector<PMArgs> host_args(n);
  for (int b = 0; b < n; ++b) host_args[b] = ps[b].a;
  DPE_TRY(cudaMemcpyAsync(d_args, host_args.data(), sizeof(PMArgs) * n, cudaMemcpyHostToDevice, s));
#ifdef DPE_CHECKED
  {
    const PMArgs &a = ps[0].a;
    long long *echo = A.get<long long>("echo", 8);
    k_echo_args<<<1, 1, 0, s>>>(d_args, echo);
    long long e[8];
    DPE_TRY(cudaMemcpyAsync(e, echo, sizeof(e), cudaMemcpyDeviceToHost, s));
    DPE_TRY(cudaStreamSynchronize(s));
    const long long h[8] = {a.W, a.H, a.N, a.P.strong_radius, a.P.strong_increment, a.P.use_edge, a.P.num_images,
                            (long long)sizeof(PMArgs)};
    for (int i = 0; i < 8; ++i)
      if (e[i] != h[i]) {
        char buf[160];
        std::snprintf(buf, sizeof(buf), "args echo mismatch at field %d: device %lld host %lld", i, e[i], h[i]);
        g_last_error = buf;
        return DPE_ERR_CUDA;
      }
  }
#endif
  SequenceGrids g;
  if (n == 1) {
    const PMArgs &a = ps[0].a;
    const Launch one{d_args, nullptr, 1};
    g.full = g.half = g.prep = g.eval = g.coop = g.sweep = one;
    g.sg = sweep_grid(a.W, a.H);
    g.fg = full_grid(a.W, a.H);
    g.hg = half_grid(a.W, a.H);
    g.cg = coop_grid(a.W, a.H);
    g.coop_smem = coop_smem_bytes(a.N - 1);
    g.lr_smem = local_refine_smem_bytes(a.N - 1);
    g.gp = list_grid(ctx, (long long)ps[0].wcap);
    g.ge = list_grid(ctx, (long long)ps[0].wcap * 10 * (a.N - 1));
  } else {
    // the problems' grids laid end to end: prefix tables per grid kind
    std::vector<int> start(6 * (n + 1), 0);
    for (int b = 0; b < n; ++b) {
      const PMArgs &a = ps[b].a;
      const dim3 f = full_grid(a.W, a.H), h = half_grid(a.W, a.H), cg = coop_grid(a.W, a.H);
      start[4 * (n + 1) + b + 1] = start[4 * (n + 1) + b] + (int)(cg.x * cg.y);
      const dim3 sg = sweep_grid(a.W, a.H);
      start[5 * (n + 1) + b + 1] = start[5 * (n + 1) + b] + (int)(sg.x * sg.y);
      g.coop_smem = std::max(g.coop_smem, coop_smem_bytes(a.N - 1));
      g.lr_smem = std::max(g.lr_smem, local_refine_smem_bytes(a.N - 1));
      start[0 * (n + 1) + b + 1] = start[0 * (n + 1) + b] + (int)(f.x * f.y);
      start[1 * (n + 1) + b + 1] = start[1 * (n + 1) + b] + (int)(h.x * h.y);
      start[2 * (n + 1) + b + 1] = start[2 * (n + 1) + b] + (int)list_grid(ctx, (long long)ps[b].wcap);
      start[3 * (n + 1) + b + 1] =
          start[3 * (n + 1) + b] + (int)list_grid(ctx, (long long)ps[b].wcap * 10 * (a.N - 1));
    }
    DPE_TRY(cudaMemcpyAsync(d_start, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    g.full = Launch{d_args, d_start + 0 * (n + 1), n};
    g.half = Launch{d_args, d_start + 1 * (n + 1), n};
    g.prep = Launch{d_args, d_start + 2 * (n + 1), n};
    g.eval = Launch{d_args, d_start + 3 * (n + 1), n};
    g.coop = Launch{d_args, d_start + 4 * (n + 1), n};
    g.cg = dim3(start[4 * (n + 1) + n]);
    g.sweep = Launch{d_args, d_start + 5 * (n + 1), n};
    g.sg = dim3(start[5 * (n + 1) + n]);
    g.fg = dim3(start[0 * (n + 1) + n]);
    g.hg = dim3(start[1 * (n + 1) + n]);
    g.gp = (unsigned)start[2 * (n + 1) + n];
    g.ge = (unsigned)start[3 * (n + 1) + n];
    // blocks keep the single-problem shapes (16x8 full, 32x4 half): only the block index is 1D
  }
  DPE_TRY(cudaEventRecord(ctx->ev0, s));
  int st = run_sequence(ctx, ps.data(), n, d_args, g);
  if (st) return st;
  DPE_TRY(cudaEventRecord(ctx->ev1, s));
  for (int b = 0; b < n; ++b)
    if ((st = copy_outputs(ctx, ps[b], problems[b], outs[b]))) return st;
  unsigned long long cnt[2 * KID_COUNT] = {};
  if (ctx->count_evals) DPE_TRY(cudaMemcpyAsync(cnt, counters, sizeof(cnt), cudaMemcpyDeviceToHost, s));
  DPE_TRY(cudaStreamSynchronize(s));
  ctx->collect();
  unsigned long long strong_total = 0, weak_total = 0;
  for (int k = 0; k < KID_COUNT; ++k) {
    ctx->kevals[k][0] += cnt[2 * k];
    ctx->kevals[k][1] += cnt[2 * k + 1];
    strong_total += cnt[2 * k];
    weak_total += cnt[2 * k + 1];
  }
  float ms = 0.f;
  DPE_TRY(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  for (int b = 0; b < n; ++b) {  // the batch's totals, reported on every output
    outs[b]->gpu_ms = ms;
    outs[b]->strong_ncc_evals = strong_total;
    outs[b]->weak_ncc_evals = weak_total;
  }
  return DPE_OK;
}

}  // namespace

extern "C" int dpe_pm_run(dpe_ctx *ctx, const dpe_problem *p, dpe_pm_out *out) {
  if (!ctx || !out) return DPE_ERR_INVALID_ARGUMENT;
  int st = check_problem(p);
  if (st) return st;
  if (!out->plane || !out->weak || !out->selected_views) return DPE_ERR_INVALID_ARGUMENT;
  return pm_run_problems(ctx, &p, 1, &out);
}

extern "C" int dpe_pm_run_batch(dpe_ctx *ctx, const dpe_problem *problems, int count, dpe_pm_out *outs) {
  if (!ctx || !problems || !outs || count < 1 || count > DPE_MAX_BATCH) return DPE_ERR_INVALID_ARGUMENT;
  std::vector<const dpe_problem *> pp(count);
  std::vector<dpe_pm_out *> po(count);
  for (int b = 0; b < count; ++b) {
    int st = check_problem(&problems[b]);
    if (st) return st;
    if (!outs[b].plane || !outs[b].weak || !outs[b].selected_views) return DPE_ERR_INVALID_ARGUMENT;
    const dpe_params &P = problems[b].params, &P0 = problems[0].params;
    if (P.state != P0.state || P.use_APD != P0.use_APD || P.use_edge != P0.use_edge ||
        P.geom_consistency != P0.geom_consistency || P.max_iterations != P0.max_iterations)
      return DPE_ERR_INVALID_ARGUMENT;  // one kernel sequence: the schedule flags must agree
    pp[b] = &problems[b];
    po[b] = &outs[b];
  }
  return pm_run_problems(ctx, pp.data(), count, po.data());
}

// ------------------------------------------------------------------ dpe_ncc_eval
namespace {
// kDeviceCheck: queries in device memory, which the host cannot validate, are checked here; a
// query outside the problem gets NaN.
template <bool kDeviceCheck>
__global__ void k_ncc_queries(const PMArgs *__restrict__ pa, int64_t n, const int32_t *px, const int32_t *py,
                              const int32_t *src, const float4 *pl, float *out) {
  const PMArgs &a = *pa;
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  if (kDeviceCheck && (src[k] < 1 || src[k] >= a.N || px[k] < 0 || px[k] >= a.W || py[k] < 0 || py[k] >= a.H)) {
    out[k] = __int_as_float(0x7fffffff);
    return;
  }
  DPE_REF_WINDOW(rw);
  build_ref_window(a, px[k], py[k], rw, KID_NCC_QUERY);
  out[k] = ncc_strong(a, px[k], py[k], src[k], pl[k], rw);
}
}  // namespace

namespace {
// Host-side checks and the upload shared by the NCC query entry points: padded images, the
// argument block and the query arrays in the context's arena.
struct QueryUpload {
  PMArgs *d_args = nullptr;
  int32_t *px = nullptr, *py = nullptr, *src = nullptr;
  float4 *plane = nullptr;
};
int check_queries(const dpe_ncc_query *q) {
  if (!q || q->count < 0) return DPE_ERR_INVALID_ARGUMENT;
  if (q->num_images < 2 || q->num_images > DPE_MAX_IMAGES || q->width < 16 || q->height < 16) return DPE_ERR_INVALID_ARGUMENT;
  if (q->params.strong_increment <= 0 || q->params.strong_radius < 0 ||
      (2 * q->params.strong_radius) / q->params.strong_increment + 1 > kMaxWin)
    return DPE_ERR_INVALID_ARGUMENT;
  for (int64_t k = 0; k < q->count; ++k)
    if (q->src[k] < 1 || q->src[k] >= q->num_images || q->px[k] < 0 || q->px[k] >= q->width || q->py[k] < 0 ||
        q->py[k] >= q->height)
      return DPE_ERR_INVALID_ARGUMENT;
  return DPE_OK;
}
int upload_queries(dpe_ctx *ctx, const dpe_ncc_query *q, QueryUpload *u) {
  cudaStream_t s = ctx->stream;
  const int W = q->width, H = q->height, N = q->num_images;
  const size_t L = (size_t)W * H, PL = (size_t)(W + 2) * (H + 2);
  Arena &A = ctx->arena;
  PMArgs a;
  std::memset(&a, 0, sizeof(a));
  a.W = W; a.H = H; a.N = N; a.pad_w = W + 2;
  a.P = q->params;
  a.P.num_images = N;
  for (int i = 0; i < N; ++i) a.cam[i] = q->cameras[i];
  set_homography_bases(a);
  float *img_pad = A.get<float>("img_pad", PL * N);
  float *stage = A.get<float>("img_stage", L * N);
  const int64_t n = q->count;
  u->px = A.get<int32_t>("q_px", n);
  u->py = A.get<int32_t>("q_py", n);
  u->src = A.get<int32_t>("q_src", n);
  u->plane = A.get<float4>("q_plane", n);
  u->d_args = A.get<PMArgs>("pm_args", 1);
  if (!A.ok()) return DPE_ERR_OUT_OF_MEMORY;
  for (int i = 0; i < N; ++i) {
    DPE_TRY(cudaMemcpyAsync(stage + L * i, q->images[i], L * 4, cudaMemcpyHostToDevice, s));
    a.img[i] = img_pad + PL * i;
    k_pad_image<<<dim3((W + 2 + 31) / 32, (H + 2 + 7) / 8), dim3(32, 8), 0, s>>>(stage + L * i, img_pad + PL * i, W, H);
    PM_LAUNCHED("k_pad_image", s);
  }
  DPE_TRY(cudaMemcpyAsync(u->px, q->px, n * 4, cudaMemcpyHostToDevice, s));
  DPE_TRY(cudaMemcpyAsync(u->py, q->py, n * 4, cudaMemcpyHostToDevice, s));
  DPE_TRY(cudaMemcpyAsync(u->src, q->src, n * 4, cudaMemcpyHostToDevice, s));
  DPE_TRY(cudaMemcpyAsync(u->plane, q->plane, n * 16, cudaMemcpyHostToDevice, s));
  DPE_TRY(cudaMemcpyAsync(u->d_args, &a, sizeof(PMArgs), cudaMemcpyHostToDevice, s));
  return DPE_OK;
}

// Cost and gradients of each query (the adjoint of k_ncc_queries).  gdn: dC/d(depth, nx, ny, nz)
// with the depth at the pixel held instead of the plane offset w = -depth * (n . ray).
// kChecked: queries come from device memory the host has not read, so a pixel or source outside
// the problem gives NaN outputs instead of an access outside the images.
template <bool kChecked>
__global__ void k_ncc_grad(const PMArgs *__restrict__ pa, int64_t n, const int32_t *px, const int32_t *py,
                           const int32_t *src, const float4 *pl, const float *upstream, float *cost, float4 *gplane,
                           float4 *gdn, float *gimg) {
  const PMArgs &a = *pa;
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  if (kChecked && (src[k] < 1 || src[k] >= a.N || px[k] < 0 || px[k] >= a.W || py[k] < 0 || py[k] >= a.H)) {
    const float nan = __int_as_float(0x7fc00000);
    cost[k] = nan;
    if (gplane) gplane[k] = make_float4(nan, nan, nan, nan);
    if (gdn) gdn[k] = make_float4(nan, nan, nan, nan);
    return;
  }
  DPE_REF_WINDOW(rw);
  build_ref_window(a, px[k], py[k], rw, KID_NCC_QUERY);
  float g[4];
  const int s = src[k];
  const float4 p = pl[k];
  cost[k] = ncc_strong_adjoint(a, px[k], py[k], s, p, rw, g, gimg ? gimg + (size_t)(s - 1) * a.W * a.H : nullptr,
                               upstream ? upstream[k] : 1.0f);
  if (!gplane) return;
  gplane[k] = make_float4(g[0], g[1], g[2], g[3]);
  // w = -depth * (n . ray), ray = Kr^-1 (x, y, 1): dC/ddepth = g_w * -(n . ray); dC/dn|depth = g_n + g_w * -depth * ray
  const dpe_camera &c = a.cam[0];
  const float ray[3] = {((float)px[k] - c.K[2]) / c.K[0], ((float)py[k] - c.K[5]) / c.K[4], 1.0f};
  const float nr = p.x * ray[0] + p.y * ray[1] + p.z * ray[2];
  const float depth = nr != 0.0f ? -p.w / nr : 0.0f;
  if (gdn) gdn[k] = make_float4(-g[3] * nr, g[0] - g[3] * depth * ray[0], g[1] - g[3] * depth * ray[1], g[2] - g[3] * depth * ray[2]);
}
}  // namespace

extern "C" int dpe_ncc_eval(dpe_ctx *ctx, const dpe_ncc_query *q, float *costs_out) {
  if (!ctx || !costs_out) return DPE_ERR_INVALID_ARGUMENT;
  int st = check_queries(q);
  if (st) return st;
  if (q->count == 0) return DPE_OK;
  DPE_TRY(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  QueryUpload u;
  if ((st = upload_queries(ctx, q, &u))) return st;
  const int64_t n = q->count;
  float *dout = ctx->arena.get<float>("q_out", n);
  if (!dout) return DPE_ERR_OUT_OF_MEMORY;
  DPE_TIMED(ctx, KID_NCC_QUERY, s, k_ncc_queries<false><<<(unsigned)((n + 127) / 128), 128, 0, s>>>(u.d_args, n, u.px, u.py, u.src, u.plane, dout));
  PM_LAUNCHED("k_ncc_queries", s);
  DPE_TRY(cudaMemcpyAsync(costs_out, dout, n * 4, cudaMemcpyDeviceToHost, s));
  DPE_TRY(cudaStreamSynchronize(s));
  ctx->collect();
  return DPE_OK;
}

extern "C" int dpe_ncc_grad(dpe_ctx *ctx, const dpe_ncc_query *q, float *costs_out, float *grad_plane_out,
                            float *grad_depth_normal_out, float *const *grad_images_out) {
  if (!ctx || !costs_out || !grad_plane_out) return DPE_ERR_INVALID_ARGUMENT;
  int st = check_queries(q);
  if (st) return st;
  if (q->count == 0) return DPE_OK;
  DPE_TRY(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  QueryUpload u;
  if ((st = upload_queries(ctx, q, &u))) return st;
  const int64_t n = q->count;
  const size_t L = (size_t)q->width * q->height;
  Arena &A = ctx->arena;
  float *dcost = A.get<float>("q_out", n);
  float4 *dgp = A.get<float4>("q_gplane", n), *dgd = A.get<float4>("q_gdn", n);
  float *dgimg = grad_images_out ? A.get<float>("q_gimg", L * (q->num_images - 1)) : nullptr;
  if (!A.ok()) return DPE_ERR_OUT_OF_MEMORY;
  if (dgimg) DPE_TRY(cudaMemsetAsync(dgimg, 0, L * (q->num_images - 1) * 4, s));
  DPE_TIMED(ctx, KID_NCC_QUERY, s, k_ncc_grad<false><<<(unsigned)((n + 127) / 128), 128, 0, s>>>(u.d_args, n, u.px, u.py, u.src, u.plane, nullptr, dcost, dgp, dgd, dgimg));
  PM_LAUNCHED("k_ncc_grad", s);
  DPE_TRY(cudaMemcpyAsync(costs_out, dcost, n * 4, cudaMemcpyDeviceToHost, s));
  DPE_TRY(cudaMemcpyAsync(grad_plane_out, dgp, n * 16, cudaMemcpyDeviceToHost, s));
  if (grad_depth_normal_out) DPE_TRY(cudaMemcpyAsync(grad_depth_normal_out, dgd, n * 16, cudaMemcpyDeviceToHost, s));
  if (dgimg)
    for (int i = 1; i < q->num_images; ++i)
      if (grad_images_out[i])
        DPE_TRY(cudaMemcpyAsync(grad_images_out[i], dgimg + L * (i - 1), L * 4, cudaMemcpyDeviceToHost, s));
  DPE_TRY(cudaStreamSynchronize(s));
  ctx->collect();
  return DPE_OK;
}

extern "C" int dpe_ncc_grad_device(dpe_ctx *ctx, const dpe_ncc_query *q, const float *upstream, float *costs_out,
                                   float *grad_plane_out, float *grad_depth_normal_out, float *grad_images_out,
                                   void *stream) {
  if (!ctx || !q || !costs_out || q->count < 0) return DPE_ERR_INVALID_ARGUMENT;
  if (q->num_images < 2 || q->num_images > DPE_MAX_IMAGES || q->width < 16 || q->height < 16) return DPE_ERR_INVALID_ARGUMENT;
  if (q->params.strong_increment <= 0 || q->params.strong_radius < 0 ||
      (2 * q->params.strong_radius) / q->params.strong_increment + 1 > kMaxWin)
    return DPE_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < q->num_images; ++i)
    if (!q->images[i]) return DPE_ERR_INVALID_ARGUMENT;
  if (q->count > 0 && (!q->px || !q->py || !q->src || !q->plane)) return DPE_ERR_INVALID_ARGUMENT;
  if (q->count == 0) return DPE_OK;
  DPE_TRY(cudaSetDevice(ctx->device));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int W = q->width, H = q->height, N = q->num_images;
  const size_t L = (size_t)W * H, PL = (size_t)(W + 2) * (H + 2);
  Arena &A = ctx->arena;
  PMArgs a;
  std::memset(&a, 0, sizeof(a));
  a.W = W; a.H = H; a.N = N; a.pad_w = W + 2;
  a.P = q->params;
  a.P.num_images = N;
  for (int i = 0; i < N; ++i) a.cam[i] = q->cameras[i];
  set_homography_bases(a);
  float *img_pad = A.get<float>("gd_img_pad", PL * N);
  PMArgs *d_args = A.get<PMArgs>("gd_args", 1);
  if (!A.ok()) return DPE_ERR_OUT_OF_MEMORY;
  for (int i = 0; i < N; ++i) {
    a.img[i] = img_pad + PL * i;
    k_pad_image<<<dim3((W + 2 + 31) / 32, (H + 2 + 7) / 8), dim3(32, 8), 0, s>>>(q->images[i], img_pad + PL * i, W, H);
    PM_LAUNCHED("k_pad_image", s);
  }
  DPE_TRY(cudaMemcpyAsync(d_args, &a, sizeof(PMArgs), cudaMemcpyHostToDevice, s));
  if (grad_images_out) DPE_TRY(cudaMemsetAsync(grad_images_out, 0, L * (N - 1) * 4, s));
  const int64_t n = q->count;
  k_ncc_grad<true><<<(unsigned)((n + 127) / 128), 128, 0, s>>>(d_args, n, q->px, q->py, q->src,
                                                               reinterpret_cast<const float4 *>(q->plane), upstream,
                                                               costs_out, reinterpret_cast<float4 *>(grad_plane_out),
                                                               reinterpret_cast<float4 *>(grad_depth_normal_out),
                                                               grad_images_out);
  PM_LAUNCHED("k_ncc_grad", s);
  // the argument block is read by the kernels above: keep the host copy alive until they ran
  DPE_TRY(cudaStreamSynchronize(s));
  return DPE_OK;
}

// Diagnostics: per-kernel attributes (registers, local memory per thread, max block size) and the
// current per-thread stack limit, as text.  Reads attributes only; launches nothing.
extern "C" int dpe_kernel_info(char *buf, int len) {
  if (!buf || len <= 0) return DPE_ERR_INVALID_ARGUMENT;
  std::string s;
  auto add = [&](const char *name, const void *fn) {
    cudaFuncAttributes at;
    char line[256];
    if (cudaFuncGetAttributes(&at, fn) != cudaSuccess) {
      cudaGetLastError();
      std::snprintf(line, sizeof(line), "%s: attributes unavailable\n", name);
    } else {
      std::snprintf(line, sizeof(line), "%s: regs %d local %zu B shared %zu B max_threads %d\n", name, at.numRegs,
                    at.localSizeBytes, at.sharedSizeBytes, at.maxThreadsPerBlock);
    }
    s += line;
  };
  add("k_init_state", (const void *)k_init_state);
  add("k_gen_edge_inform", (const void *)k_gen_edge_inform);
  add("k_find_nearest_strong", (const void *)k_find_nearest_strong);
  add("k_gen_neighbours", (const void *)k_gen_neighbours);
  add("k_random_init", (const void *)k_random_init<DPE_STAGE_FP32>);
  add("k_strong_update", (const void *)k_strong_update<DPE_STAGE_FP32, false>);
  add("k_ransac_fit_plane", (const void *)k_ransac_fit_plane);
  add("k_weak_prepare", (const void *)k_weak_prepare);
  add("k_weak_eval", (const void *)k_weak_eval<false, DPE_STAGE_FP32>);
  add("k_weak_decide", (const void *)k_weak_decide);
  add("k_weak_finish", (const void *)k_weak_finish<DPE_STAGE_FP32>);
  add("k_filter_strong", (const void *)k_filter_strong);
  add("k_depth_to_weak", (const void *)k_depth_to_weak<DPE_STAGE_FP32>);
  add("k_local_refine", (const void *)k_local_refine<DPE_STAGE_FP32>);
  size_t stack = 0;
  cudaDeviceGetLimit(&stack, cudaLimitStackSize);
  char line[96];
  std::snprintf(line, sizeof(line), "stack limit %zu B\n", stack);
  s += line;
  std::snprintf(buf, (size_t)len, "%s", s.c_str());
  return DPE_OK;
}

// ------------------------------------------------------------------ allocation-free NCC queries
namespace {
// Scratch of dpe_ncc_eval_noalloc: the per-call argument block followed by the clamp-padded
// images.  Every GPU that loads the library holds these 16 MiB until the process exits.  Nothing
// in it needs to start at zero: each call writes the whole argument block and every padded texel
// it reads before the query kernel runs.
constexpr size_t kStaticScratchBytes = size_t(16) << 20;
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];
constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
unsigned char *g_static_addr[kMaxDevices] = {};

size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

// Writes the call's argument block into the static scratch.  The block travels as a kernel
// parameter (captured by value at launch), so no host buffer has to outlive the call.
__global__ void k_store_args(const __grid_constant__ PMArgs a, PMArgs *dst) {
  static_assert(sizeof(PMArgs) % 4 == 0, "argument block is copied as 32-bit words");
  const uint32_t *s = reinterpret_cast<const uint32_t *>(&a);
  uint32_t *d = reinterpret_cast<uint32_t *>(dst);
  for (int i = threadIdx.x; i < (int)(sizeof(PMArgs) / 4); i += blockDim.x) d[i] = s[i];
}
}  // namespace

extern "C" int dpe_ncc_eval_noalloc(const dpe_ncc_query *q, float *costs_out, void *stream) {
  if (!q || !costs_out || q->count < 0) return DPE_ERR_INVALID_ARGUMENT;
  if (q->num_images < 2 || q->num_images > DPE_MAX_IMAGES || q->width < 16 || q->height < 16) return DPE_ERR_INVALID_ARGUMENT;
  if (q->params.strong_increment <= 0 || q->params.strong_radius < 0 ||
      (2 * q->params.strong_radius) / q->params.strong_increment + 1 > kMaxWin)
    return DPE_ERR_INVALID_ARGUMENT;
  const int W = q->width, H = q->height, N = q->num_images;
  for (int i = 0; i < N; ++i)
    if (!q->images[i]) return DPE_ERR_INVALID_ARGUMENT;
  if (q->count > 0 && (!q->px || !q->py || !q->src || !q->plane)) return DPE_ERR_INVALID_ARGUMENT;
  const size_t PL = (size_t)(W + 2) * (H + 2);
  const size_t img_bytes = round256(PL * sizeof(float));
  const size_t need = round256(sizeof(PMArgs)) + (size_t)N * img_bytes;
  if (need > kStaticScratchBytes) {
    char buf[200];
    std::snprintf(buf, sizeof(buf), "dpe_ncc_eval_noalloc: %d padded %dx%d images need %zu bytes of scratch; the "
                  "static array holds %zu", N, W + 2, H + 2, need, kStaticScratchBytes);
    g_last_error = buf;
    return DPE_ERR_CAPACITY;
  }
  if (q->count == 0) return DPE_OK;
  int dev = 0;
  DPE_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return DPE_ERR_NO_DEVICE;
  unsigned char *base = nullptr;
  {
    // one-time set-up per device, with that device current: the device address of the array
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_addr[dev]) {
      void *ptr = nullptr;
      DPE_TRY(cudaGetSymbolAddress(&ptr, g_static_scratch));
      g_static_addr[dev] = static_cast<unsigned char *>(ptr);
    }
    base = g_static_addr[dev];
  }
  PMArgs a;
  std::memset(&a, 0, sizeof(a));
  a.W = W; a.H = H; a.N = N; a.pad_w = W + 2;
  a.P = q->params;
  a.P.num_images = N;
  for (int i = 0; i < N; ++i) a.cam[i] = q->cameras[i];
  set_homography_bases(a);
  unsigned char *img_base = base + round256(sizeof(PMArgs));
  for (int i = 0; i < N; ++i) a.img[i] = reinterpret_cast<const float *>(img_base + (size_t)i * img_bytes);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_store_args<<<1, 256, 0, s>>>(a, reinterpret_cast<PMArgs *>(base));
  DPE_LAUNCHED("k_store_args", s);
  for (int i = 0; i < N; ++i) {
    k_pad_image<<<dim3((W + 2 + 31) / 32, (H + 2 + 7) / 8), dim3(32, 8), 0, s>>>(
        q->images[i], reinterpret_cast<float *>(img_base + (size_t)i * img_bytes), W, H);
    DPE_LAUNCHED("k_pad_image", s);
  }
  const int64_t n = q->count;
  k_ncc_queries<true><<<(unsigned)((n + 127) / 128), 128, 0, s>>>(reinterpret_cast<const PMArgs *>(base), n, q->px,
                                                                    q->py, q->src,
                                                                    reinterpret_cast<const float4 *>(q->plane),
                                                                    costs_out);
  DPE_LAUNCHED("k_ncc_queries", s);
  return DPE_OK;
}

// ------------------------------------------------------------------ statistics
extern "C" int dpe_ctx_set_options(dpe_ctx *ctx, const dpe_options *opt) {
  if (!ctx || !opt) return DPE_ERR_INVALID_ARGUMENT;
  if (opt->staging != DPE_STAGE_FP32 && opt->staging != DPE_STAGE_FP16 && opt->staging != DPE_STAGE_BF16)
    return DPE_ERR_INVALID_ARGUMENT;
  if (opt->gn_refine != 0 && opt->gn_refine != 1) return DPE_ERR_INVALID_ARGUMENT;
  ctx->opt = *opt;
  return DPE_OK;
}

extern "C" int dpe_ctx_set_profiling(dpe_ctx *ctx, int on) {
  if (!ctx) return DPE_ERR_INVALID_ARGUMENT;
  ctx->profile = on != 0;
  return DPE_OK;
}

extern "C" int dpe_ctx_reset_kernel_stats(dpe_ctx *ctx) {
  if (!ctx) return DPE_ERR_INVALID_ARGUMENT;
  for (int k = 0; k < KID_COUNT; ++k) {
    ctx->kms[k] = 0.0;
    ctx->klaunch[k] = 0;
    ctx->kevals[k][0] = ctx->kevals[k][1] = 0;
  }
  return DPE_OK;
}

extern "C" int dpe_ctx_get_kernel_stats(dpe_ctx *ctx, dpe_kernel_stat *out, int capacity, int *count) {
  if (!ctx || !count || (capacity > 0 && !out)) return DPE_ERR_INVALID_ARGUMENT;
  int n = 0;
  for (int k = 0; k < KID_COUNT; ++k) {
    if (ctx->klaunch[k] == 0 && ctx->kevals[k][0] == 0 && ctx->kevals[k][1] == 0) continue;
    if (n < capacity) {
      std::snprintf(out[n].name, sizeof(out[n].name), "%s", kKernelNames[k]);
      out[n].launches = ctx->klaunch[k];
      out[n].ms = ctx->kms[k];
      out[n].strong_ncc_evals = ctx->kevals[k][0];
      out[n].weak_ncc_evals = ctx->kevals[k][1];
    }
    ++n;
  }
  *count = n;
  return n > capacity ? DPE_ERR_CAPACITY : DPE_OK;
}

extern "C" int dpe_ctx_set_autotune(dpe_ctx *ctx, int on) {
  if (!ctx) return DPE_ERR_INVALID_ARGUMENT;
  ctx->tuner.enabled = on != 0;
  return DPE_OK;
}

extern "C" int dpe_ctx_get_tuning(dpe_ctx *ctx, dpe_tuning_entry *out, int capacity, int *count) {
  if (!ctx || !count || (capacity > 0 && !out)) return DPE_ERR_INVALID_ARGUMENT;
  int n = 0;
  for (auto &kv : ctx->tuner.table) {
    TuneEntry &e = kv.second;
    tune_harvest(ctx, e);
    if (n < capacity) {
      dpe_tuning_entry &o = out[n];
      std::memset(&o, 0, sizeof(o));
      const int kid = (int)(kv.first / 64);
      std::snprintf(o.name, sizeof(o.name), "%s", kid >= 0 && kid < KID_COUNT ? kKernelNames[kid] : "?");
      o.size_class = (int)(kv.first % 64);
      o.candidates = e.ncand;
      o.chosen = e.chosen;
      const bool carve = kid == KID_STRONG_UPDATE || kid == KID_DEPTH_TO_WEAK || kid == KID_LOCAL_REFINE;
      if (e.chosen >= 0) {
        if (carve) o.carveout = kCarveCands[e.chosen];
        else { o.block_x = (int)kShapeCands[e.chosen].x; o.block_y = (int)kShapeCands[e.chosen].y; }
      }
      for (int i = 0; i < e.ncand && i < 8; ++i) o.mean_ms[i] = e.count[i] ? (float)(e.sum[i] / e.count[i]) : 0.f;
    }
    ++n;
  }
  *count = n;
  return n > capacity ? DPE_ERR_CAPACITY : DPE_OK;
}

namespace {
// 8 independent FMA chains per thread; 2 FLOP per FMA.
__global__ void k_fma_throughput(float *out, int iters, float a, float b) {
  float x0 = threadIdx.x * 1e-3f, x1 = x0 + 1.f, x2 = x0 + 2.f, x3 = x0 + 3.f;
  float x4 = x0 + 4.f, x5 = x0 + 5.f, x6 = x0 + 6.f, x7 = x0 + 7.f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
      x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
    }
  }
  const float r = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (r == 1234.5f) out[blockIdx.x] = r;
}
}  // namespace

extern "C" int dpe_fp32_peak(dpe_ctx *ctx, double *tflops) {
  if (!ctx || !tflops) return DPE_ERR_INVALID_ARGUMENT;
  DPE_TRY(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  int sms = 0;
  DPE_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
  float *out = ctx->arena.get<float>("fma_out", 4096);
  if (!out) return DPE_ERR_OUT_OF_MEMORY;
  const int blocks = sms * 8, threads = 256, iters = 4096;
  double best = 0.0;
  for (int rep = 0; rep < 4; ++rep) {
    DPE_TRY(cudaEventRecord(ctx->ev0, s));
    k_fma_throughput<<<blocks, threads, 0, s>>>(out, iters, 0.999f, 1e-3f);
    DPE_LAUNCHED("k_fma_throughput", s);
    DPE_TRY(cudaEventRecord(ctx->ev1, s));
    DPE_TRY(cudaEventSynchronize(ctx->ev1));
    float ms = 0.f;
    DPE_TRY(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    const double flops = 2.0 * 32.0 * (double)iters * blocks * threads;
    if (rep > 0) best = std::max(best, flops / (ms * 1e-3) / 1e12);
  }
  *tflops = best;
  return DPE_OK;
}

// Statistics switch: count NCC evaluations in dpe_pm_run (adds device atomics; off by default).
extern "C" int dpe_ctx_set_eval_counting(dpe_ctx *ctx, int on) {
  if (!ctx) return DPE_ERR_INVALID_ARGUMENT;
  ctx->count_evals = on != 0;
  return DPE_OK;
}
