// kernel_host.cpp -- TEST INFRASTRUCTURE: the CUDA PatchMatch kernel source compiled for the host.
//
// Every kernel of dpe-mvs-fast_b200/csrc/pm_kernels.cuh is executed here thread by thread on the
// CPU, in the launch order of dpe_pm_run, so that the kernels' logic can be compared with the
// oracle without a GPU (bit for bit: both sides run IEEE float without contraction) and checked
// under AddressSanitizer / UBSan.  The few device intrinsics the kernels use get host stand-ins.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

using std::max;
using std::min;
static dim3 blockIdx, threadIdx, blockDim, gridDim;
#undef __global__
#undef __device__
#undef __host__
#undef __forceinline__
#undef __launch_bounds__
#undef __grid_constant__
#undef __constant__
#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __launch_bounds__(...)
#define __grid_constant__
#define __constant__
#define __restrict__
static inline unsigned __umulhi(unsigned a, unsigned b) { return (unsigned)(((unsigned long long)a * b) >> 32); }
template <class T> static inline T __ldg(const T *p) { return *p; }
// Kernels with block barriers run here only through launch_phased (their phases in lock-step); a
// sequential launch of one would ignore its barriers, so the stand-in refuses to run.
static inline void __syncthreads() { std::abort(); }
static inline int __syncthreads_or(int) { std::abort(); }
static inline unsigned atomicOr(unsigned *, unsigned) { std::abort(); }
// the device's correctly rounded, never-contracted arithmetic intrinsics
static inline float __fmul_rn(float a, float b) { volatile float r = a * b; return r; }
static inline float __fadd_rn(float a, float b) { volatile float r = a + b; return r; }
static inline float __fsub_rn(float a, float b) { volatile float r = a - b; return r; }
static inline float __fdiv_rn(float a, float b) { volatile float r = a / b; return r; }
static inline float __fsqrt_rn(float a) { volatile float r = std::sqrt(a); return r; }
static inline unsigned long long atomicAdd(unsigned long long *p, unsigned long long v) {
  const unsigned long long o = *p;
  *p += v;
  return o;
}
static inline unsigned int __float_as_uint(float f) {
  unsigned int u;
  std::memcpy(&u, &f, 4);
  return u;
}
static inline float __uint_as_float(unsigned int u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}
static inline float atomicAdd(float *p, float v) {
  const float o = *p;
  *p += v;
  return o;
}
using std::isnan;
using std::isfinite;
#include "../../dpe-mvs-fast_b200/csrc/pm_kernels.cuh"
using namespace dpe;

template <class K, class... Args> static void launch(dim3 grid, dim3 block, K k, Args... args) {
  blockDim = block;
  gridDim = grid;
  for (unsigned by = 0; by < grid.y; ++by)
    for (unsigned bx = 0; bx < grid.x; ++bx)
      for (unsigned ty = 0; ty < block.y; ++ty)
        for (unsigned tx = 0; tx < block.x; ++tx) {
          blockIdx = dim3(bx, by, 1);
          threadIdx = dim3(tx, ty, 1);
          k(args...);
        }
}
// A block-cooperative kernel given as phases (the code between its barriers): every thread of a
// block runs phase p before any runs phase p + 1, over one zeroed shared-memory buffer per block.
template <class F> static void launch_phased(dim3 grid, dim3 block, size_t smem_bytes, int phases, F phase) {
  blockDim = block;
  gridDim = grid;
  std::vector<float4> smem((smem_bytes + 15) / 16);
  for (unsigned by = 0; by < grid.y; ++by)
    for (unsigned bx = 0; bx < grid.x; ++bx) {
      std::fill(smem.begin(), smem.end(), float4{0, 0, 0, 0});
      for (int p = 0; p < phases; ++p)
        for (unsigned ty = 0; ty < block.y; ++ty)
          for (unsigned tx = 0; tx < block.x; ++tx) {
            blockIdx = dim3(bx, by, 1);
            threadIdx = dim3(tx, ty, 1);
            phase(p, smem.data());
          }
    }
}
template <class T> static T *alloc(size_t n) { return (T *)calloc(n, sizeof(T)); }

// The kernel sequence of dpe_pm_run (dpe-mvs-fast_b200/csrc/capi.cu), host memory only.
extern "C" int host_pm_run(const dpe_problem *p, dpe_pm_out *out) {
  const int W = p->width, H = p->height, N = p->num_images;
  const size_t L = (size_t)W * H, PL = (size_t)(W + 2) * (H + 2);
  PMArgs a;
  memset(&a, 0, sizeof(a));
  a.W = W; a.H = H; a.N = N; a.pad_w = W + 2;
  a.P = p->params;
  a.P.num_images = N;
  for (int i = 0; i < N; ++i) a.cam[i] = p->cameras[i];
  set_homography_bases(a);
  a.key[0] = (uint32_t)p->seed;
  a.key[1] = (uint32_t)(p->seed >> 32);
  std::vector<float *> imgs;
  for (int i = 0; i < N; ++i) {
    float *d = alloc<float>(PL);
    launch(dim3((W + 2 + 31) / 32, (H + 2 + 7) / 8), dim3(32, 8), k_pad_image, p->images[i], d, W, H);
    a.img[i] = d;
    imgs.push_back(d);

    if (a.P.geom_consistency) a.dep[i] = p->depths[i];
  }
  a.plane = alloc<float4>(L); a.plane_snap = alloc<float4>(L); a.fit_plane = alloc<float4>(L);
  a.cost = alloc<float>(L); a.cost_snap = alloc<float>(L); a.complexity = alloc<float>(L);
  a.views = alloc<uint32_t>(L); a.rng_ctr = alloc<uint32_t>(L); a.vweight = alloc<uint4>(L);
  a.weak = alloc<uint8_t>(L); a.reliable = alloc<uint8_t>(L); a.nmap = alloc<int32_t>(L); a.radius = alloc<int32_t>(L);
  int *weak_flag = alloc<int>(L);
  a.neigh = alloc<short2>(L * kNeighbours); a.lab_bound = alloc<short2>(L * 8);
  a.edge_neigh = alloc<short2>(L * 8); a.nearest = alloc<short2>(L);
  const Launch one{&a, nullptr, 1};
  a.lowW = p->low_width; a.lowH = p->low_height;
  a.edge = p->edge; a.edge_low = p->edge_low_res; a.label = p->label;
  const dim3 fg((W + 15) / 16, (H + 7) / 8), fb(16, 8), hg((W + 31) / 32, ((H + 1) / 2 + 3) / 4), hb(32, 4);
  launch(fg, fb, k_init_state, one, (const float4 *)p->plane_in, p->selected_views_in, p->weak_in, weak_flag);
  int acc = 0;
  for (size_t i = 0; i < L; ++i) { a.nmap[i] = acc; acc += weak_flag[i]; }
  launch(fg, fb, k_gen_edge_inform, one);
  launch(fg, fb, k_find_nearest_strong, one);
  launch(fg, fb, k_gen_neighbours, one);
  const dim3 lg(7), lb(32);  // strided work lists: any grid covers them
  launch(fg, fb, k_neighbour_update, one);
  // WEAK pixels per colour in raster order (the cub select of dpe_pm_run)
  const size_t wcap = (L + 1) / 2;
  std::vector<int> wlist(2 * wcap), wcount(2, 0);
  std::vector<float2> wtab;
  std::vector<float4> wwin, whyp, wstate;
  std::vector<float> wcost, wgeom, wcost_r, wgeom_r;
  if (a.P.use_APD) {
    for (size_t i = 0; i < L; ++i) {
      const int x = (int)(i % W), y = (int)(i / W), c = (x + y) & 1;
      if (a.weak[i] == DPE_WEAK) wlist[c * wcap + wcount[c]++] = (int)i;
    }
    const int n = N - 1, side = (2 * a.P.weak_radius) / a.P.weak_increment + 1;
    a.wtaps = side * side;
    a.wtab_stride = kMaxWin * kMaxWin + 8 * a.wtaps;
    wtab.resize(wcap * a.wtab_stride); wwin.resize(wcap * kNeighbours); whyp.resize(wcap * 5);
    wstate.resize(wcap * 2); wcost.resize(wcap * 10 * n); wgeom.resize(wcap * 10 * n);
    wcost_r.resize(wcap * 5 * n); wgeom_r.resize(wcap * 5 * n);
    a.wlist[0] = wlist.data(); a.wlist[1] = wlist.data() + wcap; a.wcount = wcount.data();
    a.wtab = wtab.data(); a.wwin = wwin.data(); a.whyp = whyp.data(); a.wstate = wstate.data();
    a.wcost = wcost.data(); a.wgeom = wgeom.data(); a.wcost_r = wcost_r.data(); a.wgeom_r = wgeom_r.data();
  }
  launch(fg, fb, k_random_init<DPE_STAGE_FP32>, one);
  for (int it = 0; it < a.P.max_iterations; ++it) {
    for (int parity = 0; parity < 2; ++parity) {
      if (a.P.use_edge) { memcpy(a.plane_snap, a.plane, L * 16); memcpy(a.cost_snap, a.cost, L * 4); }
      launch_phased(dim3((W + kCoopPix - 1) / kCoopPix, (H + 1) / 2), dim3(kCoopThreads), coop_smem_bytes(N - 1),
                    kStrongPhases, [&](int ph, void *sm) {
                      strong_update_phase<DPE_STAGE_FP32, false>(ph, one, it, parity, sm);
                    });
    }
    launch(fg, fb, k_ransac_fit_plane, one);
    if (a.P.use_APD)
      for (int parity = 0; parity < 2; ++parity) {
        launch(lg, lb, k_weak_prepare, one, parity);
        launch(lg, lb, k_weak_eval<false, DPE_STAGE_FP32>, one, parity);
        launch(lg, lb, k_weak_decide, one, it, parity);
        launch(lg, lb, k_weak_eval<true, DPE_STAGE_FP32>, one, parity);
        launch(lg, lb, k_weak_finish<DPE_STAGE_FP32>, one, parity);
      }
  }
  launch(fg, fb, k_get_depth_normal, one);
  for (int parity = 0; parity < 2; ++parity) launch(hg, hb, k_filter_strong, one, parity);
  const dim3 sg((W + kCoopPix - 1) / kCoopPix, H);
  launch_phased(sg, dim3(kCoopThreads), sizeof(SweepPixel) * kCoopPix, kSweepPhases,
                [&](int ph, void *sm) { depth_to_weak_phase<DPE_STAGE_FP32>(ph, one, sm); });
  launch_phased(sg, dim3(kCoopThreads), local_refine_smem_bytes(N - 1), kSweepPhases,
                [&](int ph, void *sm) { local_refine_phase<DPE_STAGE_FP32>(ph, one, sm); });
  memcpy(out->plane, a.plane, L * 16);
  memcpy(out->weak, a.weak, L);
  memcpy(out->selected_views, a.views, L * 4);
  if (out->costs) memcpy(out->costs, a.cost, L * 4);
  for (float *d : imgs) free(d);
  free(a.plane); free(a.plane_snap); free(a.fit_plane); free(a.cost); free(a.cost_snap); free(a.complexity);
  free(a.views); free(a.rng_ctr); free(a.vweight); free(a.weak); free(a.reliable); free(a.nmap); free(a.radius);
  free(weak_flag); free(a.neigh); free(a.lab_bound); free(a.edge_neigh); free(a.nearest);
  return 0;
}
