// scene.cu -- the whole-scene schedule with device-resident state (dpe_scene_run).
//
// The reference runs main()'s loop on the host: per pyramid level one FIRST_INIT/REFINE_INIT
// call and three geom REFINE_ITER calls for every view (main.cpp:385-457), each call uploading its
// inputs, running RunPatchMatch and downloading planes/weak/views into the StateStore; then
// RunFusion.  Here the image pyramid, the StateStore, ProcessProblem's result assembly and the
// nearest-neighbour state rescale between levels live on the device, and every call reads its
// inputs from and writes its result to HBM.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "ctx.h"

namespace {

// u8 -> float (Mat::convertTo, CV_32FC1)
__global__ void k_gray_to_float(const uint8_t *__restrict__ src, float *__restrict__ dst, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (float)src[i];
}

// cv::resize INTER_LINEAR on a float image (SceneCache::GetGrayFloatImage, DPE.cpp:728-735):
// source coordinate (d + 0.5) * scale - 0.5, clamped at the borders, horizontal then vertical.
__global__ void k_resize_linear(const float *__restrict__ src, int sw, int sh, float *__restrict__ dst, int dw, int dh,
                                double scale_x, double scale_y) {
  const int dx = blockIdx.x * blockDim.x + threadIdx.x;
  const int dy = blockIdx.y * blockDim.y + threadIdx.y;
  if (dx >= dw || dy >= dh) return;
  float fx = (float)((dx + 0.5) * scale_x - 0.5);
  int sx = (int)floorf(fx);
  fx -= sx;
  if (sx < 0) { fx = 0.f; sx = 0; }
  if (sx >= sw - 1) { fx = 0.f; sx = sw - 1; }
  float fy = (float)((dy + 0.5) * scale_y - 0.5);
  int sy = (int)floorf(fy);
  fy -= sy;
  if (sy < 0) { fy = 0.f; sy = 0; }
  if (sy >= sh - 1) { fy = 0.f; sy = sh - 1; }
  const int sx1 = min(sx + 1, sw - 1), sy1 = min(sy + 1, sh - 1);
  const float *r0 = src + (size_t)sy * sw, *r1 = src + (size_t)sy1 * sw;
  const float h0 = r0[sx] * (1.f - fx) + r0[sx1] * fx;
  const float h1 = r1[sx] * (1.f - fx) + r1[sx1] * fx;
  dst[(size_t)dy * dw + dx] = h0 * (1.f - fy) + h1 * fy;
}

// RescaleMatToTargetSize (DPE.cpp:1313-1335): nearest neighbour with o = (int)(r / scale).
template <class T>
__global__ void k_rescale_nearest(const T *__restrict__ src, int sw, int sh, T *__restrict__ dst, int dw, int dh) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y * blockDim.y + threadIdx.y;
  if (c >= dw || r >= dh) return;
  const float scale_x = dw / (float)sw, scale_y = dh / (float)sh;
  const int oc = (int)(c / scale_x), orow = (int)(r / scale_y);
  if (orow < 0 || oc < 0 || orow >= sh || oc >= sw) return;
  dst[(size_t)r * dw + c] = src[(size_t)orow * sw + oc];
}

// ProcessProblem's result assembly (main.cpp:266-279): depths outside [dmin, dmax] become 0 and
// their pixels UNKNOWN; the state keeps (world normal, depth), the view mask and the pixel state.
__global__ void k_store_result(const float4 *__restrict__ plane, const uint8_t *__restrict__ weak_in,
                               const uint32_t *__restrict__ views_in, int n, float dmin, float dmax,
                               float4 *__restrict__ st_plane, float *__restrict__ st_depth, uint8_t *__restrict__ st_weak,
                               uint32_t *__restrict__ st_views) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 p = plane[i];
  uint8_t w = weak_in[i];
  if (p.w < dmin || p.w > dmax) {
    p.w = 0.0f;
    w = DPE_UNKNOWN;
  }
  st_plane[i] = p;
  st_depth[i] = p.w;
  st_weak[i] = w;
  st_views[i] = views_in[i];
}

__global__ void k_depth_from_plane(const float4 *__restrict__ plane, float *__restrict__ depth, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) depth[i] = plane[i].w;
}

__global__ void k_split_normal(const float4 *__restrict__ plane, float *__restrict__ normal, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 p = plane[i];
  normal[3 * i] = p.x;
  normal[3 * i + 1] = p.y;
  normal[3 * i + 2] = p.z;
}

uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// ComputeRoundNum (main.cpp:223-238)
int round_num(int W, int H) {
  int m = std::max(W, H), r = 1;
  while (m > 800) { m /= 2; r++; }
  return r;
}

// SceneCache::GetCamera scaling of K to the target size (DPE.cpp:739-760)
dpe_camera camera_at(const dpe_camera &c0, int W0, int H0, int w, int h) {
  dpe_camera c = c0;
  const float sx = w / (float)W0, sy = h / (float)H0;
  c.K[0] *= sx; c.K[2] *= sx; c.K[4] *= sy; c.K[5] *= sy;
  c.width = w; c.height = h;
  return c;
}

struct ViewState {
  float *img;   // float gray at the current level
  float4 *plane;
  float *depth;
  uint8_t *weak;
  uint32_t *views;
};

}  // namespace

extern "C" int dpe_scene_run(dpe_ctx *ctx, const dpe_scene *sc, const dpe_schedule *sch, dpe_scene_out *out) {
  if (!ctx || !sc || !sch || !out || sc->num_views < 2 || !sc->views) return DPE_ERR_INVALID_ARGUMENT;
  if (sc->memory != DPE_MEM_HOST && sc->memory != DPE_MEM_DEVICE) return DPE_ERR_INVALID_ARGUMENT;
  const int V = sc->num_views, W = sc->width, H = sc->height;
  if (W < 16 || H < 16) return DPE_ERR_INVALID_ARGUMENT;
  const int L = sch->num_levels > 0 ? sch->num_levels : round_num(W, H);
  if (L > 8 || (W >> (L - 1)) < 16 || (H >> (L - 1)) < 16) return DPE_ERR_INVALID_ARGUMENT;
  if (sch->refine_calls < 0 || sch->max_iterations < 0) return DPE_ERR_INVALID_ARGUMENT;
  if (sch->batch_views != 0 && sch->batch_views != 1) return DPE_ERR_INVALID_ARGUMENT;
  if (sch->batch_views && sc->num_views > DPE_MAX_BATCH) return DPE_ERR_INVALID_ARGUMENT;
  if (sch->device_edges != 0 && sch->device_edges != 1) return DPE_ERR_INVALID_ARGUMENT;
  if (sch->device_labels != 0 && sch->device_labels != 1) return DPE_ERR_INVALID_ARGUMENT;
  const bool given_edges = sc->views[0].edges != nullptr, given_labels = sc->views[0].labels != nullptr;
  if ((sch->device_edges && given_edges) || (sch->device_labels && given_labels)) return DPE_ERR_INVALID_ARGUMENT;
  const bool have_edges = given_edges || sch->device_edges;
  const bool have_labels = given_labels || sch->device_labels;
  for (int v = 0; v < V; ++v) {
    const dpe_scene_view &sv = sc->views[v];
    if (!sv.gray || sv.num_src < 1 || sv.num_src > DPE_MAX_IMAGES - 1 || !sv.src_views) return DPE_ERR_INVALID_ARGUMENT;
    for (int j = 0; j < sv.num_src; ++j)
      if (sv.src_views[j] < 0 || sv.src_views[j] >= V || sv.src_views[j] == v) return DPE_ERR_INVALID_ARGUMENT;
    if ((sv.edges != nullptr) != given_edges || (sv.labels != nullptr) != given_labels) return DPE_ERR_INVALID_ARGUMENT;
    if (sch->fuse_mode >= 0 && !sv.bgr) return DPE_ERR_INVALID_ARGUMENT;
  }
  DPE_TRY(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  Arena &A = ctx->arena;
  const bool host = sc->memory == DPE_MEM_HOST;
  const size_t LF = (size_t)W * H;

  // PatchMatchParams::high_res_img, which selects EdgeSegment's downsampling
  int high_res_img = 1;
  {
    dpe_params d;
    dpe_params_default(&d);
    high_res_img = d.high_res_img ? 1 : 0;
  }
  if (sch->device_labels && ((W / (high_res_img ? 4 : 2)) < 1 || (H / (high_res_img ? 4 : 2)) < 1))
    return DPE_ERR_INVALID_ARGUMENT;

  // level sizes (SceneCache::GetGrayFloatImage: round(cols / scale_size))
  std::vector<int> lw(L), lh(L), lscale(L);
  for (int l = 0; l < L; ++l) {
    lscale[l] = 1 << (L - 1 - l);
    const float f = 1.0f / (float)lscale[l];
    lw[l] = (int)std::lround(W * f);
    lh[l] = (int)std::lround(H * f);
  }

  // ---- device buffers
  std::vector<ViewState> st(V);
  uint8_t *gray_dev = host ? A.get<uint8_t>("sc_gray", LF * V) : nullptr;
  float *gray_full = A.get<float>("sc_grayf", LF * V);
  float *img_lvl = A.get<float>("sc_img", LF * V);
  float4 *planes = A.get<float4>("sc_plane", LF * V);
  float4 *planes_tmp = A.get<float4>("sc_plane_tmp", LF);
  float *depths = A.get<float>("sc_depth", LF * V);
  uint8_t *weaks = A.get<uint8_t>("sc_weak", LF * V);
  uint8_t *weak_tmp = A.get<uint8_t>("sc_weak_tmp", LF);
  uint32_t *views = A.get<uint32_t>("sc_views", LF * V);
  uint32_t *views_tmp = A.get<uint32_t>("sc_views_tmp", LF);
  float4 *out_plane = A.get<float4>("sc_out_plane", LF);
  uint8_t *out_weak = A.get<uint8_t>("sc_out_weak", LF);
  uint32_t *out_views = A.get<uint32_t>("sc_out_views", LF);
  // per-view outputs of a batched call
  float4 *bout_plane = sch->batch_views ? A.get<float4>("sc_bout_plane", LF * V) : nullptr;
  uint8_t *bout_weak = sch->batch_views ? A.get<uint8_t>("sc_bout_weak", LF * V) : nullptr;
  uint32_t *bout_views = sch->batch_views ? A.get<uint32_t>("sc_bout_views", LF * V) : nullptr;
  if (!A.ok()) return DPE_ERR_OUT_OF_MEMORY;
  for (int v = 0; v < V; ++v)
    st[v] = ViewState{img_lvl + LF * v, planes + LF * v, depths + LF * v, weaks + LF * v, views + LF * v};

  // edge / label maps per level (uploaded when given in host memory)
  std::vector<std::vector<const uint8_t *>> edge(V, std::vector<const uint8_t *>(L, nullptr));
  std::vector<std::vector<const int32_t *>> label(V, std::vector<const int32_t *>(L, nullptr));
  if (have_edges || have_labels) {
    size_t per_view = 0;
    for (int l = 0; l < L; ++l) per_view += (size_t)lw[l] * lh[l];
    uint8_t *e_dev = ((host && given_edges) || sch->device_edges) ? A.get<uint8_t>("sc_edges", per_view * V) : nullptr;
    if (sch->device_edges && dpe_edge_reserve(ctx, (size_t)lw[L - 1] * lh[L - 1]) != DPE_OK) return DPE_ERR_OUT_OF_MEMORY;
    int32_t *l_dev = ((host && given_labels) || sch->device_labels) ? A.get<int32_t>("sc_labels", per_view * V) : nullptr;
    if (!A.ok()) return DPE_ERR_OUT_OF_MEMORY;
    size_t off = 0;
    for (int v = 0; v < V; ++v)
      for (int l = 0; l < L; ++l) {
        const size_t n = (size_t)lw[l] * lh[l];
        if (sch->device_edges) {
          edge[v][l] = e_dev + off;  // made when the level image is
        } else if (have_edges) {
          if (host) {
            DPE_TRY(cudaMemcpyAsync(e_dev + off, sc->views[v].edges[l], n, cudaMemcpyHostToDevice, s));
            edge[v][l] = e_dev + off;
          } else {
            edge[v][l] = sc->views[v].edges[l];
          }
        }
        if (sch->device_labels) {
          label[v][l] = l_dev + off;  // made at the start of the level
        } else if (have_labels) {
          if (host) {
            DPE_TRY(cudaMemcpyAsync(l_dev + off, sc->views[v].labels[l], n * 4, cudaMemcpyHostToDevice, s));
            label[v][l] = l_dev + off;
          } else {
            label[v][l] = sc->views[v].labels[l];
          }
        }
        off += n;
      }
  }
  for (int v = 0; v < V; ++v) {
    const uint8_t *g = sc->views[v].gray;
    if (host) {
      DPE_TRY(cudaMemcpyAsync(gray_dev + LF * v, g, LF, cudaMemcpyHostToDevice, s));
      g = gray_dev + LF * v;
    }
    k_gray_to_float<<<(unsigned)((LF + 255) / 256), 256, 0, s>>>(g, gray_full + LF * v, (int)LF);
    DPE_LAUNCHED("k_gray_to_float", s);
  }

  cudaEvent_t e0, e1, ef;
  DPE_TRY(cudaEventCreate(&e0));
  DPE_TRY(cudaEventCreate(&e1));
  DPE_TRY(cudaEventCreate(&ef));
  struct EventGuard {
    cudaEvent_t a, b, c;
    ~EventGuard() { cudaEventDestroy(a); cudaEventDestroy(b); cudaEventDestroy(c); }
  } guard{e0, e1, ef};
  DPE_TRY(cudaEventRecord(e0, s));

  int calls = 0;
  const dim3 b2(32, 8);
  for (int l = 0; l < L; ++l) {
    const int w = lw[l], h = lh[l];
    const size_t n = (size_t)w * h;
    const dim3 g2((w + 31) / 32, (h + 7) / 8);
    // image pyramid level
    for (int v = 0; v < V; ++v) {
      if (lscale[l] == 1) {
        DPE_TRY(cudaMemcpyAsync(st[v].img, gray_full + LF * v, LF * 4, cudaMemcpyDeviceToDevice, s));
      } else {
        k_resize_linear<<<g2, b2, 0, s>>>(gray_full + LF * v, W, H, st[v].img, w, h, (double)W / w, (double)H / h);
        DPE_LAUNCHED("k_resize_linear", s);
      }
      // the level's edge map (GetProblemEdges computes it from this same resize, main.cpp:170-178)
      if (sch->device_edges) {
        const int est = dpe_edge_map_device(ctx, st[v].img, nullptr, w, h, const_cast<uint8_t *>(edge[v][l]));
        if (est != DPE_OK) return est;
      }
      // and its label map, from the full-resolution 8-bit image (main.cpp:199-214)
      if (sch->device_labels) {
        const uint8_t *g8 = host ? gray_dev + LF * v : sc->views[v].gray;
        const int lst = dpe_edge_labels_device(ctx, g8, W, H, L - 1 - l, high_res_img, const_cast<int32_t *>(label[v][l]),
                                               w, h);
        if (lst != DPE_OK) return lst;
      }
    }
    // state from the previous level, rescaled (DPE::InuputInitialization, DPE.cpp:1019-1052)
    if (l > 0) {
      const int pw = lw[l - 1], ph = lh[l - 1];
      for (int v = 0; v < V; ++v) {
        k_rescale_nearest<float4><<<g2, b2, 0, s>>>(st[v].plane, pw, ph, planes_tmp, w, h);
        k_rescale_nearest<uint8_t><<<g2, b2, 0, s>>>(st[v].weak, pw, ph, weak_tmp, w, h);
        k_rescale_nearest<uint32_t><<<g2, b2, 0, s>>>(st[v].views, pw, ph, views_tmp, w, h);
        DPE_LAUNCHED("k_rescale_nearest", s);
        DPE_TRY(cudaMemcpyAsync(st[v].plane, planes_tmp, n * sizeof(float4), cudaMemcpyDeviceToDevice, s));
        DPE_TRY(cudaMemcpyAsync(st[v].weak, weak_tmp, n, cudaMemcpyDeviceToDevice, s));
        DPE_TRY(cudaMemcpyAsync(st[v].views, views_tmp, n * 4, cudaMemcpyDeviceToDevice, s));
        k_depth_from_plane<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(st[v].plane, st[v].depth, (int)n);
        DPE_LAUNCHED("k_depth_from_plane", s);
      }
    }
    for (int call = 0; call <= sch->refine_calls; ++call) {
      // The problem of view v in this call (main.cpp:390-457 parameters).
      auto make_problem = [&](int v, dpe_problem &p) {
        const dpe_scene_view &sv = sc->views[v];
        std::memset(&p, 0, sizeof(p));
        p.width = w; p.height = h; p.num_images = 1 + sv.num_src;
        p.memory = DPE_MEM_DEVICE;
        p.images[0] = st[v].img;
        p.cameras[0] = camera_at(sv.camera, W, H, w, h);
        for (int j = 0; j < sv.num_src; ++j) {
          const int id = sv.src_views[j];
          p.images[1 + j] = st[id].img;
          p.cameras[1 + j] = camera_at(sc->views[id].camera, W, H, w, h);
        }
        dpe_params &P = p.params;
        dpe_params_default(&P);
        P.num_images = p.num_images;
        P.max_scale_size = 1 << (L - 1);
        P.scale_size = lscale[l];
        P.max_iterations = sch->max_iterations;
        P.depth_min = sv.camera.depth_min * 0.6f;
        P.depth_max = sv.camera.depth_max * 1.2f;
        if (call == 0) {
          // main.cpp:398-419
          if (l == 0) {
            P.state = DPE_FIRST_INIT; P.use_APD = 0; P.use_edge = 0;
          } else {
            P.state = DPE_REFINE_INIT; P.use_APD = 1; P.use_edge = 1;
            P.ransac_threshold = (float)(0.01 - l * 0.00125);
            P.rotate_time = std::min(1 << l, 4);
          }
          P.geom_consistency = 0;
          P.weak_peak_radius = 6;
        } else {
          // main.cpp:428-445
          P.state = DPE_REFINE_ITER;
          P.use_APD = l > 0; P.use_edge = l > 0;
          P.ransac_threshold = (float)(0.01 - l * 0.00125);
          P.rotate_time = std::min(1 << l, 4);
          P.geom_consistency = 1;
          P.weak_peak_radius = std::max(4 - 2 * (call - 1), 2);
        }
        if (!have_edges) { P.use_edge = 0; P.use_limit = 0; }
        if (!have_labels) P.use_label = 0;
        if (P.state != DPE_FIRST_INIT) {
          p.plane_in = reinterpret_cast<const float *>(st[v].plane);
          p.selected_views_in = st[v].views;
        }
        p.weak_in = st[v].weak;
        if (have_edges) {
          p.edge = edge[v][l];
          p.edge_low_res = edge[v][0];
          p.low_width = lw[0];
          p.low_height = lh[0];
        }
        if (have_labels) p.label = label[v][l];
        if (P.geom_consistency) {
          p.depths[0] = st[v].depth;
          for (int j = 0; j < sv.num_src; ++j) p.depths[1 + j] = st[sv.src_views[j]].depth;
        }
        p.seed = mix64(sch->seed ^ ((uint64_t)l << 48) ^ ((uint64_t)call << 40) ^ (uint64_t)v);
      };
      auto store = [&](int v, const dpe_problem &p, float4 *op, uint8_t *ow, uint32_t *ov) -> int {
        k_store_result<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(op, ow, ov, (int)n, p.params.depth_min,
                                                                   p.params.depth_max, st[v].plane, st[v].depth,
                                                                   st[v].weak, st[v].views);
        DPE_LAUNCHED("k_store_result", s);
        return DPE_OK;
      };
      if (!sch->batch_views) {
        // the reference's order: view by view, each reading the depths its predecessors just wrote
        for (int v = 0; v < V; ++v) {
          dpe_problem p;
          make_problem(v, p);
          dpe_pm_out o;
          std::memset(&o, 0, sizeof(o));
          o.plane = reinterpret_cast<float *>(out_plane);
          o.weak = out_weak;
          o.selected_views = out_views;
          const int rc = dpe_pm_run(ctx, &p, &o);
          if (rc != DPE_OK) return rc;
          store(v, p, out_plane, out_weak, out_views);
          ++calls;
        }
      } else {
        // all views of the call in one batch, each reading the previous call's depths
        std::vector<dpe_problem> probs(V);
        std::vector<dpe_pm_out> outs(V);
        for (int v = 0; v < V; ++v) {
          make_problem(v, probs[v]);
          std::memset(&outs[v], 0, sizeof(dpe_pm_out));
          outs[v].plane = reinterpret_cast<float *>(bout_plane + LF * v);
          outs[v].weak = bout_weak + LF * v;
          outs[v].selected_views = bout_views + LF * v;
        }
        const int rc = dpe_pm_run_batch(ctx, probs.data(), V, outs.data());
        if (rc != DPE_OK) return rc;
        for (int v = 0; v < V; ++v) store(v, probs[v], bout_plane + LF * v, bout_weak + LF * v, bout_views + LF * v);
        calls += V;
      }
    }
  }
  DPE_TRY(cudaEventRecord(ef, s));

  // ---- outputs at the finest level
  const int wf = lw[L - 1], hf = lh[L - 1];
  const size_t nf = (size_t)wf * hf;
  float *fnormal = A.get<float>("sc_fnormal", nf * V * 3);
  if (!fnormal) return DPE_ERR_OUT_OF_MEMORY;
  for (int v = 0; v < V; ++v) {
    k_split_normal<<<(unsigned)((nf + 255) / 256), 256, 0, s>>>(st[v].plane, fnormal + nf * 3 * v, (int)nf);
    DPE_LAUNCHED("k_split_normal", s);
  }
  float fusion_ms = 0.f;
  if (sch->fuse_mode >= 0) {
    uint8_t *bgr_dev = host ? A.get<uint8_t>("sc_bgr", LF * 3 * V) : nullptr;
    if (host && !bgr_dev) return DPE_ERR_OUT_OF_MEMORY;
    std::vector<dpe_fusion_view> fv(V);
    for (int v = 0; v < V; ++v) {
      const dpe_scene_view &sv = sc->views[v];
      const uint8_t *bgr = sv.bgr;
      if (host) {
        DPE_TRY(cudaMemcpyAsync(bgr_dev + LF * 3 * v, sv.bgr, LF * 3, cudaMemcpyHostToDevice, s));
        bgr = bgr_dev + LF * 3 * v;
      }
      fv[v].width = wf; fv[v].height = hf;
      fv[v].depth = st[v].depth;
      fv[v].normal = fnormal + nf * 3 * v;
      fv[v].weak = st[v].weak;
      fv[v].bgr = bgr;
      fv[v].block_mask = nullptr;
      fv[v].camera = sv.camera;  // RescaleImageAndCamera is the identity at full resolution
      fv[v].num_src = sv.num_src;
      fv[v].src_views = sv.src_views;
    }
    dpe_fusion_in fin;
    fin.num_views = V; fin.views = fv.data(); fin.mode = sch->fuse_mode; fin.memory = DPE_MEM_DEVICE;
    fin.min_consistent = sch->min_consistent;
    const int rc = dpe_fuse(ctx, &fin, &out->fusion);
    if (rc != DPE_OK) return rc;
    fusion_ms = out->fusion.gpu_ms;
  }
  DPE_TRY(cudaEventRecord(e1, s));
  const cudaMemcpyKind d2o = out->out_memory == DPE_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  for (int v = 0; v < V; ++v) {
    if (out->depth && out->depth[v]) DPE_TRY(cudaMemcpyAsync(out->depth[v], st[v].depth, nf * 4, d2o, s));
    if (out->normal && out->normal[v]) DPE_TRY(cudaMemcpyAsync(out->normal[v], fnormal + nf * 3 * v, nf * 12, d2o, s));
    if (out->weak && out->weak[v]) DPE_TRY(cudaMemcpyAsync(out->weak[v], st[v].weak, nf, d2o, s));
    if (out->selected_views && out->selected_views[v])
      DPE_TRY(cudaMemcpyAsync(out->selected_views[v], st[v].views, nf * 4, d2o, s));
  }
  DPE_TRY(cudaStreamSynchronize(s));
  if (sch->device_edges) {
    const int est = dpe_edge_check(ctx);
    if (est != DPE_OK) return est;
  }
  if (sch->device_labels) {
    const int lst = dpe_edge_labels_check(ctx);
    if (lst != DPE_OK) return lst;
  }
  float ms = 0.f;
  DPE_TRY(cudaEventElapsedTime(&ms, e0, e1));
  out->gpu_ms = ms;
  out->fusion_ms = fusion_ms;
  out->num_levels = L;
  out->calls = calls;
  return DPE_OK;
}
