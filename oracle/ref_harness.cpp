// ref_harness.cpp -- TEST INFRASTRUCTURE: drives the reference's OWN per-view PatchMatch and
// fusion code, compiled for the CPU (oracle/_ref/libref.so, built by oracle/Makefile from
// DPE.cu and DPE.cpp where they lie, behind the host stand-ins of oracle/refshim/).
//
// ref_pm_call does what ProcessProblem does for one reference view (main.cpp:241-264): it lays the
// inputs out as the reference reads them (images/<id>.jpg, cams/<id>_cam.txt, the result folder's
// edges_<scale>.dmb / labels_<scale>.dmb, and a StateStore holding weak / depth / normal / views),
// then runs the reference's DPE constructor, InuputInitialization, SupportInitialization,
// CudaSpaceInitialization, SetDataPassHelperInCuda and RunPatchMatch, and returns the buffers
// RunPatchMatch copies back (DPE.cu:3258-3260) plus the final per-pixel costs.  Only the CUDA
// runtime, the texture unit, the random generator and OpenCV's file decoding are stand-ins.
//
// ref_fuse runs the reference's RunFusion (DPE.cpp:1387-1548) on views handed over through the
// same StateStore and reads back the PLY it writes.
//
// Both return the cameras and parameters the reference derived from its files, so the CPU
// oracle can be run on exactly the same numbers.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <string>
#include <vector>

#include "refshim/boost/filesystem.hpp"
#include "refshim/cuda_runtime.h"
#include "refshim/curand_kernel.h"
#include "refshim/opencv2/opencv.hpp"
#include "../include/dpe_b200.h"

// The harness reads the private device buffers of class DPE (costs, radius) after the reference
// has filled them.
#define private public
#include "DPE.h"
#undef private

extern "C" long long ref_guard_violations();
extern "C" void ref_set_launch_threads(int n);
void ref_set_serial_kernels(const std::vector<const void *> &kernels);

// the reference's red / black strong-update kernels (DPE.cu:1904-1942)
void BlackPixelUpdateStrong(const int iter, DataPassHelper *helper);
void RedPixelUpdateStrong(const int iter, DataPassHelper *helper);

namespace {

std::string g_error;

std::string id8(int id) {
  char b[16];
  std::snprintf(b, sizeof(b), "%08d", id);
  return b;
}

// cams/<id>_cam.txt in the format ReadCamera parses (DPE.cpp:341-382): "extrinsic", 3 rows of
// [R | t], the homogeneous row, "intrinsic", 3 rows of K, then depth_min interval depth_num
// depth_max.  %.9g round-trips every float.
bool write_camera(const std::string &path, const dpe_camera &c) {
  FILE *f = std::fopen(path.c_str(), "w");
  if (!f) return false;
  std::fprintf(f, "extrinsic\n");
  for (int i = 0; i < 3; ++i)
    std::fprintf(f, "%.9g %.9g %.9g %.9g\n", c.R[3 * i], c.R[3 * i + 1], c.R[3 * i + 2], c.t[i]);
  std::fprintf(f, "0 0 0 1\n\nintrinsic\n");
  for (int i = 0; i < 3; ++i) std::fprintf(f, "%.9g %.9g %.9g\n", c.K[3 * i], c.K[3 * i + 1], c.K[3 * i + 2]);
  std::fprintf(f, "\n%.9g %.9g %d %.9g\n", c.depth_min, (c.depth_max - c.depth_min) / 192.0f, 192, c.depth_max);
  std::fclose(f);
  return true;
}

bool write_pnm(const std::string &path, const unsigned char *data, int w, int h, int channels) {
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  std::fprintf(f, "%s\n%d %d\n255\n", channels == 3 ? "P6" : "P5", w, h);
  std::fwrite(data, 1, (size_t)w * h * channels, f);
  std::fclose(f);
  return true;
}

cv::Mat mat_from(const void *src, int rows, int cols, int type) {
  cv::Mat m(rows, cols, type);
  std::memcpy(m.data, src, (size_t)rows * m.step[0]);
  return m;
}

PatchMatchParams to_reference(const dpe_params &p) {
  PatchMatchParams r;
  r.max_iterations = p.max_iterations;
  r.num_images = p.num_images;
  r.sigma_spatial = p.sigma_spatial;
  r.sigma_color = p.sigma_color;
  r.top_k = p.top_k;
  r.depth_min = p.depth_min;
  r.depth_max = p.depth_max;
  r.geom_consistency = p.geom_consistency != 0;
  r.strong_radius = p.strong_radius;
  r.strong_increment = p.strong_increment;
  r.weak_radius = p.weak_radius;
  r.weak_increment = p.weak_increment;
  r.use_APD = p.use_APD != 0;
  r.use_edge = p.use_edge != 0;
  r.use_limit = p.use_limit != 0;
  r.use_label = p.use_label != 0;
  r.use_radius = p.use_radius != 0;
  r.high_res_img = p.high_res_img != 0;
  r.max_scale_size = p.max_scale_size;
  r.scale_size = p.scale_size;
  r.weak_peak_radius = p.weak_peak_radius;
  r.rotate_time = p.rotate_time;
  r.ransac_threshold = p.ransac_threshold;
  r.geom_factor = p.geom_factor;
  r.state = (RunState)p.state;
  return r;
}

dpe_params from_reference(const PatchMatchParams &r) {
  dpe_params p;
  p.max_iterations = r.max_iterations;
  p.num_images = r.num_images;
  p.sigma_spatial = r.sigma_spatial;
  p.sigma_color = r.sigma_color;
  p.top_k = r.top_k;
  p.depth_min = r.depth_min;
  p.depth_max = r.depth_max;
  p.geom_consistency = r.geom_consistency;
  p.strong_radius = r.strong_radius;
  p.strong_increment = r.strong_increment;
  p.weak_radius = r.weak_radius;
  p.weak_increment = r.weak_increment;
  p.use_APD = r.use_APD;
  p.use_edge = r.use_edge;
  p.use_limit = r.use_limit;
  p.use_label = r.use_label;
  p.use_radius = r.use_radius;
  p.high_res_img = r.high_res_img;
  p.max_scale_size = r.max_scale_size;
  p.scale_size = r.scale_size;
  p.weak_peak_radius = r.weak_peak_radius;
  p.rotate_time = r.rotate_time;
  p.ransac_threshold = r.ransac_threshold;
  p.geom_factor = r.geom_factor;
  p.state = r.state;
  return p;
}

void to_abi_camera(const Camera &c, dpe_camera *o) {
  static_assert(sizeof(Camera) == sizeof(dpe_camera), "dpe_camera mirrors Camera byte for byte");
  std::memcpy(o, &c, sizeof(Camera));
}

int log2_exact(int v) {
  int s = 0;
  while ((1 << s) < v) ++s;
  return (1 << s) == v ? s : -1;
}

}  // namespace

extern "C" {

const char *ref_last_error() { return g_error.c_str(); }

// One per-view call of the reference.  `pr` holds host memory only: images must carry integer
// grey levels 0..255 (they are handed to the reference as 8-bit files), cameras carry the
// cam-file depth range (the reference scales it by 0.6 / 1.2 itself), and pr->params.scale_size
// must be 1 (the images are given at the level's size).  With edges, pr->params.max_scale_size
// names the low-resolution map's level when high_res_img is set.  radius_init 1 starts radius
// at strong_radius (the oracle's deviation from the reference's uninitialised read); 0 leaves
// the freshly allocated (zero) buffer.  serial_race 1 runs the two edge-aware strong-update
// kernels one thread at a time (a deterministic result, the one a serial run gives); 0 runs
// every kernel's blocks in parallel, as for timing.  Outputs: plane (float4 per pixel), weak, views, costs,
// and the cameras / params the reference used.  Returns 0, or 1 with ref_last_error().
int ref_pm_call(const dpe_problem *pr, const char *work_dir, int threads, int radius_init, int serial_race,
                float *plane_out,
                uint8_t *weak_out, uint32_t *views_out, float *costs_out, dpe_camera *cams_out,
                dpe_params *params_out, long long *guard_writes) {
  try {
    namespace fs = std::filesystem;
    const int W = pr->width, H = pr->height, N = pr->num_images;
    if (pr->memory != DPE_MEM_HOST || N < 2 || N > MAX_IMAGES || pr->params.scale_size != 1) {
      g_error = "ref_pm_call: host memory, 2..32 images and scale_size 1 only";
      return 1;
    }
    const fs::path dense(work_dir);
    fs::create_directories(dense / "images");
    fs::create_directories(dense / "cams");
    const fs::path result = dense / "DPE" / id8(0);
    fs::create_directories(result);
    std::vector<unsigned char> gray((size_t)W * H);
    for (int i = 0; i < N; ++i) {
      for (size_t k = 0; k < gray.size(); ++k) {
        const float v = pr->images[i][k];
        if (!(v >= 0.0f && v <= 255.0f) || v != std::floor(v)) {
          g_error = "ref_pm_call: images must hold integer grey levels";
          return 1;
        }
        gray[k] = (unsigned char)v;
      }
      if (!write_pnm((dense / "images" / (id8(i) + ".jpg")).string(), gray.data(), W, H, 1) ||
          !write_camera((dense / "cams" / (id8(i) + "_cam.txt")).string(), pr->cameras[i])) {
        g_error = "ref_pm_call: cannot write the input files";
        return 1;
      }
    }
    const dpe_params &p = pr->params;
    if (p.use_edge || p.use_limit) {
      int max_scale = 0;
      if (p.high_res_img) max_scale = log2_exact(p.max_scale_size);
      const bool same = pr->low_width == W && pr->low_height == H;
      if (max_scale < 0 || (max_scale == 0) != same) {
        g_error = "ref_pm_call: max_scale_size must name the level of edge_low_res";
        return 1;
      }
      WriteBinMat(path((result / "edges_0.dmb").string()), mat_from(pr->edge, H, W, CV_8UC1));
      if (!same)
        WriteBinMat(path((result / ("edges_" + std::to_string(max_scale) + ".dmb")).string()),
                    mat_from(pr->edge_low_res, pr->low_height, pr->low_width, CV_8UC1));
    }
    if (p.use_label) WriteBinMat(path((result / "labels_0.dmb").string()), mat_from(pr->label, H, W, CV_32SC1));

    // the reference's per-view state (StateStore, DPE.h:113-123)
    StateStore store;
    {
      cv::Mat weak = pr->weak_in ? mat_from(pr->weak_in, H, W, CV_8UC1) : cv::Mat(H, W, CV_8UC1, cv::Scalar(STRONG));
      cv::Mat depth(H, W, CV_32FC1), normal(H, W, CV_32FC3);
      if (pr->plane_in) {
        for (int k = 0; k < W * H; ++k) {
          reinterpret_cast<float *>(depth.data)[k] = pr->plane_in[4 * k + 3];
          for (int c = 0; c < 3; ++c) reinterpret_cast<float *>(normal.data)[3 * k + c] = pr->plane_in[4 * k + c];
        }
      } else if (p.geom_consistency && pr->depths[0]) {
        depth = mat_from(pr->depths[0], H, W, CV_32FC1);
      }
      cv::Mat views = pr->selected_views_in ? mat_from(pr->selected_views_in, H, W, CV_32SC1)
                                            : cv::Mat::zeros(H, W, CV_32SC1);
      store.Put(0, depth, normal, weak, views);
      if (p.geom_consistency)
        for (int i = 1; i < N; ++i)
          store.Put(i, mat_from(pr->depths[i], H, W, CV_32FC1), cv::Mat(), cv::Mat(), cv::Mat());
    }

    Problem problem;
    problem.index = 0;
    problem.ref_image_id = 0;
    for (int i = 1; i < N; ++i) problem.src_image_ids.push_back(i);
    problem.dense_folder = path(dense.string());
    problem.result_folder = path(result.string());
    problem.scale_size = 1;
    problem.params = to_reference(p);
    problem.show_medium_result = false;
    problem.iteration = 0;

    ref_set_launch_threads(threads);
    // In the edge-aware branch a strong-update thread reads the cost and plane of an up-left
    // same-colour pixel that another thread of the launch may be writing (quirk Q1): those two
    // kernels run one thread at a time, so the result is the one of a serial run.
    if (serial_race)
      ref_set_serial_kernels({(const void *)&BlackPixelUpdateStrong, (const void *)&RedPixelUpdateStrong});
    else
      ref_set_serial_kernels({});
    ref_rng_configure(W, pr->seed);
    SceneCache cache(problem.dense_folder);
    DPE dpe(problem, &cache, &store, nullptr);
    dpe.InuputInitialization();
    dpe.SupportInitialization();
    dpe.CudaSpaceInitialization();
    dpe.SetDataPassHelperInCuda();
    if (radius_init && dpe.radius_cuda)
      for (int k = 0; k < W * H; ++k) dpe.radius_cuda[k] = dpe.params_host.strong_radius;
    dpe.RunPatchMatch();
    if (guard_writes) *guard_writes = ref_guard_violations();

    for (int r = 0; r < H; ++r)
      for (int c = 0; c < W; ++c) {
        const float4 pl = dpe.GetPlaneHypothesis(r, c);
        float *o = plane_out + 4 * ((size_t)r * W + c);
        o[0] = pl.x; o[1] = pl.y; o[2] = pl.z; o[3] = pl.w;
      }
    cv::Mat st = dpe.GetPixelStates(), sv = dpe.GetSelectedViews();
    std::memcpy(weak_out, st.data, (size_t)W * H);
    std::memcpy(views_out, sv.data, (size_t)W * H * 4);
    if (costs_out) std::memcpy(costs_out, dpe.costs_cuda, (size_t)W * H * 4);
    for (int i = 0; i < N; ++i) to_abi_camera(dpe.cameras[i], &cams_out[i]);
    *params_out = from_reference(dpe.params_host);
    return 0;
  } catch (const std::exception &e) {
    g_error = std::string("ref_pm_call: ") + e.what();
    return 1;
  }
}

// The reference's fusion over `in` (host memory; mode and min_consistent ignored: the reference
// computes in float with its own rules): variant 0 RunFusion (DPE.cpp:1387-1548, the ETH rule),
// 1 RunFusion_TAT_Intermediate (DPE.cpp:1550-1718), 2 RunFusion_TAT_advanced (DPE.cpp:1720-1867).
// Each view's colour image must already be at its depth map's size (RescaleImageAndCamera then
// clones it) and its camera is written to cams/ as given.  Block masks, when any view has one, go
// to blocks/mask_<id>.jpg for every view (all 255 where a view has none: nothing skipped).
// Writes up to `capacity` points (xyz, bgr in the PLY's blue, green, red order) and sets *count.
int ref_fuse(const dpe_fusion_in *in, int variant, const char *work_dir, float *xyz, uint8_t *bgr, int64_t capacity,
             int64_t *count) {
  try {
    namespace fs = std::filesystem;
    if (variant < 0 || variant > 2) {
      g_error = "ref_fuse: variant 0 (ETH), 1 (TAT intermediate) or 2 (TAT advanced)";
      return 1;
    }
    const fs::path dense(work_dir);
    fs::create_directories(dense / "images");
    fs::create_directories(dense / "cams");
    const fs::path out_dir = variant == 0 ? dense / "out" : dense / "DPE";
    fs::create_directories(out_dir);
    bool any_block = false;
    for (int i = 0; i < in->num_views; ++i) any_block = any_block || in->views[i].block_mask;
    if (any_block) fs::create_directories(dense / "blocks");
    StateStore store;
    std::vector<Problem> problems;
    for (int i = 0; i < in->num_views; ++i) {
      const dpe_fusion_view &v = in->views[i];
      const size_t npix = (size_t)v.width * v.height;
      // PPM stores RGB; imread returns BGR, so the file gets the channels reversed
      std::vector<unsigned char> rgb(npix * 3);
      for (size_t k = 0; k < npix; ++k) {
        rgb[3 * k] = v.bgr[3 * k + 2]; rgb[3 * k + 1] = v.bgr[3 * k + 1]; rgb[3 * k + 2] = v.bgr[3 * k];
      }
      if (!write_pnm((dense / "images" / (id8(i) + ".jpg")).string(), rgb.data(), v.width, v.height, 3) ||
          !write_camera((dense / "cams" / (id8(i) + "_cam.txt")).string(), v.camera)) {
        g_error = "ref_fuse: cannot write the input files";
        return 1;
      }
      if (any_block) {
        std::vector<unsigned char> full(npix, 255);
        if (!write_pnm((dense / "blocks" / ("mask_" + std::to_string(i) + ".jpg")).string(),
                       v.block_mask ? v.block_mask : full.data(), v.width, v.height, 1)) {
          g_error = "ref_fuse: cannot write a block mask";
          return 1;
        }
      }
      const fs::path result = dense / "DPE" / id8(i);
      fs::create_directories(result);
      cv::Mat depth = mat_from(v.depth, v.height, v.width, CV_32FC1);
      cv::Mat normal = mat_from(v.normal, v.height, v.width, CV_32FC3);
      if (variant == 0) {
        cv::Mat weak = v.weak ? mat_from(v.weak, v.height, v.width, CV_8UC1)
                              : cv::Mat(v.height, v.width, CV_8UC1, cv::Scalar(STRONG));
        store.Put(i, depth, normal, weak, cv::Mat());
      } else {  // the TAT rules read the result folders (DPE.cpp:1589-1594)
        WriteBinMat(path((result / "depths.dmb").string()), depth);
        WriteBinMat(path((result / "normals.dmb").string()), normal);
      }
      Problem pb;
      pb.index = i;
      pb.ref_image_id = i;
      for (int j = 0; j < v.num_src; ++j) pb.src_image_ids.push_back(v.src_views[j]);
      pb.dense_folder = path(dense.string());
      pb.result_folder = path(result.string());
      problems.push_back(pb);
    }
    if (variant == 0) RunFusion(path(dense.string()), path(out_dir.string()), problems, &store);
    else if (variant == 1) RunFusion_TAT_Intermediate(path(dense.string()), problems);
    else RunFusion_TAT_advanced(path(dense.string()), problems);
    // the binary PLY of ExportPointCloud (DPE.cpp:532-572): header, then x y z float + 3 uchar
    std::ifstream ply((out_dir / "DPE.ply").string(), std::ios::binary);
    std::string line;
    int64_t n = -1;
    while (std::getline(ply, line)) {
      if (line.rfind("element vertex ", 0) == 0) n = std::stoll(line.substr(15));
      if (line == "end_header") break;
    }
    if (n < 0) {
      g_error = "ref_fuse: no PLY header";
      return 1;
    }
    *count = n;
    for (int64_t k = 0; k < n && k < capacity; ++k) {
      ply.read(reinterpret_cast<char *>(xyz + 3 * k), 12);
      ply.read(reinterpret_cast<char *>(bgr + 3 * k), 3);
    }
    return 0;
  } catch (const std::exception &e) {
    g_error = std::string("ref_fuse: ") + e.what();
    return 1;
  }
}

// The reference's Connect (DPE.cpp:27-134) on a binary 8-bit image: labels (rows x cols) and the
// pixel count per final label (label_cnt); *num_labels = labels including 0.
int ref_connect(const uint8_t *img, int cols, int rows, int32_t *labels, int32_t *counts, int counts_capacity,
                int *num_labels) {
  cv::Mat src = mat_from(img, rows, cols, CV_8UC1);
  cv::Mat lab = cv::Mat::zeros(rows, cols, CV_32SC1);
  std::vector<int> cnt;
  Connect(src, lab, cnt);
  std::memcpy(labels, lab.data, (size_t)rows * cols * 4);
  for (int i = 0; i < (int)cnt.size() && i < counts_capacity; ++i) counts[i] = cnt[i];
  *num_labels = (int)cnt.size();
  return (int)cnt.size() > counts_capacity ? 1 : 0;
}

// The reference's Roberts cross (DPE.cpp:9-25) on an 8-bit image.
int ref_roberts(const uint8_t *img, int cols, int rows, uint8_t *out) {
  cv::Mat r = Roberts(mat_from(img, rows, cols, CV_8UC1));
  std::memcpy(out, r.data, (size_t)rows * cols);
  return 0;
}

}  // extern "C"
