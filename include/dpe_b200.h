/*
 * dpe_b200.h -- C ABI of the B200-native DPE-MVS PatchMatch + fusion path.
 *
 * The reference exposes this path as a C++ class and a free function:
 *   class DPE                    DPE.h:140-243 (setup: DPE.cpp:934-1252, kernels: DPE.cu:1-3262)
 *   RunFusion(...)               DPE.h:95-96, DPE.cpp:1387-1548
 * and its only caller is ProcessProblem / main (main.cpp:241-466).  Each entry point below
 * names the reference interface it replaces.  All structs are plain C (no C++ or torch types),
 * every call returns an int status (DPE_OK == 0) and never exits the process.
 *
 * Threading: one dpe_ctx per host thread.  Calls are stream-ordered on the context's stream and
 * return after the work has completed.
 */
#ifndef DPE_B200_H_
#define DPE_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DPE_MAX_IMAGES 32     /* main.h:42  MAX_IMAGES      */
#define DPE_NEIGHBOUR_NUM 9   /* main.h:43  NEIGHBOUR_NUM   */

/* ---- status codes (replace CudaSafeCall's exit(EXIT_FAILURE), DPE.cpp:646-679) ---- */
enum {
  DPE_OK = 0,
  DPE_ERR_INVALID_ARGUMENT = 1,  /* null pointer, bad size, >32 images, bad enum ... */
  DPE_ERR_CUDA = 2,              /* a CUDA runtime call failed                       */
  DPE_ERR_OUT_OF_MEMORY = 3,     /* device allocation failed                         */
  DPE_ERR_CAPACITY = 4,          /* caller-provided output buffer too small          */
  DPE_ERR_NO_DEVICE = 5,         /* no CUDA device / wrong device index              */
  DPE_ERR_DEVICE_TIMEOUT = 6     /* a bounded device-side wait gave up               */
};

/* pixel states, main.h:70-74 */
enum { DPE_WEAK = 0, DPE_STRONG = 1, DPE_UNKNOWN = 2 };
/* run states, main.h:64-68 */
enum { DPE_FIRST_INIT = 0, DPE_REFINE_INIT = 1, DPE_REFINE_ITER = 2 };
/* where the pointers of a problem live */
enum { DPE_MEM_HOST = 0, DPE_MEM_DEVICE = 1 };
/* fusion arithmetic for the consistency test */
enum { DPE_FUSE_FP64 = 0, DPE_FUSE_FLOAT = 1 };

/* Camera, byte-identical to the reference struct (main.h:53-62): K, R row-major 3x3, t, centre c
 * (computed in double by ReadCamera, DPE.cpp:366-369), image size, depth range from the cam file. */
typedef struct dpe_camera {
  float K[9];
  float R[9];
  float t[3];
  float c[3];
  int height;
  int width;
  float depth_min;
  float depth_max;
} dpe_camera;

/* PatchMatchParams (main.h:81-109) with the bools widened to int. */
typedef struct dpe_params {
  int max_iterations;
  int num_images;
  float sigma_spatial;
  float sigma_color;
  int top_k;
  float depth_min;
  float depth_max;
  int geom_consistency;
  int strong_radius;
  int strong_increment;
  int weak_radius;
  int weak_increment;
  int use_APD;
  int use_edge;
  int use_limit;
  int use_label;
  int use_radius;
  int high_res_img;
  int max_scale_size;
  int scale_size;
  int weak_peak_radius;
  int rotate_time;
  float ransac_threshold;
  float geom_factor;
  int state; /* DPE_FIRST_INIT / DPE_REFINE_INIT / DPE_REFINE_ITER */
} dpe_params;

/* One per-view PatchMatch call: the inputs DPE::InuputInitialization / SupportInitialization /
 * CudaSpaceInitialization gather (DPE.cpp:934-1214).  All pointers are host or device memory
 * according to `memory`.  Image 0 is the reference view, 1..num_images-1 the sources. */
typedef struct dpe_problem {
  int width;
  int height;
  int num_images;                       /* 2..32 */
  const float *images[DPE_MAX_IMAGES];  /* gray float W*H row-major (SceneCache::GetGrayFloatImage) */
  dpe_camera cameras[DPE_MAX_IMAGES];   /* K scaled to W,H (SceneCache::GetCamera, DPE.cpp:739-760) */
  dpe_params params;                    /* depth_min/max already x0.6 / x1.2 (DPE.cpp:953-954) */
  const float *plane_in;                /* float4 per pixel (world normal xyz, depth); REFINE_* only */
  const uint32_t *selected_views_in;    /* per pixel view bitmask; NULL = zeros                  */
  const uint8_t *weak_in;               /* per pixel state; read when use_APD, else all STRONG  */
  const uint8_t *edge;                  /* W*H edge map (edges_<scale>.dmb); when use_edge||use_limit */
  const uint8_t *edge_low_res;          /* low_width*low_height (edges_<max_scale>.dmb)          */
  int low_width;
  int low_height;
  const int32_t *label;                 /* W*H labels (labels_<scale>.dmb); when use_label      */
  const float *depths[DPE_MAX_IMAGES];  /* W*H depth maps of every image; when geom_consistency */
  uint64_t seed;                        /* Philox key of this call's random streams             */
  int memory;                           /* DPE_MEM_HOST or DPE_MEM_DEVICE                        */
} dpe_problem;

/* Outputs of one call (the three D2H copies of DPE.cu:3258-3260, plus optional costs).
 * Caller-allocated, in the memory space named by dpe_problem.memory. */
typedef struct dpe_pm_out {
  float *plane;              /* float4 per pixel: world normal xyz, depth (after GetDepthandNormal) */
  uint8_t *weak;             /* per pixel state after DepthToWeak                                   */
  uint32_t *selected_views;  /* per pixel view bitmask                                              */
  float *costs;              /* optional (may be NULL): final per-pixel cost                         */
  float gpu_ms;              /* device time of the kernel sequence (DPE::GetLastGpuTimeMs)           */
  uint64_t strong_ncc_evals; /* number of strong-window NCC evaluations (filled when counting on)   */
  uint64_t weak_ncc_evals;   /* number of deformable (weak) NCC evaluations                          */
} dpe_pm_out;

/* ---- fusion (RunFusion, DPE.cpp:1387-1548) ---- */
typedef struct dpe_fusion_view {
  int width;
  int height;
  const float *depth;          /* W*H, <= 0 means no depth                             */
  const float *normal;         /* W*H*3 world normals                                  */
  const uint8_t *weak;         /* W*H pixel states                                     */
  const uint8_t *bgr;          /* W*H*3 colour at depth resolution                     */
  const uint8_t *block_mask;   /* optional W*H; pixels < 128 are skipped (blocks/)    */
  dpe_camera camera;           /* camera at depth resolution                           */
  int num_src;
  const int *src_views;        /* host array of view indices (into the views array)   */
} dpe_fusion_view;

typedef struct dpe_fusion_in {
  int num_views;
  const dpe_fusion_view *views;  /* host array, in pair.txt order */
  int mode;                      /* DPE_FUSE_FP64 or DPE_FUSE_FLOAT */
  int memory;                    /* where depth/normal/weak/bgr/block_mask live */
  int min_consistent;            /* consistent sources a point needs; <= 1 is the reference rule
                                    num_consistent >= 1 (DPE.cpp:1520) */
} dpe_fusion_in;

typedef struct dpe_fusion_out {
  int64_t capacity;      /* points the buffers below can hold                       */
  int64_t count;         /* points produced (set even when capacity is too small)   */
  float *xyz;            /* capacity*3, host memory                                  */
  uint8_t *bgr;          /* capacity*3, host memory (PLY diffuse_blue/green/red)     */
  int32_t *origin;       /* optional capacity*2: (view index, pixel index) per point */
  uint8_t *num_consistent; /* optional capacity: consistent sources per point        */
  float gpu_ms;
} dpe_fusion_out;

/* ---- NCC evaluation at explicit (pixel, plane, source) queries ----
 * The memory space of every pointer below is set by the entry point that takes the query:
 * host memory for dpe_ncc_eval and dpe_ncc_grad, device memory for dpe_ncc_grad_device and
 * dpe_ncc_eval_noalloc. */
typedef struct dpe_ncc_query {
  int width;
  int height;
  int num_images;
  const float *images[DPE_MAX_IMAGES];  /* W*H float images; memory space: see above */
  dpe_camera cameras[DPE_MAX_IMAGES];
  dpe_params params;                    /* strong_radius/increment, sigmas */
  int64_t count;
  const int32_t *px;      /* count pixel x */
  const int32_t *py;      /* count pixel y */
  const int32_t *src;     /* count source index 1..num_images-1 */
  const float *plane;     /* count*4 plane in reference-camera coordinates (n, distance) */
} dpe_ncc_query;

/* ---- whole-scene schedule (the pyramid / call loop of main.cpp:321-466, without file I/O) ---- */
typedef struct dpe_scene_view {
  const uint8_t *gray;            /* W*H gray image at full resolution (imread GRAYSCALE)           */
  const uint8_t *bgr;             /* W*H*3 colour image for fusion; NULL when not fusing            */
  dpe_camera camera;              /* as read from cams/ (full resolution)                          */
  int num_src;
  const int *src_views;           /* host array: view indices (pair.txt sources with score > 0)    */
  const uint8_t *const *edges;    /* host array, one map per level (level 0 = coarsest), or NULL   */
  const int32_t *const *labels;   /* host array, one map per level, or NULL                         */
} dpe_scene_view;

typedef struct dpe_schedule {
  int num_levels;       /* 0: the reference rule, halve max(W,H) until <= 800 (main.cpp:223-238) */
  int refine_calls;     /* geom-consistency REFINE_ITER calls per level (main.cpp:422: 3)        */
  int max_iterations;   /* red/black iterations per call (main.cpp:418, 444: 3)                  */
  int fuse_mode;        /* DPE_FUSE_FP64 / DPE_FUSE_FLOAT, or -1 for no fusion                   */
  int min_consistent;   /* fusion: consistent sources per point (<= 1: the reference rule)        */
  uint64_t seed;        /* base of the per-call random streams                                    */
  int batch_views;      /* 0: views one after another within a call, each reading the depths its
                           predecessors wrote (the reference's order); 1: all views of a call in one
                           dpe_pm_run_batch, each reading the previous call's depths            */
  int device_edges;     /* 1: each level's edge map is made on the device from the level image
                           (GetProblemEdges' EdgeSegment mode 0, main.cpp:170-197; dpe_edge_map);
                           views[].edges must then be NULL                                       */
  int device_labels;    /* 1: each level's label map is made on the device from the full-resolution
                           image (GetProblemEdges' EdgeSegment mode 1, main.cpp:199-214;
                           dpe_edge_labels); views[].labels must then be NULL                      */
} dpe_schedule;

typedef struct dpe_scene {
  int num_views;
  int width;                      /* full resolution, equal for every view (CheckImages)          */
  int height;
  const dpe_scene_view *views;    /* host array, pair.txt order                                    */
  int memory;                     /* where gray / bgr / edges / labels live                        */
} dpe_scene;

/* per kernel class statistics (dpe_ctx_get_kernel_stats) */
typedef struct dpe_kernel_stat {
  char name[32];
  int64_t launches;           /* launches timed while profiling was on            */
  double ms;                  /* summed device time of those launches              */
  uint64_t strong_ncc_evals;  /* strong-window NCC evaluations while counting      */
  uint64_t weak_ncc_evals;    /* deformable-window NCC evaluations while counting  */
} dpe_kernel_stat;

typedef struct dpe_scene_out {
  float **depth;                  /* optional host array of num_views pointers: final W*H depth    */
  float **normal;                 /* optional: W*H*3 world normals                                 */
  uint8_t **weak;                 /* optional: W*H pixel states                                    */
  uint32_t **selected_views;      /* optional: W*H view masks                                      */
  int out_memory;                 /* memory space the pointers above refer to                      */
  dpe_fusion_out fusion;          /* fused points (host memory), when fuse_mode >= 0               */
  float gpu_ms;                   /* device time of the whole schedule including fusion            */
  float fusion_ms;
  int num_levels;
  int calls;                      /* per-view PatchMatch calls run                                 */
} dpe_scene_out;

/* ---- context ---- */
typedef struct dpe_ctx dpe_ctx;

typedef struct dpe_limits {
  int max_width;      /* 0 = no preallocation */
  int max_height;
  int max_images;
} dpe_limits;

/* Human-readable text of a status code. */
const char *dpe_status_string(int status);

/* Text of the last CUDA failure on the calling host thread (failing call or kernel, CUDA error
 * name and message); empty when there was none.  Replaces CudaSafeCall's stderr message
 * (DPE.cpp:646-679).  Setting DPE_DEBUG_SYNC=1 in the environment synchronises after every
 * kernel so that an execution error names its kernel (the reference's DPE_DEBUG_SYNC build
 * option, DPE.cu:3-7). */
const char *dpe_last_error(void);

/* PatchMatchParams default member initialisers (main.h:81-109). */
void dpe_params_default(dpe_params *params);

/* Replaces the process-wide GpuWorkspace (DPE.cpp:775-837) and cudaSetDevice (main.cpp:343):
 * a context owns the device arena, a stream and events on `device`. */
int dpe_ctx_create(int device, const dpe_limits *limits, dpe_ctx **out);
int dpe_ctx_destroy(dpe_ctx *ctx);

/* Replaces DPE::CudaSpaceInitialization + SetDataPassHelperInCuda + RunPatchMatch and the
 * getters GetPlaneHypothesis / GetPixelStates / GetSelectedViews / GetLastGpuTimeMs
 * (DPE.cpp:1071-1288, DPE.cu:3130-3262) for one reference view. */
int dpe_pm_run(dpe_ctx *ctx, const dpe_problem *problem, dpe_pm_out *out);

/* Batched form of dpe_pm_run (no reference counterpart; the reference runs one view per call):
 * `count` independent per-view problems, each with its own size, images, cameras, inputs and
 * seed, run through ONE kernel sequence -- every kernel is launched once for the whole batch, its
 * grid the problems' grids laid end to end, so small views fill the GPU together.  The problems
 * must agree on the schedule flags (params.state, use_APD, use_edge, geom_consistency,
 * max_iterations); other parameters may differ.  Each problem's result equals its dpe_pm_run
 * result.  outs[b].gpu_ms and the evaluation counts are the batch's totals.  count <=
 * DPE_MAX_BATCH.
 * It takes no dpe_schedule: it is one call of the schedule for many views, and each problem
 * already carries that call's parameters.  The schedule across calls and pyramid levels (levels,
 * refine calls, iterations, fusion) is dpe_scene_run's dpe_schedule, whose batch_views = 1 runs
 * every call through this entry point. */
#define DPE_MAX_BATCH 256
int dpe_pm_run_batch(dpe_ctx *ctx, const dpe_problem *problems, int count, dpe_pm_out *outs);

/* Replaces the compute of RunFusion (DPE.cpp:1387-1548): returns the fused points in the
 * reference order (view order, then raster order).  Writing the PLY stays with the caller
 * (ExportPointCloud, DPE.cpp:532-572). */
int dpe_fuse(dpe_ctx *ctx, const dpe_fusion_in *in, dpe_fusion_out *out);

/* The two Tanks-and-Temples fusion rules, which the reference declares beside RunFusion
 * (DPE.h:97-98) for its TAT runs:
 *   DPE_TAT_INTERMEDIATE  RunFusion_TAT_Intermediate (DPE.cpp:1550-1718): a pixel is kept at the
 *                         first k in 2..num_src for which at least k sources have reprojection
 *                         error < 0.25 k, relative depth difference < k / 3500 and normal angle
 *                         < 3k + 4 degrees; its colour is the mean of the reference pixel and
 *                         those sources' pixels.
 *   DPE_TAT_ADVANCED      RunFusion_TAT_advanced (DPE.cpp:1720-1867): the same without the angle
 *                         bound, relative depth < k / 3000, colour of the reference pixel only.
 * As in the reference, a source's differences persist from pixel to pixel within a view: a
 * source that is out of the image, masked or without depth at a pixel counts with the values of
 * the last pixel of the view where it was tested (the difference vector is set once per view,
 * DPE.cpp:1640 / 1804).  A kept pixel masks itself; only the masks of sources are read.
 * `weak` may be NULL and `min_consistent` is not used; `num_consistent` receives the number of
 * sources counted at the accepting k.  Views, points and errors otherwise as dpe_fuse. */
enum { DPE_TAT_INTERMEDIATE = 0, DPE_TAT_ADVANCED = 1 };
int dpe_fuse_tat(dpe_ctx *ctx, const dpe_fusion_in *in, int variant, dpe_fusion_out *out);

/* The edge map of EdgeSegment (DPE.cpp:136-250) as GetProblemEdges requests it for a pyramid level
 * (EdgeSegment(scale, image, 0, true, high_res_img), main.cpp:182-197): cv::Canny with aperture 3,
 * the L2 gradient and thresholds (1 - 0.67) * median and median of the image's histogram, then the
 * border rule of DPE.cpp:239-250.  `image` is the level image converted to 8 bits (width*height,
 * row-major), `edge_out` receives width*height values 0 / 255; both in `memory`.  The reference
 * writes the result to edges_<scale>.dmb; dpe_scene_run can make these maps itself
 * (dpe_schedule.device_edges). */
int dpe_edge_map(dpe_ctx *ctx, const uint8_t *image, int width, int height, int memory, uint8_t *edge_out);

/* The label map of EdgeSegment (DPE.cpp:136-291) as GetProblemEdges requests it for a pyramid level
 * (EdgeSegment(scale, image_uint, 1, false, high_res_img), main.cpp:199-214): from the
 * full-resolution 8-bit image `gray` (width*height), halved when high_res_img and halved again, a
 * Roberts gradient thresholded at 4 (6 without high_res_img), the reference's region labelling
 * Connect, Hough segments drawn across the outer border of every weak region of at least
 * width*height / (1024 << 2*scale) pixels, the map resized to the level, thresholded,
 * border-ruled and labelled again.  `labels_out` receives round(width / 2^scale) *
 * round(height / 2^scale) int32 labels: 0 on edges, -1 on regions of at most that many pixels,
 * otherwise the region number.  The resize, Hough transform and line drawing are OpenCV's
 * (cv::resize INTER_LINEAR, cv::HoughLinesP, cv::line) in their integer forms, bit for bit.  The
 * reference writes the result to labels_<scale>.dmb; dpe_scene_run can make these maps itself
 * (dpe_schedule.device_labels). */
int dpe_edge_labels(dpe_ctx *ctx, const uint8_t *gray, int width, int height, int scale, int high_res_img, int memory,
                    int32_t *labels_out);

/* Replaces main()'s PatchMatch schedule and fusion (main.cpp:385-461) for a whole scene, with every
 * view's state kept in device memory between calls: per level the float image pyramid
 * (SceneCache::GetGrayFloatImage, DPE.cpp:720-737), one FIRST_INIT / REFINE_INIT call and
 * `refine_calls` geom REFINE_ITER calls per view in pair.txt order (Gauss-Seidel across views),
 * ProcessProblem's result assembly (main.cpp:266-279), nearest-neighbour state rescale between
 * levels (RescaleMatToTargetSize, DPE.cpp:1313-1335), then RunFusion.  Edge and label maps are
 * host preprocessing (EdgeSegment) and are passed in. */
int dpe_scene_run(dpe_ctx *ctx, const dpe_scene *scene, const dpe_schedule *schedule, dpe_scene_out *out);

/* Strong bilateral NCC (ComputeBilateralNCCOld, DPE.cu:696-782) at explicit queries; test and
 * measurement entry point.  Every pointer of `q` and `costs_out` is HOST memory; the call copies
 * the inputs to the context's device and returns after the costs are back on the host. */
int dpe_ncc_eval(dpe_ctx *ctx, const dpe_ncc_query *q, float *costs_out);

/* Adjoint of dpe_ncc_eval: the strong NCC and its gradient at explicit queries.  Every pointer
 * of `q` and every output buffer is HOST memory, as for dpe_ncc_eval.
 * The reference has no gradient; this is the differentiable form of ComputeBilateralNCCOld
 * (DPE.cu:696-782) for plane refinement and autograd harnesses.
 *   grad_plane_out        [count][4] dC/d(nx, ny, nz, w) of the query's plane (n, w) in
 *                         reference-camera coordinates (the layout of dpe_ncc_query::plane);
 *   grad_depth_normal_out [count][4] dC/d(depth, nx, ny, nz) with the pixel's depth held fixed
 *                         instead of w (w = -depth * n . Kr^-1 (x, y, 1)); may be NULL;
 *   grad_images_out       NULL, or num_images pointers (entry 0 unused, NULL entries skipped) to
 *                         width x height float buffers receiving d(sum of all query costs) /
 *                         d(source image pixel).
 * The gradient is zero where the cost is the constant 2 (centre outside the source, flat window)
 * or clamped to [0, 2]. */
int dpe_ncc_grad(dpe_ctx *ctx, const dpe_ncc_query *q, float *costs_out, float *grad_plane_out,
                 float *grad_depth_normal_out, float *const *grad_images_out);

/* dpe_ncc_grad on device memory, for autograd callers whose tensors stay on the GPU (no
 * reference counterpart).  Every pointer of `q`, `upstream` and the outputs is DEVICE memory of the
 * context's device; the work runs on `stream` (a cudaStream_t; NULL: the default stream) and the
 * call returns when it has completed.
 *   upstream              NULL, or count weights: each query's contribution to grad_images_out is
 *                         scaled by its weight (the gradient of sum_k upstream[k] * C_k), so a
 *                         backward pass gives the image gradient in one call;
 *   grad_plane_out        NULL, or [count][4] dC/d(nx, ny, nz, w) (unweighted, as dpe_ncc_grad);
 *   grad_depth_normal_out NULL, or [count][4] dC/d(depth, nx, ny, nz);
 *   grad_images_out       NULL, or (num_images - 1) consecutive width x height float planes, one per
 *                         source image (image 1 first); zeroed by the call before accumulating.
 * Queries whose pixel or source index lies outside the problem get NaN outputs. */
int dpe_ncc_grad_device(dpe_ctx *ctx, const dpe_ncc_query *q, const float *upstream, float *costs_out,
                        float *grad_plane_out, float *grad_depth_normal_out, float *grad_images_out, void *stream);

/* Allocation-free variant of dpe_ncc_eval for callers that cannot allocate device memory: code
 * hosted by a framework that owns and budgets all device memory through its own allocator (a
 * private cudaMalloc there would bypass its accounting), and real-time paths that must not pay
 * for cudaMalloc / cudaFree, which may synchronise the device.  It has no counterpart in the
 * reference.
 *
 * Every pointer in `q` (images, px, py, src, plane) and `costs_out` is DEVICE memory owned by the
 * caller; `plane` is 16-byte aligned.  The call needs no dpe_ctx: it enqueues its work on `stream`
 * (a cudaStream_t; NULL is the default stream) of the calling thread's current device and returns
 * before the work completes -- synchronise the stream before reading `costs_out`.  Queries whose
 * pixel or source index lies outside the problem get NaN.
 *
 * Scratch (the argument block and the clamp-padded images) lives in one statically allocated
 * 16 MiB array in device memory, which every GPU that loads this library holds until the process
 * exits.  A problem is accepted when 256-byte-rounded sizeof(argument block) plus num_images x
 * 256-byte-rounded (width + 2) x (height + 2) x 4 bytes fits in 16 MiB (e.g. up to 12 images of
 * 640x480); larger ones return DPE_ERR_CAPACITY with the sizes in dpe_last_error().  The first
 * call on a device resolves the array's device address (cudaGetSymbolAddress) with that device
 * current; make that first call before any stream capture.  All calls share the one array and
 * it keeps the previous call's contents, so calls that overlap on the GPU (different streams or
 * host threads without ordering between them) race and corrupt each other's results. */
int dpe_ncc_eval_noalloc(const dpe_ncc_query *q, float *costs_out, void *stream);

/* ---- view selection: the pair scores behind pair.txt ----
 * The reference's view selection (colmap2mvsnet.py:280-302 calc_score, 405-419 in
 * processing_single_scene) scores every image pair (i, j), i < j, by the 2D observations of
 * image i whose 3D point image j also observes (an observation listed twice counts twice), and
 * sets the score to 0 when the 75th percentile (element int(0.75 n) of the sorted list) of those
 * observations' triangulation angles is below 1 degree.  Points are given densely indexed (the
 * caller maps COLMAP's point ids to 0..num_points-1; -1 is an observation without a point). */
typedef struct dpe_sparse_model {
  int num_images;
  const double *centers;        /* num_images*3 camera centres -R^T t (host memory)         */
  const int64_t *obs_offsets;   /* num_images+1: image i's observations are
                                   obs_point[obs_offsets[i] .. obs_offsets[i+1])             */
  const int32_t *obs_point;     /* dense point index per observation, or -1                  */
  int64_t num_points;
  const double *points;         /* num_points*3 xyz                                          */
} dpe_sparse_model;
/* scores_out: num_images x num_images doubles (host memory), symmetric, 0 on the diagonal: the
 * matrix `score` that processing_single_scene ranks for each view's sources. */
int dpe_view_scores(dpe_ctx *ctx, const dpe_sparse_model *m, double *scores_out);

/* ---- options: the precision and differentiation forms of the path (no reference counterpart) */
enum { DPE_STAGE_FP32 = 0, DPE_STAGE_FP16 = 1, DPE_STAGE_BF16 = 2 };
typedef struct dpe_options {
  /* Storage of the source images the cost kernels sample (DPE_STAGE_*).  FP16 / BF16 keep each
   * padded texel and its right neighbour in one 32-bit word; the bilinear interpolation, the
   * moments and the NCC stay FP32, as do the reference image and the window weights.  Images of
   * 8-bit integers are exact in both (the finest pyramid level); interpolated pyramid levels are
   * rounded.  Default DPE_STAGE_FP32: sources sampled as FP32 values, from BF16 pairs when every
   * source texel of the call is exact in BF16 (checked on the device), which gives the same
   * results with half the gather bytes. */
  int staging;
  /* 1: every strong-update iteration adds one Gauss-Newton plane hypothesis, built from the
   * adjoint of the strong NCC (dpe_ncc_grad) over the pixel's sampled sources, and keeps it when
   * it lowers the pixel's cost like the reference's random hypotheses.  Default 0: the
   * reference's refinement only. */
  int gn_refine;
} dpe_options;
/* Applies to the following dpe_pm_run / dpe_scene_run calls of the context. */
int dpe_ctx_set_options(dpe_ctx *ctx, const dpe_options *opt);

/* Statistics switch: when on, dpe_pm_run counts its NCC evaluations into
 * dpe_pm_out.strong_ncc_evals / weak_ncc_evals (device atomics; off by default).  The reference
 * has no counterpart (it prints stage times only, main.cpp:17-45). */
int dpe_ctx_set_eval_counting(dpe_ctx *ctx, int on);

/* Per-kernel device timing (an event pair around every launch while on; off by default), the
 * statistics accumulated since the last reset, and a reset.  No reference counterpart (the
 * reference times the whole launch sequence with one event pair, DPE.cu:3132-3239). */
int dpe_ctx_set_profiling(dpe_ctx *ctx, int on);
int dpe_ctx_reset_kernel_stats(dpe_ctx *ctx);
int dpe_ctx_get_kernel_stats(dpe_ctx *ctx, dpe_kernel_stat *out, int capacity, int *count);

/* Launch tuner (no reference counterpart; the reference launches fixed 16x16 blocks).  For each
 * (kernel, size class = floor(log2 of the call's pixels)) the context's first launches cycle
 * through candidate settings that change no result -- the block shape of the random
 * initialisation (16x8, 32x4, 8x16, 64x2, 8x8; single-problem calls only) and the shared-memory
 * carveout of the strong update (driver default, 100, 75, 50 %), the two kernels whose launches
 * of one size class do the same work -- each timed by an event pair on the context's stream, and
 * keep the fastest mean after 2 samples each.  On by default; dpe_ctx_set_autotune(ctx, 0) uses
 * the first candidate throughout. */
int dpe_ctx_set_autotune(dpe_ctx *ctx, int on);
typedef struct dpe_tuning_entry {
  char name[32];      /* kernel class, as in dpe_kernel_stat                                   */
  int size_class;     /* floor(log2(pixels of the call or batch))                              */
  int candidates;     /* settings tried                                                        */
  int chosen;         /* index of the kept setting; -1 while still measuring                   */
  int block_x;        /* block shape of the kept setting (shape-tuned kernels; else 0)         */
  int block_y;
  int carveout;       /* carveout of the kept setting in percent, -1 the driver default
                         (carveout-tuned kernels; else 0)                                      */
  float mean_ms[8];   /* mean measured time per candidate (0: no sample)                       */
} dpe_tuning_entry;
int dpe_ctx_get_tuning(dpe_ctx *ctx, dpe_tuning_entry *out, int capacity, int *count);

/* Number of kernels this library has launched in the process (all contexts). */
uint64_t dpe_launch_count(void);

/* Measured FP32 FMA throughput of the context's device in TFLOP/s (a dependent-chain FMA kernel
 * over every SM): the roofline denominator of the NCC cost kernels, which are FP32-issue bound. */
int dpe_fp32_peak(dpe_ctx *ctx, double *tflops);

#ifdef __cplusplus
}
#endif
#endif /* DPE_B200_H_ */
