// views.cu -- view selection for pair.txt on the GPU: the score of every image pair
// (calc_score, colmap2mvsnet.py:280-302) that processing_single_scene ranks to choose each
// view's sources (colmap2mvsnet.py:405-419).
//
// The reference scores a pair (i, j), i < j, by walking image i's 2D observations and keeping
// those whose 3D point image j also observes (an observation listed twice counts twice); the
// score is their number, or 0 when the 75th percentile of their triangulation angles is below 1
// degree.  It runs one Python job per pair over all pairs.  Here the observations become
// (point, image) keys, sorted once; the runs of one point are its track, and every pair of images
// in a track adds image i's multiplicity to the pair's count and that many copies of the angle to
// the pair's angle list.  One segmented sort of the angle lists gives each percentile.
//
// Compiled with -fmad=false: the angles are double expressions written in the reference's order.
#include <cub/cub.cuh>

#include <cmath>
#include <cstring>

#include "ctx.h"

namespace {

constexpr unsigned long long kNoPoint = ~0ull;

// One key per observation: point * N + image, or kNoPoint for an observation without a 3D point.
__global__ void k_obs_keys(const long long *offsets, const int32_t *obs_point, int N, unsigned long long *keys) {
  const int img = blockIdx.x;
  const long long a = offsets[img], b = offsets[img + 1];
  for (long long k = a + threadIdx.x; k < b; k += blockDim.x) {
    const int p = obs_point[k];
    keys[k] = p < 0 ? kNoPoint : (unsigned long long)p * (unsigned long long)N + (unsigned long long)img;
  }
}

// calc_score's angle for point p between cameras a and b (colmap2mvsnet.py:291-292), in degrees.
__device__ __forceinline__ double tri_angle(const double *ca, const double *cb, const double *p) {
  const double d0 = ca[0] - p[0], d1 = ca[1] - p[1], d2 = ca[2] - p[2];
  const double e0 = cb[0] - p[0], e1 = cb[1] - p[1], e2 = cb[2] - p[2];
  const double dot = d0 * e0 + d1 * e1 + d2 * e2;
  const double na = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
  const double nb = sqrt(e0 * e0 + e1 * e1 + e2 * e2);
  return (180.0 / 3.14159265358979323846) * acos(dot / na / nb);
}

// Run r of the sorted keys is (point, image a, multiplicity); the later runs of the same point are
// the track's images b > a.  Pass 0 counts, pass 1 writes the angles at the pairs' cursors.
template <int kPass>
__global__ void k_track_pairs(const unsigned long long *run_key, const int *run_len, const int *num_runs, int N,
                              const double *centers, const double *points, unsigned long long *count,
                              unsigned long long *cursor, double *angles) {
  const int R = *num_runs;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
    const unsigned long long k = run_key[r];
    if (k == kNoPoint) continue;
    const unsigned long long p = k / (unsigned long long)N;
    const int a = (int)(k - p * (unsigned long long)N);
    const unsigned long long m = (unsigned long long)run_len[r];
    for (int r2 = r + 1; r2 < R; ++r2) {
      const unsigned long long k2 = run_key[r2];
      if (k2 == kNoPoint || k2 / (unsigned long long)N != p) break;
      const int b = (int)(k2 - p * (unsigned long long)N);
      const size_t pair = (size_t)a * N + b;
      if (kPass == 0) {
        atomicAdd(&count[pair], m);
      } else {
        const double th = tri_angle(centers + 3 * a, centers + 3 * b, points + 3 * p);
        const unsigned long long at = atomicAdd(&cursor[pair], m);
        for (unsigned long long c = 0; c < m; ++c) angles[at + c] = th;
      }
    }
  }
}

// Scores from the sorted angle lists: the count, or 0 when angle[int(0.75 * count)] < 1 degree
// (colmap2mvsnet.py:297-301); written symmetric, with 0 on the diagonal.
__global__ void k_pair_scores(const unsigned long long *count, const unsigned long long *offset, const double *sorted,
                              int N, double *scores) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)N * N) return;
  const int a = (int)(q / N), b = (int)(q % N);
  if (a > b) return;
  double s = 0.0;
  if (a < b) {
    const unsigned long long n = count[q];
    if (n > 0) {
      const double t = sorted[offset[q] + (3 * n) / 4];  // int(len * 0.75), exact for len < 2^51
      s = t < 1.0 ? 0.0 : (double)n;
    }
  }
  scores[(size_t)a * N + b] = s;
  scores[(size_t)b * N + a] = s;
}

__global__ void k_segment_ends(const unsigned long long *offset, const unsigned long long *count, long long n,
                               unsigned long long *end) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) end[q] = offset[q] + count[q];
}

}  // namespace

extern "C" int dpe_view_scores(dpe_ctx *ctx, const dpe_sparse_model *m, double *scores_out) {
  if (!ctx || !m || !scores_out || m->num_images < 1 || !m->centers || !m->obs_offsets) return DPE_ERR_INVALID_ARGUMENT;
  const int N = m->num_images;
  const long long nobs = m->obs_offsets[N];
  if (m->obs_offsets[0] != 0 || nobs < 0 || (nobs > 0 && !m->obs_point) || m->num_points < 0 ||
      (m->num_points > 0 && !m->points))
    return DPE_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < N; ++i)
    if (m->obs_offsets[i + 1] < m->obs_offsets[i]) return DPE_ERR_INVALID_ARGUMENT;
  for (long long k = 0; k < nobs; ++k)
    if (m->obs_point[k] >= m->num_points || m->obs_point[k] < -1) return DPE_ERR_INVALID_ARGUMENT;
  if ((unsigned long long)m->num_points * (unsigned long long)N >= kNoPoint / 2) return DPE_ERR_INVALID_ARGUMENT;
  DPE_TRY(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  Arena &A = ctx->arena;
  const size_t NN = (size_t)N * N;
  long long *d_off = A.get<long long>("v_off", N + 1);
  int32_t *d_obs = A.get<int32_t>("v_obs", nobs + 1);
  double *d_centers = A.get<double>("v_centers", 3 * (size_t)N);
  double *d_points = A.get<double>("v_points", 3 * (size_t)m->num_points + 3);
  unsigned long long *keys = A.get<unsigned long long>("v_keys", nobs + 1);
  unsigned long long *keys_sorted = A.get<unsigned long long>("v_keys_sorted", nobs + 1);
  unsigned long long *run_key = A.get<unsigned long long>("v_run_key", nobs + 1);
  int *run_len = A.get<int>("v_run_len", nobs + 1);
  int *num_runs = A.get<int>("v_num_runs", 1);
  unsigned long long *count = A.get<unsigned long long>("v_count", NN);
  unsigned long long *offset = A.get<unsigned long long>("v_offset", NN + 1);
  unsigned long long *cursor = A.get<unsigned long long>("v_cursor", NN);
  unsigned long long *end = A.get<unsigned long long>("v_end", NN);
  double *d_scores = A.get<double>("v_scores", NN);
  if (!A.ok()) return DPE_ERR_OUT_OF_MEMORY;
  DPE_TRY(cudaMemcpyAsync(d_off, m->obs_offsets, (N + 1) * sizeof(long long), cudaMemcpyHostToDevice, s));
  if (nobs > 0) DPE_TRY(cudaMemcpyAsync(d_obs, m->obs_point, nobs * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  DPE_TRY(cudaMemcpyAsync(d_centers, m->centers, 3 * (size_t)N * sizeof(double), cudaMemcpyHostToDevice, s));
  if (m->num_points > 0)
    DPE_TRY(cudaMemcpyAsync(d_points, m->points, 3 * (size_t)m->num_points * sizeof(double), cudaMemcpyHostToDevice, s));
  DPE_TRY(cudaMemsetAsync(count, 0, NN * sizeof(unsigned long long), s));
  DPE_TRY(cudaMemsetAsync(num_runs, 0, sizeof(int), s));
  if (nobs > 0) {
    k_obs_keys<<<N, 256, 0, s>>>(d_off, d_obs, N, keys);
    DPE_LAUNCHED("k_obs_keys", s);
    size_t tmp_sort = 0, tmp_rle = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, tmp_sort, keys, keys_sorted, (int)nobs, 0, 64, s);
    cub::DeviceRunLengthEncode::Encode(nullptr, tmp_rle, keys_sorted, run_key, run_len, num_runs, (int)nobs, s);
    void *tmp = A.get<uint8_t>("v_tmp", std::max(tmp_sort, tmp_rle) + 16);
    if (!A.ok()) return DPE_ERR_OUT_OF_MEMORY;
    DPE_TRY(cub::DeviceRadixSort::SortKeys(tmp, tmp_sort, keys, keys_sorted, (int)nobs, 0, 64, s));
    DPE_TRY(cub::DeviceRunLengthEncode::Encode(tmp, tmp_rle, keys_sorted, run_key, run_len, num_runs, (int)nobs, s));
    const unsigned grid = (unsigned)std::min<long long>((nobs + 127) / 128, (long long)ctx->sms * 16);
    k_track_pairs<0><<<grid, 128, 0, s>>>(run_key, run_len, num_runs, N, d_centers, d_points, count, nullptr, nullptr);
    DPE_LAUNCHED("k_track_pairs", s);
  }
  size_t tmp_scan = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp_scan, count, offset, (int)NN, s);
  void *tmp2 = A.get<uint8_t>("v_tmp_scan", tmp_scan + 16);
  if (!A.ok()) return DPE_ERR_OUT_OF_MEMORY;
  DPE_TRY(cub::DeviceScan::ExclusiveSum(tmp2, tmp_scan, count, offset, (int)NN, s));
  unsigned long long total = 0;
  if (NN > 0) {
    unsigned long long last_off = 0, last_cnt = 0;
    DPE_TRY(cudaMemcpyAsync(&last_off, offset + NN - 1, 8, cudaMemcpyDeviceToHost, s));
    DPE_TRY(cudaMemcpyAsync(&last_cnt, count + NN - 1, 8, cudaMemcpyDeviceToHost, s));
    DPE_TRY(cudaStreamSynchronize(s));
    total = last_off + last_cnt;
  }
  double *angles = A.get<double>("v_angles", total + 1);
  double *angles_sorted = A.get<double>("v_angles_sorted", total + 1);
  if (!A.ok()) return DPE_ERR_OUT_OF_MEMORY;
  if (total > 0) {
    DPE_TRY(cudaMemcpyAsync(cursor, offset, NN * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, s));
    const unsigned grid = (unsigned)std::min<long long>((nobs + 127) / 128, (long long)ctx->sms * 16);
    k_track_pairs<1><<<grid, 128, 0, s>>>(run_key, run_len, num_runs, N, d_centers, d_points, count, cursor, angles);
    DPE_LAUNCHED("k_track_pairs", s);
    k_segment_ends<<<(unsigned)((NN + 255) / 256), 256, 0, s>>>(offset, count, (long long)NN, end);
    DPE_LAUNCHED("k_segment_ends", s);
    size_t tmp_seg = 0;
    cub::DeviceSegmentedRadixSort::SortKeys(nullptr, tmp_seg, angles, angles_sorted, (long long)total, (long long)NN,
                                            offset, end, 0, 64, s);
    void *tmp3 = A.get<uint8_t>("v_tmp_seg", tmp_seg + 16);
    if (!A.ok()) return DPE_ERR_OUT_OF_MEMORY;
    DPE_TRY(cub::DeviceSegmentedRadixSort::SortKeys(tmp3, tmp_seg, angles, angles_sorted, (long long)total,
                                                    (long long)NN, offset, end, 0, 64, s));
  }
  k_pair_scores<<<(unsigned)((NN + 255) / 256), 256, 0, s>>>(count, offset, angles_sorted, N, d_scores);
  DPE_LAUNCHED("k_pair_scores", s);
  DPE_TRY(cudaMemcpyAsync(scores_out, d_scores, NN * sizeof(double), cudaMemcpyDeviceToHost, s));
  DPE_TRY(cudaStreamSynchronize(s));
  return DPE_OK;
}
