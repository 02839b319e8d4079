// fusion_oracle.cpp -- CPU restatement of RunFusion (DPE.cpp:1387-1548), ETH variant, and of
// the two TAT variants RunFusion_TAT_Intermediate (DPE.cpp:1550-1718) and RunFusion_TAT_advanced
// (DPE.cpp:1720-1867).
//
// TEST INFRASTRUCTURE ONLY: the checker for the fusion kernels.
// PARITY PINNED to the reference itself: the float mode gives the same points, coordinates and
// colours bit for bit as the reference's own RunFusion compiled for the CPU (oracle/_ref, driven
// by oracle/ref_harness.cpp; tests/test_ref_oracle.py).  The TAT variants are checked against an
// independent numpy restatement (tests/test_fusion_tat.py) and their golden fixtures.
// The loop order is the
// reference's: views in pair.txt order, pixels in raster order, sources in list order, with the
// consumed-pixel masks updated as points are accepted, so the result depends on that order
// exactly as the reference's does.  Two arithmetic modes:
//   DPE_FUSE_FP64  -- the reprojection / relative-depth / angle test and the score in double;
//   DPE_FUSE_FLOAT -- the reference's float arithmetic (pow/sqrt of the reprojection error in
//                     double as C++ promotes them, DPE.cpp:1504).
// In both modes the emitted coordinates are the float back-projection of DPE.cpp:1337-1359 and
// the colour is the float mean truncated to uchar (ExportPointCloud, DPE.cpp:549-551).
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle_common.h"

namespace oracle {

// Get3DPointonWorld, DPE.cpp:1337-1359 (recomputes the centre from R, t in float)
template <class T> static inline void world_point(T x, T y, T depth, const dpe_camera &c, T out[3]) {
  const T px = depth * (x - (T)c.K[2]) / (T)c.K[0];
  const T py = depth * (y - (T)c.K[5]) / (T)c.K[4];
  const T pz = depth;
  const T tx = (T)c.R[0] * px + (T)c.R[3] * py + (T)c.R[6] * pz;
  const T ty = (T)c.R[1] * px + (T)c.R[4] * py + (T)c.R[7] * pz;
  const T tz = (T)c.R[2] * px + (T)c.R[5] * py + (T)c.R[8] * pz;
  const T Cx = -((T)c.R[0] * (T)c.t[0] + (T)c.R[3] * (T)c.t[1] + (T)c.R[6] * (T)c.t[2]);
  const T Cy = -((T)c.R[1] * (T)c.t[0] + (T)c.R[4] * (T)c.t[1] + (T)c.R[7] * (T)c.t[2]);
  const T Cz = -((T)c.R[2] * (T)c.t[0] + (T)c.R[5] * (T)c.t[1] + (T)c.R[8] * (T)c.t[2]);
  out[0] = tx + Cx; out[1] = ty + Cy; out[2] = tz + Cz;
}
// ProjectCamera, DPE.cpp:1361-1371
template <class T> static inline void project(const T X[3], const dpe_camera &c, T &u, T &v, T &depth) {
  const T tx = (T)c.R[0] * X[0] + (T)c.R[1] * X[1] + (T)c.R[2] * X[2] + (T)c.t[0];
  const T ty = (T)c.R[3] * X[0] + (T)c.R[4] * X[1] + (T)c.R[5] * X[2] + (T)c.t[1];
  const T tz = (T)c.R[6] * X[0] + (T)c.R[7] * X[1] + (T)c.R[8] * X[2] + (T)c.t[2];
  depth = (T)c.K[6] * tx + (T)c.K[7] * ty + (T)c.K[8] * tz;
  u = ((T)c.K[0] * tx + (T)c.K[1] * ty + (T)c.K[2] * tz) / depth;
  v = ((T)c.K[3] * tx + (T)c.K[4] * ty + (T)c.K[5] * tz) / depth;
}

}  // namespace oracle

using namespace oracle;

extern "C" int oracle_fuse(const dpe_fusion_in *in, dpe_fusion_out *out) {
  if (!in || !out || in->memory != DPE_MEM_HOST) return DPE_ERR_INVALID_ARGUMENT;
  const int nv = in->num_views;
  std::vector<std::vector<uint8_t>> masks(nv);
  for (int i = 0; i < nv; ++i) masks[i].assign((size_t)in->views[i].width * in->views[i].height, 0);
  int64_t count = 0;
  for (int i = 0; i < nv; ++i) {
    const dpe_fusion_view &V = in->views[i];
    const int cols = V.width, rows = V.height, ns = V.num_src;
    std::vector<int> used_c(ns), used_r(ns);
    for (int r = 0; r < rows; ++r)
      for (int c = 0; c < cols; ++c) {
        const size_t pix = (size_t)r * cols + c;
        if (V.block_mask && V.block_mask[pix] < 128) continue;
        if (masks[i][pix] == 1) continue;
        const float ref_depth = V.depth[pix];
        if (ref_depth <= 0.0) continue;
        const float *rn = &V.normal[3 * pix];
        float Xf[3];
        world_point<float>((float)c, (float)r, ref_depth, V.camera, Xf);
        double Xd[3];
        world_point<double>((double)c, (double)r, (double)ref_depth, V.camera, Xd);
        int n_cons = 0;
        float dyn_f = 0.0f;
        double dyn_d = 0.0;
        for (int j = 0; j < ns; ++j) {
          used_c[j] = -1; used_r[j] = -1;
          const int s = V.src_views[j];
          const dpe_fusion_view &S = in->views[s];
          int src_r, src_c;
          if (in->mode == DPE_FUSE_FP64) {
            double u, v, pd;
            project<double>(Xd, S.camera, u, v, pd);
            src_r = f2i(v + 0.5); src_c = f2i(u + 0.5);
          } else {
            float u, v, pd;
            project<float>(Xf, S.camera, u, v, pd);
            src_r = f2i(v + 0.5f); src_c = f2i(u + 0.5f);
          }
          if (!(src_c >= 0 && src_c < S.width && src_r >= 0 && src_r < S.height)) continue;
          const size_t sp = (size_t)src_r * S.width + src_c;
          if (masks[s][sp] == 1) continue;
          const float src_depth = S.depth[sp];
          if (src_depth <= 0.0) continue;
          const float *sn = &S.normal[3 * sp];
          bool ok;
          if (in->mode == DPE_FUSE_FP64) {
            double T[3], u, v, pd;
            world_point<double>((double)src_c, (double)src_r, (double)src_depth, S.camera, T);
            project<double>(T, V.camera, u, v, pd);
            const double ex = (double)c - u, ey = (double)r - v;
            const double reproj = std::sqrt(ex * ex + ey * ey);
            const double rel = std::fabs(pd - (double)ref_depth) / (double)ref_depth;
            const double dot = (double)rn[0] * sn[0] + (double)rn[1] * sn[1] + (double)rn[2] * sn[2];
            double ang = std::acos(dot);
            if (ang != ang) ang = 0.0;
            ok = reproj < 2.0 && rel < 0.01 && ang < (double)0.174533f;
            if (ok) dyn_d += std::exp(-(reproj + 200.0 * rel + ang * 10.0));
          } else {
            float T[3], u, v, pd;
            world_point<float>((float)src_c, (float)src_r, src_depth, S.camera, T);
            project<float>(T, V.camera, u, v, pd);
            const float ex = (float)c - u, ey = (float)r - v;
            const float reproj = (float)std::sqrt((double)ex * (double)ex + (double)ey * (double)ey);
            const float rel = std::fabs(pd - ref_depth) / ref_depth;
            const float dot = rn[0] * sn[0] + rn[1] * sn[1] + rn[2] * sn[2];
            float ang = std::acos(dot);
            if (ang != ang) ang = 0.0f;
            ok = reproj < 2.0f && rel < 0.01f && ang < 0.174533f;
            if (ok) dyn_f += (float)std::exp(-(double)(reproj + 200 * rel + ang * 10));
          }
          if (ok) { used_c[j] = src_c; used_r[j] = src_r; n_cons++; }
        }
        const float factor = V.weak[pix] == DPE_WEAK ? 0.45f : 0.3f;
        // the reference rule is n >= 1 (DPE.cpp:1520); min_consistent > 1 raises it
        const int need = in->min_consistent > 1 ? in->min_consistent : 1;
        const bool accept = in->mode == DPE_FUSE_FP64 ? (n_cons >= need && dyn_d > (double)factor * n_cons)
                                                      : (n_cons >= need && dyn_f > factor * n_cons);
        if (!accept) continue;
        const uint8_t *rc = &V.bgr[3 * pix];
        float col[3] = {(float)rc[0], (float)rc[1], (float)rc[2]};
        for (int j = 0; j < ns; ++j) {
          if (used_c[j] == -1) continue;
          const int s = V.src_views[j];
          const size_t sp = (size_t)used_r[j] * in->views[s].width + used_c[j];
          masks[s][sp] = 1;
          const uint8_t *sc = &in->views[s].bgr[3 * sp];
          col[0] += sc[0]; col[1] += sc[1]; col[2] += sc[2];
        }
        col[0] /= (n_cons + 1); col[1] /= (n_cons + 1); col[2] /= (n_cons + 1);
        if (count < out->capacity) {
          out->xyz[3 * count] = Xf[0]; out->xyz[3 * count + 1] = Xf[1]; out->xyz[3 * count + 2] = Xf[2];
          out->bgr[3 * count] = (uint8_t)col[0]; out->bgr[3 * count + 1] = (uint8_t)col[1]; out->bgr[3 * count + 2] = (uint8_t)col[2];
          if (out->origin) { out->origin[2 * count] = i; out->origin[2 * count + 1] = (int32_t)pix; }
          if (out->num_consistent) out->num_consistent[count] = (uint8_t)n_cons;
        }
        count++;
      }
  }
  out->count = count;
  out->gpu_ms = 0.0f;
  return count > out->capacity ? DPE_ERR_CAPACITY : DPE_OK;
}

// RunFusion_TAT_Intermediate (DPE.cpp:1550-1718) and RunFusion_TAT_advanced (DPE.cpp:1720-1867),
// as the reference runs them: one pass per view in order, pixels in raster order, and a per-view
// vector of per-source differences that a pixel overwrites only for the sources it can test
// (DPE.cpp:1640 / 1804), so an untestable source counts with the values it had at the last
// tested pixel.  FLOAT mode is the reference's float arithmetic (the reprojection error's pow /
// sqrt in double as C++ promotes them, DPE.cpp:1672 / 1838); FP64 mode evaluates the
// differences in double and compares them with the same float bounds.
extern "C" int oracle_fuse_tat(const dpe_fusion_in *in, int variant, dpe_fusion_out *out) {
  if (!in || !out || in->memory != DPE_MEM_HOST) return DPE_ERR_INVALID_ARGUMENT;
  if (variant != DPE_TAT_INTERMEDIATE && variant != DPE_TAT_ADVANCED) return DPE_ERR_INVALID_ARGUMENT;
  const bool inter = variant == DPE_TAT_INTERMEDIATE;
  const float dist_base = 0.25f;
  const float depth_base = inter ? 1.0f / 3500.0f : 1.0f / 3000.0f;
  const float angle_base = 0.06981317007977318f;
  const float angle_grad = 0.05235987755982988f;
  struct Diff { double dist, depth, angle; int sr, sc; bool use; };
  const int nv = in->num_views;
  std::vector<std::vector<uint8_t>> masks(nv);
  for (int i = 0; i < nv; ++i) masks[i].assign((size_t)in->views[i].width * in->views[i].height, 0);
  int64_t count = 0;
  for (int i = 0; i < nv; ++i) {
    const dpe_fusion_view &V = in->views[i];
    const int cols = V.width, rows = V.height, ns = V.num_src;
    const double big = std::numeric_limits<float>::max();
    std::vector<Diff> diff(ns, Diff{big, big, big, 0, 0, false});
    for (int r = 0; r < rows; ++r)
      for (int c = 0; c < cols; ++c) {
        const size_t pix = (size_t)r * cols + c;
        if (V.block_mask && V.block_mask[pix] < 128) continue;
        const float ref_depth = V.depth[pix];
        if (ref_depth <= 0.0) continue;
        const float *rn = &V.normal[3 * pix];
        float Xf[3];
        world_point<float>((float)c, (float)r, ref_depth, V.camera, Xf);
        double Xd[3];
        world_point<double>((double)c, (double)r, (double)ref_depth, V.camera, Xd);
        for (int j = 0; j < ns; ++j) {
          const dpe_fusion_view &S = in->views[V.src_views[j]];
          int src_r, src_c;
          if (in->mode == DPE_FUSE_FP64) {
            double u, v, pd;
            project<double>(Xd, S.camera, u, v, pd);
            src_r = f2i(v + 0.5); src_c = f2i(u + 0.5);
          } else {
            float u, v, pd;
            project<float>(Xf, S.camera, u, v, pd);
            src_r = f2i(v + 0.5f); src_c = f2i(u + 0.5f);
          }
          if (!(src_c >= 0 && src_c < S.width && src_r >= 0 && src_r < S.height)) continue;
          const size_t sp = (size_t)src_r * S.width + src_c;
          if (masks[V.src_views[j]][sp] == 1) continue;
          const float src_depth = S.depth[sp];
          if (src_depth <= 0.0) continue;
          const float *sn = &S.normal[3 * sp];
          Diff &d = diff[j];
          if (in->mode == DPE_FUSE_FP64) {
            double T[3], u, v, pd;
            world_point<double>((double)src_c, (double)src_r, (double)src_depth, S.camera, T);
            project<double>(T, V.camera, u, v, pd);
            const double ex = (double)c - u, ey = (double)r - v;
            d.dist = std::sqrt(ex * ex + ey * ey);
            d.depth = std::fabs(pd - (double)ref_depth) / (double)ref_depth;
            const double a = std::acos((double)rn[0] * sn[0] + (double)rn[1] * sn[1] + (double)rn[2] * sn[2]);
            d.angle = a != a ? 0.0 : a;
          } else {
            float T[3], u, v, pd;
            world_point<float>((float)src_c, (float)src_r, src_depth, S.camera, T);
            project<float>(T, V.camera, u, v, pd);
            const float ex = (float)c - u, ey = (float)r - v;
            d.dist = (float)std::sqrt((double)ex * (double)ex + (double)ey * (double)ey);
            d.depth = std::fabs(pd - ref_depth) / ref_depth;
            const float a = std::acos(rn[0] * sn[0] + rn[1] * sn[1] + rn[2] * sn[2]);
            d.angle = a != a ? 0.0f : a;
          }
          d.sr = src_r;
          d.sc = src_c;
        }
        for (int k = 2; k <= ns; ++k) {
          const float bd = (float)k * dist_base, bz = (float)k * depth_base, ba = (float)k * angle_grad + angle_base;
          int n = 0;
          for (int j = 0; j < ns; ++j) {
            const Diff &d = diff[j];
            bool ok;
            if (in->mode == DPE_FUSE_FP64)
              ok = d.dist < (double)bd && d.depth < (double)bz && (!inter || d.angle < (double)ba);
            else
              ok = (float)d.dist < bd && (float)d.depth < bz && (!inter || (float)d.angle < ba);
            diff[j].use = ok;
            n += ok ? 1 : 0;
          }
          if (n < k) continue;
          const uint8_t *rc = &V.bgr[3 * pix];
          float col[3] = {(float)rc[0], (float)rc[1], (float)rc[2]};
          if (inter) {
            for (int j = 0; j < ns; ++j) {
              if (!diff[j].use) continue;
              const dpe_fusion_view &S = in->views[V.src_views[j]];
              const uint8_t *sc = &S.bgr[3 * ((size_t)diff[j].sr * S.width + diff[j].sc)];
              col[0] += (float)sc[0]; col[1] += (float)sc[1]; col[2] += (float)sc[2];
            }
            col[0] /= (n + 1.0f); col[1] /= (n + 1.0f); col[2] /= (n + 1.0f);
          }
          if (count < out->capacity) {
            out->xyz[3 * count] = Xf[0]; out->xyz[3 * count + 1] = Xf[1]; out->xyz[3 * count + 2] = Xf[2];
            out->bgr[3 * count] = (uint8_t)col[0]; out->bgr[3 * count + 1] = (uint8_t)col[1];
            out->bgr[3 * count + 2] = (uint8_t)col[2];
            if (out->origin) { out->origin[2 * count] = i; out->origin[2 * count + 1] = (int32_t)pix; }
            if (out->num_consistent) out->num_consistent[count] = (uint8_t)n;
          }
          count++;
          masks[i][pix] = 1;
          break;
        }
      }
  }
  out->count = count;
  out->gpu_ms = 0.0f;
  return count > out->capacity ? DPE_ERR_CAPACITY : DPE_OK;
}
