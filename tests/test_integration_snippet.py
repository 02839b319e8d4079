"""The C++ binding that INTEGRATION.md shows a maintainer adding to the reference host compiles: its
code blocks are extracted, put in one translation unit with the reference's own headers (DPE.h,
main.h, behind the OpenCV / Boost / CUDA stand-ins of oracle/refshim) and this library's
include/dpe_b200.h, linked against libdpe_sm100.so, and the program runs the C-ABI's status paths
(no device is needed for those)."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFERENCE = os.environ.get("DPE_REFERENCE_DIR", "/root/reference")

pytestmark = pytest.mark.skipif(not os.path.exists(os.path.join(REFERENCE, "DPE.h")),
                                reason="the reference headers are absent")

PRELUDE = r"""
#include <cstring>
#include <iostream>
#include "DPE.h"
#include "dpe_b200.h"

// INTEGRATION.md: "CopyParams copies PatchMatchParams into dpe_params one field at a time"
static void CopyParams(const PatchMatchParams &r, dpe_params *p) {
  p->max_iterations = r.max_iterations; p->num_images = r.num_images; p->sigma_spatial = r.sigma_spatial;
  p->sigma_color = r.sigma_color; p->top_k = r.top_k; p->depth_min = r.depth_min; p->depth_max = r.depth_max;
  p->geom_consistency = r.geom_consistency; p->strong_radius = r.strong_radius;
  p->strong_increment = r.strong_increment; p->weak_radius = r.weak_radius; p->weak_increment = r.weak_increment;
  p->use_APD = r.use_APD; p->use_edge = r.use_edge; p->use_limit = r.use_limit; p->use_label = r.use_label;
  p->use_radius = r.use_radius; p->high_res_img = r.high_res_img; p->max_scale_size = r.max_scale_size;
  p->scale_size = r.scale_size; p->weak_peak_radius = r.weak_peak_radius; p->rotate_time = r.rotate_time;
  p->ransac_threshold = r.ransac_threshold; p->geom_factor = r.geom_factor; p->state = r.state;
}
"""

MAIN = r"""
int main() {
  // status paths, no device needed: every entry point rejects null arguments without exiting
  if (dpe_pm_run(nullptr, nullptr, nullptr) != DPE_ERR_INVALID_ARGUMENT) return 1;
  if (dpe_fuse(nullptr, nullptr, nullptr) != DPE_ERR_INVALID_ARGUMENT) return 2;
  if (dpe_scene_run(nullptr, nullptr, nullptr, nullptr) != DPE_ERR_INVALID_ARGUMENT) return 3;
  if (std::strcmp(dpe_status_string(DPE_OK), "ok") != 0) return 4;
  dpe_params p;
  dpe_params_default(&p);
  PatchMatchParams ref;  // the reference's member defaults (state has none)
  ref.state = FIRST_INIT;
  dpe_params q;
  CopyParams(ref, &q);
  if (std::memcmp(&p, &q, sizeof(p)) != 0) return 5;
  std::cout << "binding ok" << std::endl;
  return 0;
}
"""


def _cpp_blocks():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    return re.findall(r"```cpp\n(.*?)```", text, flags=re.S)


def test_integration_binding_compiles_and_runs(tmp_path):
    blocks = _cpp_blocks()
    assert len(blocks) >= 2
    body = []
    for b in blocks:
        b = b.replace('#include "dpe_b200.h"\n', "")
        if b.lstrip().startswith("//") and "dpe_edge_map(ctx" in b:
            # statements, not a definition: wrap them in a function of the names they use
            b = ("static void EdgeBinding(dpe_ctx *ctx, const cv::Mat &level_u8, cv::Mat &edge, const cv::Mat "
                 "&image_uint, cv::Mat &label, int scale, const PatchMatchParams &params) {\n" + b + "}\n")
        body.append(b)
    src = tmp_path / "binding.cpp"
    src.write_text(PRELUDE + "\n".join(body) + MAIN)
    exe = tmp_path / "binding"
    lib_dir = os.path.join(ROOT, "dpe-mvs-fast_b200")
    cmd = ["g++", "-std=c++17", "-w", "-I", os.path.join(ROOT, "oracle", "refshim"), "-I", REFERENCE, "-I",
           os.path.join(ROOT, "include"), str(src), "-o", str(exe), "-L", lib_dir, "-ldpe_sm100",
           f"-Wl,-rpath,{lib_dir}", "-Wl,--unresolved-symbols=ignore-in-object-files"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0 and "binding ok" in out.stdout, (out.returncode, out.stdout, out.stderr)
