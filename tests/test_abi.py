"""CPU tests of the C-ABI boundary: the library loads, exports what include/*.h declares, and its
struct layouts agree with the ctypes mirror.  No compute calls (no GPU here)."""
import ctypes as C
import glob
import os
import re
import subprocess

import pytest

import dpe_b200 as D

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = set()
    for hdr in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(hdr).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(dpe_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = _declared_functions()
    for n in ("dpe_ctx_create", "dpe_ctx_destroy", "dpe_pm_run", "dpe_fuse", "dpe_ncc_eval"):
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = D.load_library()
    missing = [n for n in _declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings_and_defaults():
    lib = D.load_library()
    assert lib.dpe_status_string(D.OK) == b"ok"
    assert b"invalid" in lib.dpe_status_string(D.ERR_INVALID_ARGUMENT)
    p = D.default_params(lib)
    # PatchMatchParams defaults, main.h:81-109
    assert (p.max_iterations, p.top_k, p.strong_radius, p.strong_increment, p.weak_radius, p.weak_increment) == (3, 4, 5, 2, 5, 5)
    assert abs(p.sigma_spatial - 5.0) < 1e-7 and abs(p.sigma_color - 3.0) < 1e-7
    assert abs(p.ransac_threshold - 0.005) < 1e-9 and abs(p.geom_factor - 0.2) < 1e-7
    assert (p.use_APD, p.use_edge, p.use_limit, p.use_label, p.use_radius, p.high_res_img) == (1, 1, 1, 1, 1, 1)


def test_null_arguments_rejected_without_device():
    lib = D.load_library()
    assert lib.dpe_pm_run(None, None, None) == D.ERR_INVALID_ARGUMENT
    assert lib.dpe_fuse(None, None, None) == D.ERR_INVALID_ARGUMENT
    assert lib.dpe_ncc_eval(None, None, None) == D.ERR_INVALID_ARGUMENT
    assert lib.dpe_ctx_destroy(None) == D.OK


def test_struct_layouts_match_header(tmp_path):
    """Compile a probe against include/dpe_b200.h and compare sizeof/offsetof with ctypes."""
    src = tmp_path / "probe.c"
    src.write_text("""
#include <stdio.h>
#include <stddef.h>
#include "dpe_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(dpe_camera), sizeof(dpe_params), sizeof(dpe_problem),
         sizeof(dpe_pm_out), sizeof(dpe_fusion_view), sizeof(dpe_fusion_in), sizeof(dpe_fusion_out), sizeof(dpe_ncc_query));
  printf("%zu %zu %zu\\n", offsetof(dpe_problem, params), offsetof(dpe_problem, seed), offsetof(dpe_fusion_view, camera));
  return 0;
}
""")
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    lines = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    sizes = [int(x) for x in lines[0].split()]
    offs = [int(x) for x in lines[1].split()]
    assert sizes == [C.sizeof(t) for t in (D.Camera, D.Params, D.Problem, D.PMOut, D.FusionView, D.FusionIn,
                                           D.FusionOut, D.NCCQuery)]
    assert sizes[0] == 112  # reference Camera, main.h:53-62
    assert offs == [D.Problem.params.offset, D.Problem.seed.offset, D.FusionView.camera.offset]


def test_python_reference_defaults_match_library():
    """dpe_b200.reference_default_params (no library) equals dpe_params_default field for field."""
    lib = D.load_library()
    a, b = D.default_params(lib), D.reference_default_params()
    for name, _ in D.Params._fields_:
        assert getattr(a, name) == getattr(b, name), name
