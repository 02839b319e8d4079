"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the cpu_baseline leg of
bench.py as the checker.  The product path never loads it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from typing import Dict, List, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "dpe-mvs-fast_b200"))
import dpe_b200 as D  # noqa: E402  (struct layouts of the shared ABI header)

LIB_PATH = os.path.join(HERE, "liboracle.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    lib.oracle_philox.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.oracle_ncc_strong.argtypes = [C.POINTER(D.NCCQuery), C.c_int, C.c_void_p]
    lib.oracle_pm_run.argtypes = [C.POINTER(D.Problem), C.POINTER(D.PMOut), C.c_int]
    lib.oracle_fuse.argtypes = [C.POINTER(D.FusionIn), C.POINTER(D.FusionOut)]
    lib.oracle_fuse_tat.argtypes = [C.POINTER(D.FusionIn), C.c_int, C.POINTER(D.FusionOut)]
    lib.oracle_connect.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    lib.oracle_resize_u8.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int]
    lib.oracle_hough_lines_p.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                         C.c_void_p]
    lib.oracle_edge_labels.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int]
    lib.oracle_set_raw_moments.argtypes = [C.c_int]
    lib.oracle_set_ref_addressing.argtypes = [C.c_int]
    lib.oracle_set_serial_race.argtypes = [C.c_int]
    lib.oracle_set_ref_homography.argtypes = [C.c_int]
    lib.oracle_ncc_strong_grad.argtypes = [C.POINTER(D.NCCQuery), C.c_void_p, C.c_void_p, C.c_void_p]
    _lib = lib
    return lib


def set_raw_moments(on: bool) -> None:
    """Select the reference's raw-moment NCC arithmetic (default: compensated, shifted moments)."""
    load().oracle_set_raw_moments(1 if on else 0)


def set_ref_addressing(on: bool) -> None:
    """Sample positions pass through the reference's tex2D(x + 0.5, y + 0.5) rounding (default: sampled
    at x, the CUDA kernels' addressing)."""
    load().oracle_set_ref_addressing(1 if on else 0)


def set_ref_homography(on: bool) -> None:
    """Compose the homography in the reference's float operation order (DPE.cu:457-517) instead of
    from camera products composed in double and rounded once (the CUDA kernels' form)."""
    load().oracle_set_ref_homography(1 if on else 0)


def set_serial_race(on: bool) -> None:
    """Resolve the edge-aware update's same-colour read race (Q1) as a serial raster-order run does
    (default: a snapshot taken before each colour pass, the CUDA kernels' resolution)."""
    load().oracle_set_serial_race(1 if on else 0)


def reference_arithmetic(on: bool) -> None:
    """Raw moments, the reference's texture addressing and its float homography together: the
    arithmetic of the reference's own DPE.cu, for bit-for-bit comparison with its host build
    (oracle/ref_py.py)."""
    set_raw_moments(on)
    set_ref_addressing(on)
    set_ref_homography(on)


def philox(ctr, key) -> np.ndarray:
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros(4, np.uint32)
    load().oracle_philox(c.ctypes.data, k.ctypes.data, out.ctypes.data)
    return out


def ncc_strong(images, cameras, params, px, py, src, planes, fp64: bool) -> np.ndarray:
    q = D.make_query(images, cameras, params, px, py, src, planes)
    out = np.zeros(len(q.keep[0]), np.float64)
    load().oracle_ncc_strong(C.byref(q.struct), 1 if fp64 else 0, out.ctypes.data)
    return out


def ncc_strong_grad(images, cameras, params, px, py, src, planes, want_images: bool = False):
    """FP64 strong NCC and its gradient: (cost (n,), dC/d(nx, ny, nz, w) (n, 4), and with
    want_images the gradient of the summed cost w.r.t. each image's pixels (list, entry 0 None))."""
    q = D.make_query(images, cameras, params, px, py, src, planes)
    n = len(q.keep[0])
    cost = np.zeros(n, np.float64)
    grad = np.zeros((n, 4), np.float64)
    gimg = None
    ptrs = None
    if want_images:
        H, W = images[0].shape
        gimg = [None] + [np.zeros((H, W), np.float64) for _ in images[1:]]
        ptrs = (C.c_void_p * len(images))(*([None] + [g.ctypes.data for g in gimg[1:]]))
    load().oracle_ncc_strong_grad(C.byref(q.struct), cost.ctypes.data, grad.ctypes.data, ptrs)
    return cost, grad, gimg


def pm_run(images, cameras, params, threads: int = 0, **kw) -> Dict:
    pr = D.build_problem(images, cameras, params, **kw)
    H, W = pr.height, pr.width
    out = dict(plane=np.zeros((H, W, 4), np.float32), weak=np.zeros((H, W), np.uint8),
               views=np.zeros((H, W), np.uint32), costs=np.zeros((H, W), np.float32))
    po = D.PMOut()
    po.plane, po.weak, po.selected_views, po.costs = (out["plane"].ctypes.data, out["weak"].ctypes.data,
                                                      out["views"].ctypes.data, out["costs"].ctypes.data)
    st = load().oracle_pm_run(C.byref(pr), C.byref(po), threads)
    if st != 0:
        raise RuntimeError(f"oracle_pm_run failed with status {st}")
    return out


def fuse(views: List[Dict], mode: int = D.FUSE_FP64, capacity: Optional[int] = None, min_consistent: int = 1) -> Dict:
    """The CPU restatement of RunFusion (DPE.cpp:1387-1548)."""
    fin, keep, cap = D.fusion_input(views, mode, D.MEM_HOST, min_consistent, capacity)
    fo, arrays = D.fusion_output(cap)
    st = load().oracle_fuse(C.byref(fin), C.byref(fo))
    if st not in (0, D.ERR_CAPACITY):
        raise RuntimeError(f"oracle_fuse failed with status {st}")
    return D.fusion_result(fo, arrays, status=st)


def fuse_tat(views: List[Dict], variant: int = D.TAT_INTERMEDIATE, mode: int = D.FUSE_FLOAT,
             capacity: Optional[int] = None) -> Dict:
    """The CPU restatement of RunFusion_TAT_Intermediate / RunFusion_TAT_advanced
    (DPE.cpp:1550-1867)."""
    fin, keep, cap = D.fusion_input(views, mode, D.MEM_HOST, 1, capacity)
    fo, arrays = D.fusion_output(cap)
    st = load().oracle_fuse_tat(C.byref(fin), variant, C.byref(fo))
    if st not in (0, D.ERR_CAPACITY):
        raise RuntimeError(f"oracle_fuse_tat failed with status {st}")
    return D.fusion_result(fo, arrays, status=st)


def connect(img: np.ndarray):
    """The CPU restatement of Connect (DPE.cpp:27-134): (labels int32, counts per label)."""
    img = np.ascontiguousarray(img, dtype=np.uint8)
    rows, cols = img.shape
    labels = np.zeros((rows, cols), np.int32)
    cap = rows * cols + 1
    counts = np.zeros(cap, np.int32)
    n = C.c_int(0)
    st = load().oracle_connect(img.ctypes.data, cols, rows, labels.ctypes.data, counts.ctypes.data, cap, C.byref(n))
    if st != 0:
        raise RuntimeError(f"oracle_connect failed with status {st}")
    return labels, counts[: n.value].copy()


def resize_u8(img: np.ndarray, width: int, height: int) -> np.ndarray:
    """cv::resize(img, (width, height), INTER_LINEAR) for an 8-bit image, restated."""
    img = np.ascontiguousarray(img, dtype=np.uint8)
    out = np.zeros((height, width), np.uint8)
    if load().oracle_resize_u8(img.ctypes.data, img.shape[1], img.shape[0], out.ctypes.data, width, height) != 0:
        raise RuntimeError("oracle_resize_u8 failed")
    return out


def hough_lines_p(img: np.ndarray, threshold: int, min_line_length: int, max_line_gap: int) -> List:
    """cv::HoughLinesP(img, 1, CV_PI / 180, threshold, min_line_length, max_line_gap), restated."""
    img = np.ascontiguousarray(img, dtype=np.uint8)
    cap = 1 << 16
    buf = np.zeros((cap, 4), np.int32)
    n = C.c_int(0)
    st = load().oracle_hough_lines_p(img.ctypes.data, img.shape[1], img.shape[0], threshold, min_line_length,
                                     max_line_gap, buf.ctypes.data, cap, C.byref(n))
    if st != 0:
        raise RuntimeError(f"oracle_hough_lines_p failed with status {st}")
    return [tuple(int(v) for v in r) for r in buf[: n.value]]


def edge_labels(gray: np.ndarray, scale: int, high_res_img: bool = True) -> np.ndarray:
    """EdgeSegment(scale, gray, 1, false, high_res_img) (DPE.cpp:136-291), restated: the int32 label
    map at the level size, 0 on edges and -1 on small regions."""
    gray = np.ascontiguousarray(gray, dtype=np.uint8)
    rows, cols = gray.shape
    f = np.float32(1.0) / np.float32(1 << scale)
    w, h = int(np.round(np.float32(cols) * f)), int(np.round(np.float32(rows) * f))
    out = np.zeros((h, w), np.int32)
    if load().oracle_edge_labels(gray.ctypes.data, cols, rows, scale, 1 if high_res_img else 0, out.ctypes.data,
                                 w, h) != 0:
        raise RuntimeError("oracle_edge_labels failed")
    return out
