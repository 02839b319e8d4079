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
    lib.oracle_set_raw_moments.argtypes = [C.c_int]
    lib.oracle_ncc_strong_grad.argtypes = [C.POINTER(D.NCCQuery), C.c_void_p, C.c_void_p, C.c_void_p]
    _lib = lib
    return lib


def set_raw_moments(on: bool) -> None:
    """Select the reference's raw-moment NCC arithmetic (default: compensated, shifted moments)."""
    load().oracle_set_raw_moments(1 if on else 0)


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
