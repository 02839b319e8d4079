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
    arr = (D.FusionView * len(views))()
    keep = []
    total = 0
    for i, v in enumerate(views):
        fv = arr[i]
        H, W = v["depth"].shape[:2]
        fv.width, fv.height = W, H
        fv.depth = v["depth"].ctypes.data
        fv.normal = v["normal"].ctypes.data
        fv.weak = v["weak"].ctypes.data
        fv.bgr = v["bgr"].ctypes.data
        fv.block_mask = v["block"].ctypes.data if v.get("block") is not None else None
        fv.camera = D.make_camera(v["camera"])
        src = np.ascontiguousarray(np.asarray(v["src"], dtype=np.int32))
        keep.append(src)
        fv.num_src = len(src)
        fv.src_views = src.ctypes.data if len(src) else None
        total += W * H
    cap = total if capacity is None else capacity
    xyz = np.zeros((max(cap, 1), 3), np.float32)
    bgr = np.zeros((max(cap, 1), 3), np.uint8)
    origin = np.zeros((max(cap, 1), 2), np.int32)
    ncons = np.zeros(max(cap, 1), np.uint8)
    fin = D.FusionIn(len(views), arr, mode, D.MEM_HOST, min_consistent)
    fo = D.FusionOut()
    fo.capacity = cap
    fo.xyz, fo.bgr, fo.origin, fo.num_consistent = xyz.ctypes.data, bgr.ctypes.data, origin.ctypes.data, ncons.ctypes.data
    st = load().oracle_fuse(C.byref(fin), C.byref(fo))
    n = int(fo.count)
    if st not in (0, D.ERR_CAPACITY):
        raise RuntimeError(f"oracle_fuse failed with status {st}")
    n_keep = min(n, cap)
    return dict(count=n, status=st, xyz=xyz[:n_keep], bgr=bgr[:n_keep], origin=origin[:n_keep],
                num_consistent=ncons[:n_keep])
