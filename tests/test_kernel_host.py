"""CPU tests of the CUDA kernel logic: pm_kernels.cuh compiled for the host (tests/kernel_host)
must reproduce the oracle bit for bit on every path of the per-view call (strong, weak, geom).
On the GPU the same source differs from the oracle only by FMA contraction and the last-ulp
behaviour of expf/sinf/cosf; that is what test_gpu_parity.py measures."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import dpe_b200 as D
import helpers as h
import oracle_py as O

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "kernel_host", "kernel_host.cpp")
LIB = os.path.join(HERE, "kernel_host", "libkernel_host.so")


def _build():
    deps = [SRC] + [os.path.join(HERE, "..", "dpe-mvs-fast_b200", "csrc", f) for f in ("pm_kernels.cuh", "dpe_device.cuh")]
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(d) for d in deps):
        cmd = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
               "-I/usr/local/cuda/include", SRC, "-o", LIB]
        subprocess.run(cmd, check=True)
    lib = C.CDLL(LIB)
    lib.host_pm_run.argtypes = [C.POINTER(D.Problem), C.POINTER(D.PMOut)]
    return lib


@pytest.fixture(scope="module")
def host_lib():
    return _build()


def _run(lib, images, cams, p, **kw):
    pr = D.build_problem(images, cams, p, **kw)
    H, W = pr.height, pr.width
    out = dict(plane=np.zeros((H, W, 4), np.float32), weak=np.zeros((H, W), np.uint8),
               views=np.zeros((H, W), np.uint32), costs=np.zeros((H, W), np.float32))
    po = D.PMOut()
    po.plane, po.weak, po.selected_views, po.costs = [out[k].ctypes.data for k in ("plane", "weak", "views", "costs")]
    lib.host_pm_run(C.byref(pr), C.byref(po))
    return out


def _assert_identical(a, b):
    for k in ("plane", "weak", "views", "costs"):
        assert np.array_equal(a[k], b[k], equal_nan=True), k


def test_first_init_bit_exact(host_lib, small_scene):
    images, cams, _ = h.view_inputs(small_scene, 0)
    p = h.first_init_params(small_scene, len(images))
    _assert_identical(_run(host_lib, images, cams, p, seed=3), O.pm_run(images, cams, p, seed=3))


@pytest.mark.parametrize("geom", [False, True])
def test_weak_path_bit_exact(host_lib, geom):
    ws = h.S.make_scene("small_weak", seed=2)
    ref = 2 if geom else 1
    images, cams, srcs = h.view_inputs(ws, ref)
    p0 = h.first_init_params(ws, len(images))
    o0 = O.pm_run(images, cams, p0, seed=21)
    state, weak = h.post_process(o0["plane"], o0["weak"], p0.depth_min, p0.depth_max)
    edge, low, label = h.synthetic_edges(ws.gray[ref])
    p = h.refine_params(ws, len(images), level=1, state=D.REFINE_ITER if geom else D.REFINE_INIT, geom=geom)
    kw = dict(plane_in=state, views_in=np.ascontiguousarray(o0["views"]), weak_in=weak, edge=edge, edge_low=low,
              label=label, seed=77)
    if geom:
        kw["depths"] = [np.ascontiguousarray(ws.depth[i].astype(np.float32)) for i in [ref] + list(srcs)]
    _assert_identical(_run(host_lib, images, cams, p, **kw), O.pm_run(images, cams, p, **kw))
