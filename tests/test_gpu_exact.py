"""The exact build (libdpe_sm100_exact.so: the kernels without multiply-add contraction, IEEE
division at every tap, and the shared exp / sin / cos of dpe_math.h) against the CPU oracle:
identical bits.  The default build differs from it by rounding only (contraction and the hardware
reciprocal), which is what the statistical bars of the other parity tests measure.

Covered: the strong NCC at random queries; a FIRST_INIT call; the weak-texture REFINE_INIT call
(APD, edges, labels); the geometric REFINE_ITER call; FP16 staging on 8-bit images against FP32.
"""
import numpy as np
import pytest

import dpe_b200 as D
import helpers as h
import oracle_py as O
from test_oracle import _random_queries

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def xctx():
    c = D.Context(0, library=D.EXACT_LIBRARY)
    yield c
    c.close()


def _same(g, o, label):
    for k in ("plane", "weak", "views", "costs"):
        eq = np.array_equal(g[k], o[k], equal_nan=True)
        if not eq:
            diff = ~((g[k] == o[k]) | (np.isnan(g[k]) & np.isnan(o[k])) if g[k].dtype.kind == "f" else (g[k] == o[k]))
            print(f"{label}: {k} differs at {int(diff.sum())} entries")
        assert eq, (label, k)


def test_exact_ncc(xctx, small_scene):
    images = [g.astype(np.float32) for g in small_scene.gray]
    cams = [h.S.camera_struct(small_scene, i) for i in range(small_scene.n)]
    p = D.default_params()
    px, py, src, planes = _random_queries(small_scene, 5000, np.random.default_rng(21), near_gt=False)
    g = xctx.ncc_eval(images, cams, p, px, py, src, planes)
    o = O.ncc_strong(images, cams, p, px, py, src, planes, fp64=False)
    assert np.array_equal(g.astype(np.float64), o)


def test_exact_first_init(xctx, small_scene):
    for ref in (0, 2):
        images, cams, _ = h.view_inputs(small_scene, ref)
        p = h.first_init_params(small_scene, len(images))
        _same(xctx.pm_run(images, cams, p, seed=1234 + ref), O.pm_run(images, cams, p, seed=1234 + ref),
              f"first-init {ref}")


@pytest.fixture(scope="module")
def weak_scene():
    return h.S.make_scene("small_weak", seed=2)


def _level1(scene, ref, seed):
    images, cams, srcs = h.view_inputs(scene, ref)
    p0 = h.first_init_params(scene, len(images))
    o0 = O.pm_run(images, cams, p0, seed=seed)
    state, weak = h.post_process(o0["plane"], o0["weak"], p0.depth_min, p0.depth_max)
    edge, low, label = h.synthetic_edges(scene.gray[ref])
    return images, cams, srcs, state, weak, np.ascontiguousarray(o0["views"]), edge, low, label


def test_exact_weak_path(xctx, weak_scene):
    images, cams, srcs, state, weak, views, edge, low, label = _level1(weak_scene, 1, seed=21)
    p = h.refine_params(weak_scene, len(images), level=1, state=D.REFINE_INIT, geom=False)
    kw = dict(plane_in=state, views_in=views, weak_in=weak, edge=edge, edge_low=low, label=label, seed=77)
    _same(xctx.pm_run(images, cams, p, **kw), O.pm_run(images, cams, p, **kw), "refine-init")


def test_exact_geom_path(xctx, weak_scene):
    images, cams, srcs, state, weak, views, edge, low, label = _level1(weak_scene, 2, seed=22)
    depths = [np.ascontiguousarray(weak_scene.depth[i].astype(np.float32)) for i in [2] + list(srcs)]
    p = h.refine_params(weak_scene, len(images), level=1, state=D.REFINE_ITER, geom=True, j=0)
    kw = dict(plane_in=state, views_in=views, weak_in=weak, edge=edge, edge_low=low, label=label, depths=depths,
              seed=78)
    _same(xctx.pm_run(images, cams, p, **kw), O.pm_run(images, cams, p, **kw), "refine-iter geom")


@pytest.mark.parametrize("staging", [D.STAGE_FP16, D.STAGE_BF16])
def test_exact_staging_on_8bit_images(xctx, small_scene, staging):
    images, cams, _ = h.view_inputs(small_scene, 1)
    p = h.first_init_params(small_scene, len(images))
    ref = xctx.pm_run(images, cams, p, seed=31)
    xctx.set_options(staging=staging)
    try:
        got = xctx.pm_run(images, cams, p, seed=31)
    finally:
        xctx.set_options()
    _same(got, ref, f"staging {staging}")
