"""GPU parity tests: the sm_100a kernels through the C-ABI against the CPU oracle.

Bars (north star): per-(pixel, hypothesis) NCC within 1e-4 absolute of the FP64 oracle; depth maps
from identical seeded hypotheses within 0.1% relative depth on >= 99.5% of pixels; fusion counts,
point order and indices bit-exact against the oracle's FP64 fusion given identical depth inputs.
"""
import numpy as np
import pytest

import dpe_b200 as D
import helpers as h
import oracle_py as O
from test_oracle import _gt_fusion_views, _random_queries

pytestmark = pytest.mark.gpu

NCC_TOL = 1e-4          # absolute, against FP64
DEPTH_REL_TOL = 1e-3    # 0.1 % relative depth
DEPTH_FRACTION = 0.995  # of pixels


def test_ncc_matches_fp64_oracle(ctx, small_scene):
    rng = np.random.default_rng(11)
    images = [g.astype(np.float32) for g in small_scene.gray]
    cams = [h.S.camera_struct(small_scene, i) for i in range(small_scene.n)]
    p = D.default_params()
    px, py, src, planes = _random_queries(small_scene, 10000, rng)
    gpu = ctx.ncc_eval(images, cams, p, px, py, src, planes)
    f64 = O.ncc_strong(images, cams, p, px, py, src, planes, fp64=True)
    err = np.abs(gpu.astype(np.float64) - f64)
    print(f"NCC max |gpu - fp64| = {err.max():.3e}, mean {err.mean():.3e}")
    assert err.max() <= NCC_TOL
    # random (far from the surface) hypotheses as well
    px, py, src, planes = _random_queries(small_scene, 10000, rng, near_gt=False)
    gpu = ctx.ncc_eval(images, cams, p, px, py, src, planes)
    f64 = O.ncc_strong(images, cams, p, px, py, src, planes, fp64=True)
    assert np.abs(gpu.astype(np.float64) - f64).max() <= NCC_TOL


def _compare_calls(g, o, label):
    dg, do = g["plane"][..., 3], o["plane"][..., 3]
    agree = h.rel_depth_agreement(dg, do, DEPTH_REL_TOL)
    weak_agree = float((g["weak"] == o["weak"]).mean())
    views_agree = float((g["views"] == o["views"]).mean())
    print(f"{label}: depth agreement {agree:.5f}, weak agreement {weak_agree:.5f}, views agreement {views_agree:.5f}")
    return agree, weak_agree


def test_pm_first_init_matches_oracle(ctx, small_scene):
    for ref in (0, 2):
        images, cams, _ = h.view_inputs(small_scene, ref)
        p = h.first_init_params(small_scene, len(images))
        g = ctx.pm_run(images, cams, p, seed=1234 + ref)
        o = O.pm_run(images, cams, p, seed=1234 + ref)
        agree, weak_agree = _compare_calls(g, o, f"first-init view {ref}")
        assert agree >= DEPTH_FRACTION
        assert weak_agree >= 0.99


def test_pm_repeatable(ctx, small_scene):
    images, cams, _ = h.view_inputs(small_scene, 1)
    p = h.first_init_params(small_scene, len(images))
    a = ctx.pm_run(images, cams, p, seed=5)
    b = ctx.pm_run(images, cams, p, seed=5)
    for k in ("plane", "weak", "views"):
        assert np.array_equal(a[k], b[k]), k


@pytest.fixture(scope="module")
def weak_scene():
    return h.S.make_scene("small_weak", seed=2)


def _level1_inputs(scene, ref, seed):
    """A REFINE_INIT input state from the oracle's FIRST_INIT call, plus edge/label maps."""
    images, cams, srcs = h.view_inputs(scene, ref)
    p0 = h.first_init_params(scene, len(images))
    o0 = O.pm_run(images, cams, p0, seed=seed)
    state, weak = h.post_process(o0["plane"], o0["weak"], p0.depth_min, p0.depth_max)
    edge, low, label = h.synthetic_edges(scene.gray[ref])
    return images, cams, srcs, state, weak, np.ascontiguousarray(o0["views"]), edge, low, label


def test_pm_refine_weak_path_matches_oracle(ctx, weak_scene):
    images, cams, srcs, state, weak, views, edge, low, label = _level1_inputs(weak_scene, 1, seed=21)
    assert (weak == D.WEAK).mean() > 0.02  # the weak-texture path is exercised
    p = h.refine_params(weak_scene, len(images), level=1, state=D.REFINE_INIT, geom=False)
    kw = dict(plane_in=state, views_in=views, weak_in=weak, edge=edge, edge_low=low, label=label, seed=77)
    g = ctx.pm_run(images, cams, p, **kw)
    o = O.pm_run(images, cams, p, **kw)
    agree, weak_agree = _compare_calls(g, o, "refine-init (APD, edge, label)")
    assert agree >= DEPTH_FRACTION
    assert weak_agree >= 0.99


def test_pm_refine_geom_matches_oracle(ctx, weak_scene):
    images, cams, srcs, state, weak, views, edge, low, label = _level1_inputs(weak_scene, 2, seed=22)
    ids = [2] + list(srcs)
    depths = [np.ascontiguousarray(weak_scene.depth[i].astype(np.float32)) for i in ids]
    p = h.refine_params(weak_scene, len(images), level=1, state=D.REFINE_ITER, geom=True, j=0)
    kw = dict(plane_in=state, views_in=views, weak_in=weak, edge=edge, edge_low=low, label=label, depths=depths, seed=78)
    g = ctx.pm_run(images, cams, p, **kw)
    o = O.pm_run(images, cams, p, **kw)
    agree, weak_agree = _compare_calls(g, o, "refine-iter (geom)")
    # With the geometric term on a near-textureless scene many hypotheses tie, and any change of
    # rounding can change which of the equally good ones wins (built with FMA contraction, the
    # kernels agreed with the oracle on 97.5 % here).  The default build no longer contracts; the
    # tap reciprocal is its only difference from the oracle, and it is held to the north-star bar
    # of 99.5 % of all pixels, besides the statistical bars on well-matched pixels and accuracy.
    dg, do = g["plane"][..., 3], o["plane"][..., 3]
    conf = np.isfinite(o["costs"]) & (o["costs"] < 0.3) & (o["weak"] == D.STRONG) & (g["weak"] == D.STRONG)
    conf_agree = h.rel_depth_agreement(dg[conf], do[conf], DEPTH_REL_TOL)
    gt = weak_scene.depth[2]
    acc_g = float((np.abs(dg - gt) / gt < 0.01).mean())
    acc_o = float((np.abs(do - gt) / gt < 0.01).mean())
    print(f"refine-iter (geom): well-matched pixels {conf.mean():.3f} agree {conf_agree:.5f}; within 1% of GT "
          f"gpu {acc_g:.4f} oracle {acc_o:.4f}")
    assert conf_agree >= 0.98
    assert abs(acc_g - acc_o) <= 0.01
    assert agree >= DEPTH_FRACTION
    assert weak_agree >= 0.99


def test_fusion_bit_exact_fp64(ctx, small_scene):
    views = _gt_fusion_views(small_scene, noise=0.002, seed=5)
    g = ctx.fuse(views, D.FUSE_FP64)
    o = O.fuse(views, D.FUSE_FP64)
    print(f"fusion points gpu {g['count']} oracle {o['count']}")
    assert g["count"] == o["count"]
    assert np.array_equal(g["origin"], o["origin"])
    assert np.array_equal(g["num_consistent"], o["num_consistent"])
    assert np.array_equal(g["xyz"], o["xyz"])
    assert np.array_equal(g["bgr"], o["bgr"])


def test_fusion_float_mode_close(ctx, small_scene):
    views = _gt_fusion_views(small_scene, noise=0.002, seed=6)
    g = ctx.fuse(views, D.FUSE_FLOAT)
    o = O.fuse(views, D.FUSE_FLOAT)
    assert abs(g["count"] - o["count"]) <= max(2, 1e-4 * o["count"])


def test_fusion_capacity_error(ctx, small_scene):
    views = _gt_fusion_views(small_scene, seed=7)
    with pytest.raises(D.DPEError) as e:
        ctx.fuse(views, D.FUSE_FP64, capacity=5)
    assert e.value.status == D.ERR_CAPACITY


def test_invalid_problems_rejected(ctx, small_scene):
    images, cams, _ = h.view_inputs(small_scene, 0)
    p = h.first_init_params(small_scene, len(images))
    with pytest.raises(D.DPEError) as e:
        ctx.pm_run(images[:1], cams[:1], p)
    assert e.value.status == D.ERR_INVALID_ARGUMENT
    p2 = h.first_init_params(small_scene, len(images))
    p2.state = D.REFINE_INIT  # needs plane_in
    with pytest.raises(D.DPEError) as e:
        ctx.pm_run(images, cams, p2)
    assert e.value.status == D.ERR_INVALID_ARGUMENT
    p3 = h.first_init_params(small_scene, len(images))
    p3.strong_radius = 9  # window wider than the 6x6 tap layout
    with pytest.raises(D.DPEError) as e:
        ctx.pm_run(images, cams, p3)
    assert e.value.status == D.ERR_INVALID_ARGUMENT
