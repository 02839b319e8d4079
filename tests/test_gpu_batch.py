"""dpe_pm_run_batch: problems of different sizes in one kernel sequence give exactly the results
of separate dpe_pm_run calls (same kernels, same per-pixel arithmetic; only the mapping of blocks
to problems differs)."""
import numpy as np
import pytest

import dpe_b200 as D
import helpers as h

pytestmark = pytest.mark.gpu


def _same(a, b):
    for k in ("plane", "weak", "views", "costs"):
        assert np.array_equal(a[k], b[k], equal_nan=True), k


def test_batch_first_init_mixed_sizes(ctx, small_scene, tiny_scene):
    import cv2

    calls = []
    for sc, ref in ((small_scene, 0), (small_scene, 2), (tiny_scene, 1)):
        images, cams, _ = h.view_inputs(sc, ref)
        calls.append(dict(images=images, cameras=cams, params=h.first_init_params(sc, len(images)), seed=100 + ref))
    # a half-size copy of a view: a third distinct grid shape
    images, cams, srcs = h.view_inputs(small_scene, 1)
    H, W = images[0].shape
    half = [np.ascontiguousarray(cv2.resize(im, (W // 2, H // 2), interpolation=cv2.INTER_LINEAR)) for im in images]
    cams2 = [h.S.camera_struct(small_scene, i, W // 2, H // 2) for i in [1] + list(srcs)]
    calls.append(dict(images=half, cameras=cams2, params=h.first_init_params(small_scene, len(half)), seed=7))
    batch = ctx.pm_run_batch(calls)
    for c, got in zip(calls, batch):
        kw = {k: v for k, v in c.items() if k not in ("images", "cameras", "params")}
        _same(got, ctx.pm_run(c["images"], c["cameras"], c["params"], **kw))


def test_batch_weak_texture_path(ctx):
    sc = h.S.make_scene("small_weak", seed=2)
    calls = []
    for ref in (1, 2):
        images, cams, _ = h.view_inputs(sc, ref)
        p0 = h.first_init_params(sc, len(images))
        o0 = ctx.pm_run(images, cams, p0, seed=40 + ref)
        state, weak = h.post_process(o0["plane"], o0["weak"], p0.depth_min, p0.depth_max)
        edge, low, label = h.synthetic_edges(sc.gray[ref])
        p = h.refine_params(sc, len(images), level=1, state=D.REFINE_INIT, geom=False)
        calls.append(dict(images=images, cameras=cams, params=p, plane_in=state, views_in=np.ascontiguousarray(o0["views"]),
                          weak_in=weak, edge=edge, edge_low=low, label=label, seed=50 + ref))
    assert all((c["weak_in"] == D.WEAK).mean() > 0.02 for c in calls)
    batch = ctx.pm_run_batch(calls)
    for c, got in zip(calls, batch):
        kw = {k: v for k, v in c.items() if k not in ("images", "cameras", "params")}
        _same(got, ctx.pm_run(c["images"], c["cameras"], c["params"], **kw))


def test_batch_rejects_mixed_schedules(ctx, small_scene):
    images, cams, _ = h.view_inputs(small_scene, 0)
    p0 = h.first_init_params(small_scene, len(images))
    p1 = h.first_init_params(small_scene, len(images))
    p1.max_iterations = 2
    with pytest.raises(D.DPEError) as e:
        ctx.pm_run_batch([dict(images=images, cameras=cams, params=p0), dict(images=images, cameras=cams, params=p1)])
    assert e.value.status == D.ERR_INVALID_ARGUMENT
