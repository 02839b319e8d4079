"""The device-resident schedule (dpe_scene_run) against the same schedule driven from the host one
per-view call at a time (dpe_pm_run on host buffers, result assembly and rescale in numpy,
restating main.cpp:385-457 / ProcessProblem / RescaleMatToTargetSize).  Same kernels and seeds on
both sides, so the final maps and the fused points must be identical."""
import numpy as np
import pytest

import dpe_b200 as D
import edges as E
import helpers as h

pytestmark = pytest.mark.gpu

MASK = (1 << 64) - 1


def mix64(z):
    z = (z + 0x9E3779B97F4A7C15) & MASK
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
    return z ^ (z >> 31)


def rescale_nearest(src, h_, w_):
    """RescaleMatToTargetSize (DPE.cpp:1313-1335)."""
    sh, sw = src.shape[:2]
    sy = np.float32(h_) / np.float32(sh)
    sx = np.float32(w_) / np.float32(sw)
    rows = (np.arange(h_, dtype=np.float32) / sy).astype(np.int32)
    cols = (np.arange(w_, dtype=np.float32) / sx).astype(np.int32)
    return np.ascontiguousarray(src[rows][:, cols])


def host_schedule(ctx, sc, edges_l, labels_l, L, rc, iters, seed):
    import cv2

    V, H, W = sc.gray.shape
    sizes = [(int(round(W * np.float32(1.0 / (1 << (L - 1 - l))))), int(round(H * np.float32(1.0 / (1 << (L - 1 - l))))))
             for l in range(L)]
    state = [None] * V
    for l in range(L):
        w, hh = sizes[l]
        scale = 1 << (L - 1 - l)
        imgs = [sc.gray[v].astype(np.float32) if scale == 1 else
                np.ascontiguousarray(cv2.resize(sc.gray[v].astype(np.float32), (w, hh), interpolation=cv2.INTER_LINEAR))
                for v in range(V)]
        if l > 0:
            state = [{k: rescale_nearest(st[k], hh, w) for k in ("plane", "weak", "views")} for st in state]
        for call in range(rc + 1):
            for v in range(V):
                ids = [v] + sc.pairs[v]
                cams = [h.S.camera_struct(sc, i, w, hh) for i in ids]
                p = D.default_params()
                p.num_images = len(ids)
                p.max_scale_size = 1 << (L - 1)
                p.scale_size = scale
                p.max_iterations = iters
                p.depth_min = np.float32(sc.spec.depth_min) * np.float32(0.6)
                p.depth_max = np.float32(sc.spec.depth_max) * np.float32(1.2)
                if call == 0:
                    if l == 0:
                        p.state, p.use_APD, p.use_edge = D.FIRST_INIT, 0, 0
                    else:
                        p.state, p.use_APD, p.use_edge = D.REFINE_INIT, 1, 1
                        p.ransac_threshold = np.float32(0.01 - l * 0.00125)
                        p.rotate_time = min(1 << l, 4)
                    p.geom_consistency, p.weak_peak_radius = 0, 6
                else:
                    p.state = D.REFINE_ITER
                    p.use_APD = p.use_edge = 1 if l > 0 else 0
                    p.ransac_threshold = np.float32(0.01 - l * 0.00125)
                    p.rotate_time = min(1 << l, 4)
                    p.geom_consistency = 1
                    p.weak_peak_radius = max(4 - 2 * (call - 1), 2)
                kw = dict(edge=edges_l[v][l], edge_low=edges_l[v][0], label=labels_l[v][l],
                          seed=mix64(seed ^ (l << 48) ^ (call << 40) ^ v))
                if p.state != D.FIRST_INIT:
                    kw.update(plane_in=state[v]["plane"], views_in=state[v]["views"])
                kw["weak_in"] = state[v]["weak"] if state[v] is not None else np.full((hh, w), D.STRONG, np.uint8)
                if p.geom_consistency:
                    kw["depths"] = [np.ascontiguousarray(state[i]["plane"][..., 3]) for i in ids]
                o = ctx.pm_run([imgs[i] for i in ids], cams, p, **kw)
                plane, weak = h.post_process(o["plane"], o["weak"], p.depth_min, p.depth_max)
                state[v] = dict(plane=plane, weak=weak, views=np.ascontiguousarray(o["views"]))
    return state


def test_scene_schedule_matches_host_driven_calls(ctx):
    sc = h.S.make_scene("small_weak", seed=3)
    V = sc.n
    L, rc, iters, seed = 2, 1, 2, 99
    edges_l, labels_l = [], []
    for v in range(V):
        ev, lv = zip(*[E.level_inputs(sc.gray[v], 1 << (L - 1 - l)) for l in range(L)])
        edges_l.append([np.ascontiguousarray(e) for e in ev])
        labels_l.append([np.ascontiguousarray(x) for x in lv])
    cams = [h.S.camera_struct(sc, v) for v in range(V)]
    res = ctx.scene_run(list(sc.gray), list(sc.bgr), cams, sc.pairs, edges_l, labels_l, num_levels=L,
                        refine_calls=rc, max_iterations=iters, fuse_mode=D.FUSE_FP64, seed=seed)
    assert res["num_levels"] == L and res["calls"] == L * (rc + 1) * V
    ref = host_schedule(ctx, sc, edges_l, labels_l, L, rc, iters, seed)
    for v in range(V):
        assert np.array_equal(res["depth"][v], ref[v]["plane"][..., 3]), v
        assert np.array_equal(res["normal"][v], ref[v]["plane"][..., :3]), v
        assert np.array_equal(res["weak"][v], ref[v]["weak"]), v
        assert np.array_equal(res["views"][v], ref[v]["views"]), v
    views = [dict(depth=np.ascontiguousarray(ref[v]["plane"][..., 3]), normal=np.ascontiguousarray(ref[v]["plane"][..., :3]),
                  weak=ref[v]["weak"], bgr=np.ascontiguousarray(sc.bgr[v]), camera=cams[v], src=sc.pairs[v])
             for v in range(V)]
    f = ctx.fuse(views, D.FUSE_FP64)
    assert res["points"] == f["count"] and np.array_equal(res["xyz"], f["xyz"])
    rel = np.abs(res["depth"][1] - sc.depth[1]) / sc.depth[1]
    print(f"scene schedule: {res['points']} points, view 1 within 1% of GT: {(rel < 0.01).mean():.3f}")
    assert (rel < 0.01).mean() > 0.5


def test_scene_batched_views(ctx):
    """batch_views=1: every call runs all views in one dpe_pm_run_batch, each reading the previous
    call's depths instead of its predecessors' (not the reference's order, so not bit-comparable);
    the result is as accurate against the ground truth as the sequential schedule's, within 3
    points, and fuses a comparable cloud."""
    sc = h.S.make_scene("small_weak", seed=3)
    V = sc.n
    L = 2
    edges_l, labels_l = [], []
    for v in range(V):
        ev, lv = zip(*[E.level_inputs(sc.gray[v], 1 << (L - 1 - l)) for l in range(L)])
        edges_l.append([np.ascontiguousarray(e) for e in ev])
        labels_l.append([np.ascontiguousarray(x) for x in lv])
    cams = [h.S.camera_struct(sc, v) for v in range(V)]
    kw = dict(num_levels=L, refine_calls=1, max_iterations=2, fuse_mode=D.FUSE_FP64, seed=5)
    seq = ctx.scene_run(list(sc.gray), list(sc.bgr), cams, sc.pairs, edges_l, labels_l, **kw)
    bat = ctx.scene_run(list(sc.gray), list(sc.bgr), cams, sc.pairs, edges_l, labels_l, batch_views=True, **kw)
    acc = lambda r: float(np.mean([(np.abs(r["depth"][v] - sc.depth[v]) / sc.depth[v] < 0.01).mean() for v in range(V)]))
    print(f"batched views: within 1% of GT sequential {acc(seq):.4f} batched {acc(bat):.4f}; points "
          f"{seq['points']} / {bat['points']}")
    assert bat["calls"] == seq["calls"]
    assert acc(bat) >= acc(seq) - 0.03
    assert abs(bat["points"] - seq["points"]) <= 0.1 * seq["points"]
