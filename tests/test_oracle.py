"""CPU tests of the oracle itself: known answers, float-vs-FP64 agreement, determinism."""
import numpy as np
import pytest

import dpe_b200 as D
import helpers as h
import oracle_py as O


# Known-answer vectors of Philox4x32-10 published with Random123 (Salmon et al., SC'11).
PHILOX_KAT = [
    ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
    ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
    ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
     [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
]


@pytest.mark.parametrize("ctr,key,expect", PHILOX_KAT)
def test_philox_known_answers(ctr, key, expect):
    assert list(O.philox(ctr, key)) == expect


def _random_queries(scene, n, rng, near_gt=True):
    H, W = scene.spec.height, scene.spec.width
    px = rng.integers(0, W, n)
    py = rng.integers(0, H, n)
    src = rng.integers(1, scene.n, n)
    cam = h.S.camera_struct(scene, 0)
    K = cam["K"].reshape(3, 3)
    planes = np.zeros((n, 4), np.float32)
    for k in range(n):
        d = scene.depth[0, py[k], px[k]] * (1 + (rng.normal(0, 0.01) if near_gt else rng.uniform(-0.3, 0.3)))
        nw = scene.normal[0, py[k], px[k]]
        R = scene.R[0]
        nr = R @ nw  # world -> reference camera
        nr = nr + rng.normal(0, 0.05, 3)
        nr /= np.linalg.norm(nr)
        X = np.array([d * (px[k] - K[0, 2]) / K[0, 0], d * (py[k] - K[1, 2]) / K[1, 1], d])
        if nr @ X > 0:
            nr = -nr
        planes[k, :3] = nr
        planes[k, 3] = -(nr @ X)
    return px, py, src, planes


def test_oracle_ncc_float_matches_fp64(small_scene):
    """The float restatement of the strong NCC agrees with its FP64 evaluation within 1e-4."""
    rng = np.random.default_rng(7)
    images = [g.astype(np.float32) for g in small_scene.gray]
    cams = [h.S.camera_struct(small_scene, i) for i in range(small_scene.n)]
    p = D.default_params()
    px, py, src, planes = _random_queries(small_scene, 4000, rng)
    f32 = O.ncc_strong(images, cams, p, px, py, src, planes, fp64=False)
    f64 = O.ncc_strong(images, cams, p, px, py, src, planes, fp64=True)
    assert np.all((f64 >= 0) & (f64 <= 2))
    assert np.max(np.abs(f32 - f64)) <= 1e-4
    # costs near the true surface are low: the NCC responds to the geometry
    assert np.median(f64[f64 < 2]) < 0.5


def test_oracle_pm_run_deterministic_and_accurate(small_scene):
    images, cams, _ = h.view_inputs(small_scene, 1)
    p = h.first_init_params(small_scene, len(images))
    a = O.pm_run(images, cams, p, seed=99)
    b = O.pm_run(images, cams, p, seed=99)
    for k in ("plane", "weak", "views", "costs"):
        assert np.array_equal(a[k], b[k], equal_nan=True), k
    d = a["plane"][..., 3]
    rel = np.abs(d - small_scene.depth[1]) / small_scene.depth[1]
    assert np.median(rel) < 0.005
    assert (rel < 0.01).mean() > 0.85
    # world normals are unit length
    nn = np.linalg.norm(a["plane"][..., :3], axis=-1)
    assert np.allclose(nn, 1.0, atol=1e-4)


def test_oracle_seed_changes_result(tiny_scene):
    images, cams, _ = h.view_inputs(tiny_scene, 0)
    p = h.first_init_params(tiny_scene, len(images), iters=1)
    a = O.pm_run(images, cams, p, seed=1)
    b = O.pm_run(images, cams, p, seed=2)
    assert not np.array_equal(a["plane"], b["plane"])


def _gt_fusion_views(scene, noise=0.0, seed=0):
    rng = np.random.default_rng(seed)
    views = []
    for v in range(scene.n):
        d = scene.depth[v].astype(np.float32).copy()
        if noise:
            d *= (1 + rng.normal(0, noise, d.shape)).astype(np.float32)
        d[rng.random(d.shape) < 0.05] = 0.0  # holes
        weak = np.where(rng.random(d.shape) < 0.3, D.WEAK, D.STRONG).astype(np.uint8)
        views.append(dict(depth=np.ascontiguousarray(d), normal=np.ascontiguousarray(scene.normal[v].astype(np.float32)),
                          weak=weak, bgr=np.ascontiguousarray(scene.bgr[v]), camera=h.S.camera_struct(scene, v),
                          src=scene.pairs[v]))
    return views


def test_oracle_fusion_modes_agree(small_scene):
    views = _gt_fusion_views(small_scene, noise=0.002, seed=3)
    a = O.fuse(views, D.FUSE_FP64)
    b = O.fuse(views, D.FUSE_FLOAT)
    assert a["count"] > 0.3 * sum(v["depth"].size for v in views) / len(views)
    assert abs(a["count"] - b["count"]) <= 0.01 * a["count"]
    # points come out in view order, then raster order
    o = a["origin"]
    key = o[:, 0].astype(np.int64) * 10**9 + o[:, 1]
    assert np.all(np.diff(key) > 0)
    assert np.all(a["num_consistent"] >= 1)


def test_oracle_fusion_capacity(small_scene):
    views = _gt_fusion_views(small_scene, seed=4)
    a = O.fuse(views, D.FUSE_FP64, capacity=10)
    assert a["status"] == D.ERR_CAPACITY and a["count"] > 10
