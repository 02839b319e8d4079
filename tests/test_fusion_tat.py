"""CPU tests of the TAT fusion restatement (RunFusion_TAT_Intermediate, DPE.cpp:1550-1718;
RunFusion_TAT_advanced, DPE.cpp:1720-1867).

The C oracle is checked against a second, independent restatement written here in numpy float32
with the sequential pixel loop spelled out, on the tiny scene with depth holes, a block mask and a
band of a source view without depth, so that sources are skipped and their differences carried
from pixel to pixel as in the reference.  The carry itself is shown to change the result.
"""
import math

import numpy as np
import pytest

import dpe_b200 as D
import helpers as h
import oracle_py as O

F = np.float32
FLT_MAX = float(np.finfo(np.float32).max)


def tat_views(scene, noise=2e-4, seed=0, dead_band=True, block=True):
    """Noisy ground-truth depth maps with 5% holes; view 1 has no depth in a vertical band and view
    2 a block mask over its left third."""
    rng = np.random.default_rng(seed)
    views = []
    for v in range(scene.n):
        d = scene.depth[v].astype(np.float32).copy()
        if noise:
            d *= (1 + rng.normal(0, noise, d.shape)).astype(np.float32)
        d[rng.random(d.shape) < 0.05] = 0.0
        W = d.shape[1]
        if dead_band and v == 1:
            d[:, W // 3: W // 2] = 0.0
        blk = None
        if block and v == 2:
            blk = np.full(d.shape, 255, np.uint8)
            blk[:, : W // 3] = 0
        views.append(dict(depth=np.ascontiguousarray(d), normal=np.ascontiguousarray(scene.normal[v].astype(np.float32)),
                          bgr=np.ascontiguousarray(scene.bgr[v]), camera=h.S.camera_struct(scene, v),
                          src=list(scene.pairs[v]), block=blk))
    return views


# ------------------------------------------------------------------ the numpy restatement
def _world(x, y, depth, cam):
    """Get3DPointonWorld (DPE.cpp:1337-1359) in float32."""
    K, R, t = cam["K"].reshape(-1).astype(F), cam["R"].reshape(-1).astype(F), cam["t"].reshape(-1).astype(F)
    px = depth * (x - K[2]) / K[0]
    py = depth * (y - K[5]) / K[4]
    pz = depth
    tx = R[0] * px + R[3] * py + R[6] * pz
    ty = R[1] * px + R[4] * py + R[7] * pz
    tz = R[2] * px + R[5] * py + R[8] * pz
    cx = -(R[0] * t[0] + R[3] * t[1] + R[6] * t[2])
    cy = -(R[1] * t[0] + R[4] * t[1] + R[7] * t[2])
    cz = -(R[2] * t[0] + R[5] * t[1] + R[8] * t[2])
    return tx + cx, ty + cy, tz + cz


def _project(X, cam):
    """ProjectCamera (DPE.cpp:1361-1371) in float32."""
    K, R, t = cam["K"].reshape(-1).astype(F), cam["R"].reshape(-1).astype(F), cam["t"].reshape(-1).astype(F)
    tx = R[0] * X[0] + R[1] * X[1] + R[2] * X[2] + t[0]
    ty = R[3] * X[0] + R[4] * X[1] + R[5] * X[2] + t[1]
    tz = R[6] * X[0] + R[7] * X[1] + R[8] * X[2] + t[2]
    d = K[6] * tx + K[7] * ty + K[8] * tz
    return (K[0] * tx + K[1] * ty + K[2] * tz) / d, (K[3] * tx + K[4] * ty + K[5] * tz) / d, d


def _trunc(a):
    a = np.asarray(a, np.float64)
    return np.where(np.isnan(a), 0, np.clip(np.trunc(a), -2.0**31, 2.0**31 - 1)).astype(np.int64)


def _acosf(x):
    out = np.zeros(x.shape, F)
    for i, v in np.ndenumerate(x):
        out[i] = F(math.acos(float(v))) if -1.0 <= float(v) <= 1.0 else F(0.0)  # NaN -> 0 (DPE.cpp:1380)
    return out


def tat_numpy(views, variant, carry=True):
    """The reference loop, float arithmetic.  carry=False resets each source's differences at every
    pixel instead (not the reference behaviour; used to show that the carry matters)."""
    inter = variant == D.TAT_INTERMEDIATE
    depth_base = F(1.0) / F(3500.0) if inter else F(1.0) / F(3000.0)
    masks = [np.zeros(v["depth"].shape, np.uint8) for v in views]
    pts = []
    for i, V in enumerate(views):
        H, W = V["depth"].shape
        rr, cc = np.mgrid[0:H, 0:W]
        X = _world(cc.astype(F), rr.astype(F), V["depth"], V["camera"])
        ns = len(V["src"])
        tested, vals = [], []
        for s in V["src"]:
            S = views[s]
            u, v, _ = _project(X, S["camera"])
            sr, sc = _trunc(v + F(0.5)), _trunc(u + F(0.5))
            inb = (sc >= 0) & (sc < S["depth"].shape[1]) & (sr >= 0) & (sr < S["depth"].shape[0])
            sr_c, sc_c = np.where(inb, sr, 0), np.where(inb, sc, 0)
            sd = S["depth"][sr_c, sc_c]
            ok = inb & (masks[s][sr_c, sc_c] != 1) & ~(sd <= 0.0)
            T = _world(sc_c.astype(F), sr_c.astype(F), sd, S["camera"])
            tu, tv, pd = _project(T, V["camera"])
            ex, ey = cc.astype(F) - tu, rr.astype(F) - tv
            dist = np.sqrt(ex.astype(np.float64) * ex.astype(np.float64) + ey.astype(np.float64) * ey.astype(np.float64)).astype(F)
            rel = np.abs(pd - V["depth"]) / V["depth"]
            rn, sn = V["normal"], S["normal"][sr_c, sc_c]
            dot = rn[..., 0] * sn[..., 0] + rn[..., 1] * sn[..., 1] + rn[..., 2] * sn[..., 2]
            ang = _acosf(np.where(ok, dot, F(1.0)))
            tested.append(ok)
            vals.append((dist, rel, ang, sr_c, sc_c))
        diff = [[FLT_MAX, FLT_MAX, FLT_MAX, 0, 0] for _ in range(ns)]
        for r in range(H):
            for c in range(W):
                if V.get("block") is not None and V["block"][r, c] < 128:
                    continue
                if V["depth"][r, c] <= 0.0:
                    continue
                if not carry:
                    diff = [[FLT_MAX, FLT_MAX, FLT_MAX, 0, 0] for _ in range(ns)]
                for j in range(ns):
                    if tested[j][r, c]:
                        diff[j] = [float(vals[j][q][r, c]) if q < 3 else int(vals[j][q][r, c]) for q in range(5)]
                for k in range(2, ns + 1):
                    bd, bz = F(k) * F(0.25), F(k) * depth_base
                    ba = F(k) * F(0.05235987755982988) + F(0.06981317007977318)
                    use = [F(d[0]) < bd and F(d[1]) < bz and (not inter or F(d[2]) < ba) for d in diff]
                    n = sum(use)
                    if n < k:
                        continue
                    col = V["bgr"][r, c].astype(F)
                    if inter:
                        for j in range(ns):
                            if use[j]:
                                col = col + views[V["src"][j]]["bgr"][diff[j][3], diff[j][4]].astype(F)
                        col = col / F(n + 1)
                    pts.append((i, r * W + c, n, X[0][r, c], X[1][r, c], X[2][r, c], *[int(x) for x in col]))
                    masks[i][r, c] = 1
                    break
    return pts


def _as_points(res):
    return [(int(o[0]), int(o[1]), int(n), F(x[0]), F(x[1]), F(x[2]), int(b[0]), int(b[1]), int(b[2]))
            for o, n, x, b in zip(res["origin"], res["num_consistent"], res["xyz"], res["bgr"])]


@pytest.fixture(scope="module")
def views(tiny_scene):
    return tat_views(tiny_scene, seed=11)


@pytest.mark.parametrize("variant", [D.TAT_INTERMEDIATE, D.TAT_ADVANCED])
def test_tat_oracle_matches_numpy_restatement(views, variant):
    o = O.fuse_tat(views, variant, D.FUSE_FLOAT)
    ref = tat_numpy(views, variant)
    assert o["count"] == len(ref) > 100
    assert _as_points(o) == ref


def test_tat_carry_changes_result(views):
    """The carried differences are not a corner case on this input: resetting them per pixel
    changes the fused set, and the oracle follows the carrying loop."""
    carried = tat_numpy(views, D.TAT_ADVANCED, carry=True)
    reset = tat_numpy(views, D.TAT_ADVANCED, carry=False)
    assert carried != reset
    assert _as_points(O.fuse_tat(views, D.TAT_ADVANCED, D.FUSE_FLOAT)) == carried


def test_tat_properties(small_scene):
    vs = tat_views(small_scene, seed=12)
    for variant in (D.TAT_INTERMEDIATE, D.TAT_ADVANCED):
        a = O.fuse_tat(vs, variant, D.FUSE_FP64)
        b = O.fuse_tat(vs, variant, D.FUSE_FLOAT)
        assert a["count"] > 0.2 * sum(v["depth"].size for v in vs) / len(vs)
        assert abs(a["count"] - b["count"]) <= 0.01 * a["count"]
        key = a["origin"][:, 0].astype(np.int64) * 10**9 + a["origin"][:, 1]
        assert np.all(np.diff(key) > 0)  # view order, raster order, each pixel at most once
        assert np.all(a["num_consistent"] >= 2)
        # no point from a blocked pixel or a pixel without depth
        for (vi, p) in a["origin"]:
            assert vs[vi]["depth"].reshape(-1)[p] > 0
            if vs[vi]["block"] is not None:
                assert vs[vi]["block"].reshape(-1)[p] >= 128
        if variant == D.TAT_ADVANCED:  # colour of the reference pixel only
            ref_col = np.stack([vs[vi]["bgr"].reshape(-1, 3)[p] for vi, p in a["origin"]])
            assert np.array_equal(a["bgr"], ref_col)
    # the stricter intermediate rule (angle bound, tighter depth) keeps no more points
    assert O.fuse_tat(vs, D.TAT_INTERMEDIATE)["count"] <= O.fuse_tat(vs, D.TAT_ADVANCED)["count"]


def test_tat_needs_two_sources(tiny_scene):
    vs = tat_views(tiny_scene, seed=13)
    for v in vs:
        v["src"] = v["src"][:1]
    assert O.fuse_tat(vs, D.TAT_ADVANCED)["count"] == 0


def test_tat_capacity(tiny_scene):
    vs = tat_views(tiny_scene, seed=14)
    r = O.fuse_tat(vs, D.TAT_ADVANCED, capacity=7)
    assert r["status"] == D.ERR_CAPACITY and r["count"] > 7 and len(r["xyz"]) == 7
