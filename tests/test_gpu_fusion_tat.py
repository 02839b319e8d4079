"""GPU parity of the TAT fusion kernels (dpe_fuse_tat) against the CPU oracle.

Bars: in FP64 mode the points (count, view and pixel of origin, consistent-source count, xyz,
colour) are bit-exact; in float mode they are bit-exact up to comparisons that land on the float
acos's last bit (CUDA's acosf and the host's may differ there), at most 1e-4 of the points.
"""
import numpy as np
import pytest

import dpe_b200 as D
import helpers as h
import oracle_py as O
from test_fusion_tat import tat_views

pytestmark = pytest.mark.gpu

VARIANTS = [D.TAT_INTERMEDIATE, D.TAT_ADVANCED]


def _same(g, o):
    assert g["count"] == o["count"]
    for k in ("origin", "num_consistent", "xyz", "bgr"):
        assert np.array_equal(g[k], o[k]), k


@pytest.mark.parametrize("variant", VARIANTS)
def test_tat_bit_exact_fp64(ctx, small_scene, variant):
    vs = tat_views(small_scene, seed=21)
    g = ctx.fuse_tat(vs, variant, D.FUSE_FP64)
    o = O.fuse_tat(vs, variant, D.FUSE_FP64)
    print(f"TAT variant {variant}: {g['count']} points")
    assert g["count"] > 1000
    _same(g, o)


@pytest.mark.parametrize("variant", VARIANTS)
def test_tat_float_mode(ctx, small_scene, variant):
    vs = tat_views(small_scene, seed=22)
    g = ctx.fuse_tat(vs, variant, D.FUSE_FLOAT)
    o = O.fuse_tat(vs, variant, D.FUSE_FLOAT)
    kg = set(map(tuple, g["origin"]))
    ko = set(map(tuple, o["origin"]))
    assert len(kg ^ ko) <= max(2, 1e-4 * o["count"])
    if kg == ko:
        _same(g, o)


@pytest.mark.parametrize("variant", VARIANTS)
def test_tat_c2_small_bit_exact(ctx, variant):
    """The benchmark's 10-view layout at 400x300 with 9 sources per view."""
    sc = h.S.make_scene("c2_small", seed=3)
    vs = tat_views(sc, noise=1e-4, seed=23)
    g = ctx.fuse_tat(vs, variant, D.FUSE_FP64)
    o = O.fuse_tat(vs, variant, D.FUSE_FP64)
    print(f"c2_small TAT variant {variant}: {g['count']} points, {g['gpu_ms']:.2f} ms")
    _same(g, o)


def test_tat_device_memory(ctx, small_scene):
    import torch

    vs = tat_views(small_scene, seed=24)
    dv = []
    for v in vs:
        d = dict(v)
        for k in ("depth", "normal", "bgr", "block"):
            if v.get(k) is not None:
                d[k] = torch.from_numpy(v[k]).cuda()
        dv.append(d)
    g = ctx.fuse_tat(dv, D.TAT_INTERMEDIATE, D.FUSE_FP64, memory=D.MEM_DEVICE)
    o = O.fuse_tat(vs, D.TAT_INTERMEDIATE, D.FUSE_FP64)
    _same(g, o)


def test_tat_errors(ctx, small_scene):
    vs = tat_views(small_scene, seed=25)
    with pytest.raises(D.DPEError) as e:
        ctx.fuse_tat(vs, D.TAT_ADVANCED, D.FUSE_FP64, capacity=5)
    assert e.value.status == D.ERR_CAPACITY
    with pytest.raises(D.DPEError) as e:
        ctx.fuse_tat(vs, 7, D.FUSE_FP64)
    assert e.value.status == D.ERR_INVALID_ARGUMENT
    bad = [dict(v) for v in vs]
    bad[0]["src"] = [0, 1]  # a view may not be its own source
    with pytest.raises(D.DPEError) as e:
        ctx.fuse_tat(bad, D.TAT_ADVANCED, D.FUSE_FP64)
    assert e.value.status == D.ERR_INVALID_ARGUMENT


def test_tat_one_source_keeps_nothing(ctx, tiny_scene):
    vs = tat_views(tiny_scene, seed=26)
    for v in vs:
        v["src"] = v["src"][:1]
    assert ctx.fuse_tat(vs, D.TAT_ADVANCED)["count"] == 0
