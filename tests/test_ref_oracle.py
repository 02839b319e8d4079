"""The oracle pinned to the reference itself.

oracle/Makefile compiles the reference's own DPE.cu and DPE.cpp for the CPU (oracle/_ref/libref.so,
behind the host stand-ins of oracle/refshim/), and oracle/ref_harness.cpp drives them the way
ProcessProblem (main.cpp:241-264) and RunFusion (DPE.cpp:1387-1548) run.  Here the restatement in
oracle/ is compared with that build on identical inputs and identical random streams.

With the reference's arithmetic selected in the oracle -- raw moments, the tex2D(x + 0.5, y + 0.5)
addressing, and the same-colour read race of the edge-aware update resolved as the serial run of the
reference's kernels resolves it -- every output is identical bit for bit: planes, pixel states,
selected views and final costs, on the first-init, weak-texture (APD, edges, limits, labels, adaptive
radius) and geometric-consistency paths, and every fused point.  Each of those three switches is one
documented difference between the reference and the oracle's default (the CUDA kernels' arithmetic),
so this test also measures what each one does to the result.

Nothing here runs on a GPU.  The reference's kernels read a little outside their buffers (Bresenham
ray ends, the edge-mode view prior); on the CPU every buffer sits between zero-filled guard zones,
so those reads read 0, and the test checks that the reference never WRITES there.
"""
import numpy as np
import pytest

import dpe_b200 as D
import helpers as h
import oracle_py as O
import ref_py as R

pytestmark = pytest.mark.skipif(not R.available(), reason="the reference sources are absent and no host build "
                                                          "of them travelled (oracle/_ref/libref.so)")

DEPTH_REL_TOL = 1e-3
DEPTH_FRACTION = 0.995


@pytest.fixture(autouse=True)
def _oracle_defaults():
    yield
    O.reference_arithmetic(False)
    O.set_serial_race(False)


def _identical(a, b):
    """Fraction of pixels whose outputs are the same bits, per output."""
    out = {}
    for k in ("plane", "weak", "views", "costs"):
        x, y = a[k], b[k]
        if x.dtype == np.float32:
            eq = x.view(np.uint32) == y.view(np.uint32)
            if eq.ndim == 3:
                eq = eq.all(-1)
        else:
            eq = x == y
        out[k] = float(eq.mean())
    return out


def _oracle_like(ref_out, images, **kw):
    """The oracle on the cameras and parameters the reference derived from its own files."""
    return O.pm_run(images, R.camera_dicts(ref_out["cameras"]), ref_out["params"], **kw)


def _weak_inputs(geom: bool):
    ws = h.S.make_scene("small_weak", seed=2)
    ref = 2 if geom else 1
    images, cams, srcs = h.view_inputs(ws, ref)
    p0 = h.first_init_params(ws, len(images))
    r0 = R.pm_call(images, cams, p0, seed=21)
    o0 = _oracle_like(r0, images, seed=21)
    state, weak = h.post_process(o0["plane"], o0["weak"], r0["params"].depth_min, r0["params"].depth_max)
    edge, low, label = h.synthetic_edges(ws.gray[ref])
    p = h.refine_params(ws, len(images), level=1, state=D.REFINE_ITER if geom else D.REFINE_INIT, geom=geom)
    p.max_scale_size = edge.shape[1] // low.shape[1]  # edges_<log2 of this>.dmb is the low-resolution map
    kw = dict(plane_in=state, views_in=np.ascontiguousarray(o0["views"]), weak_in=weak, edge=edge, edge_low=low,
              label=label, seed=77)
    if geom:
        # the reference reads every view's depth from its state; the reference view's is the state's
        kw["depths"] = [np.ascontiguousarray(state[..., 3])] + [np.ascontiguousarray(ws.depth[i].astype(np.float32))
                                                               for i in srcs]
    return ws, ref, images, cams, p, kw


def test_first_init_bit_identical_to_reference(small_scene):
    images, cams, _ = h.view_inputs(small_scene, 0)
    p = h.first_init_params(small_scene, len(images))
    r = R.pm_call(images, cams, p, seed=1234)
    assert r["guard_writes"] == 0
    O.reference_arithmetic(True)
    same = _identical(r, _oracle_like(r, images, seed=1234))
    print("first init, reference arithmetic:", same)
    assert all(v == 1.0 for v in same.values()), same
    # the oracle's default arithmetic (compensated moments, the kernels' texture addressing) meets
    # the parity bar against the reference's own result
    O.reference_arithmetic(False)
    o = _oracle_like(r, images, seed=1234)
    agree = h.rel_depth_agreement(o["plane"][..., 3], r["plane"][..., 3], DEPTH_REL_TOL)
    print(f"first init, default arithmetic: depth agreement {agree:.5f}, identical {_identical(r, o)}")
    assert agree >= DEPTH_FRACTION


_CALLS = {}


def _reference_call(geom: bool):
    """The reference's weak-texture (geom False) or geometric (geom True) call, run once per module."""
    if geom not in _CALLS:
        ws, ref, images, cams, p, kw = _weak_inputs(geom)
        _CALLS[geom] = (ws, ref, images, kw, R.pm_call(images, cams, p, **kw))
    return _CALLS[geom]


@pytest.mark.parametrize("geom", [False, True], ids=["weak_refine_init", "geom_refine_iter"])
def test_weak_and_geom_paths_bit_identical_to_reference(geom):
    ws, ref, images, kw, r = _reference_call(geom)
    assert r["guard_writes"] == 0
    assert (r["weak"] == D.WEAK).mean() > 0.02  # the weak-texture pass has work
    O.reference_arithmetic(True)
    O.set_serial_race(True)
    same = _identical(r, _oracle_like(r, images, **kw))
    print(f"{'geom' if geom else 'weak'} path, reference arithmetic + serial race:", same)
    assert all(v == 1.0 for v in same.values()), same


def test_race_resolution_is_the_only_edge_mode_difference():
    """With the reference's arithmetic but the oracle's snapshot resolution of the same-colour race
    (the CUDA kernels' resolution), the edge-aware geometric call differs from the serial reference
    run: the race decides which of two valid readings propagates.  Both are the reference's method;
    their accuracy against ground truth agrees."""
    ws, ref, images, kw, r = _reference_call(True)
    O.reference_arithmetic(True)
    O.set_serial_race(False)
    o = _oracle_like(r, images, **kw)
    agree = h.rel_depth_agreement(o["plane"][..., 3], r["plane"][..., 3], DEPTH_REL_TOL)
    gt = ws.depth[ref].astype(np.float64)

    def acc(plane):
        d = plane[..., 3].astype(np.float64)
        return float((np.abs(d - gt) <= 0.01 * gt).mean())

    print(f"snapshot vs serial race: depth agreement {agree:.4f}; GT accuracy {acc(o['plane']):.4f} vs "
          f"{acc(r['plane']):.4f}")
    assert abs(acc(o["plane"]) - acc(r["plane"])) <= 0.02


def test_fusion_bit_identical_to_reference():
    from test_oracle import _gt_fusion_views

    sc = h.S.make_scene("small", seed=5)
    views = _gt_fusion_views(sc, noise=0.002, seed=9)
    r = R.fuse(views)
    o = O.fuse(views, D.FUSE_FLOAT)
    print(f"fusion: reference {r['count']} points, oracle {o['count']}")
    assert r["count"] == o["count"] > 1000
    assert np.array_equal(r["xyz"].view(np.uint32), o["xyz"].view(np.uint32))
    assert np.array_equal(r["bgr"], o["bgr"])


def test_reference_build_rejects_inputs_it_cannot_take(small_scene):
    images, cams, _ = h.view_inputs(small_scene, 0)
    p = h.first_init_params(small_scene, len(images))
    bad = [images[0] + 0.5] + images[1:]  # the reference reads 8-bit image files
    with pytest.raises(RuntimeError, match="integer grey levels"):
        R.pm_call(bad, cams, p, seed=1)


@pytest.mark.parametrize("variant", ["intermediate", "advanced"])
def test_tat_fusion_bit_identical_to_reference(variant):
    """RunFusion_TAT_Intermediate / RunFusion_TAT_advanced (DPE.cpp:1550-1867), block masks included,
    against the oracle's float mode."""
    from test_fusion_tat import tat_views

    sc = h.S.make_scene("small", seed=5)
    views = tat_views(sc, noise=2e-4, seed=19)
    o = O.fuse_tat(views, D.TAT_INTERMEDIATE if variant == "intermediate" else D.TAT_ADVANCED, D.FUSE_FLOAT)
    r = R.fuse(views, R.TAT_INTERMEDIATE if variant == "intermediate" else R.TAT_ADVANCED)
    print(f"TAT {variant}: reference {r['count']} points, oracle {o['count']}")
    assert r["count"] == o["count"] > 1000
    assert np.array_equal(r["xyz"].view(np.uint32), o["xyz"].view(np.uint32))
    assert np.array_equal(r["bgr"], o["bgr"])


def test_label_map_parts_bit_identical_to_reference():
    """Roberts (DPE.cpp:9-25) and Connect (DPE.cpp:27-134), which EdgeSegment's label map is built
    from: the oracle's Connect and the host preprocessing's Roberts against the reference's own."""
    import edges as E
    from test_labels import _random_masks, _scene_masks

    rng = np.random.default_rng(11)
    for d in _random_masks(12, 5) + _scene_masks()[:2]:
        a, ca = O.connect(d)
        b, cb = R.connect(d)
        assert np.array_equal(a, b) and np.array_equal(ca, cb)
    for shape in ((48, 64), (121, 163)):
        img = rng.integers(0, 256, shape).astype(np.uint8)
        assert np.array_equal(E.roberts(img), R.roberts(img))
