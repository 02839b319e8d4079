"""GPU parity of the device label maps (dpe_edge_labels, dpe_schedule.device_labels) against the CPU
restatement of EdgeSegment's mode 1 (oracle/label_oracle.cpp, itself pinned to cv2 and to a
line-by-line restatement of Connect): identical int32 maps, and a whole schedule with device-made
edge and label maps identical to one fed the host's maps."""
import numpy as np
import pytest

import dpe_b200 as D
import edges as E
import helpers as h
import oracle_py as O

pytestmark = pytest.mark.gpu


def _check(ctx, gray, scale, high_res_img=True):
    g = ctx.edge_labels(gray, scale, high_res_img)
    o = O.edge_labels(gray, scale, high_res_img)
    assert g.shape == o.shape
    assert np.array_equal(g, o), int((g != o).sum())
    return o


@pytest.mark.parametrize("name,scale", [("small_weak", 0), ("c2_small", 0), ("c2_small", 1), ("c2_small", 2)])
def test_edge_labels_match_oracle(ctx, name, scale):
    sc = h.S.make_scene(name, seed=2)
    for v in range(3):
        o = _check(ctx, sc.gray[v], scale)
    print(f"{name} scale {scale}: {int(o.max())} regions, {int((o == -1).sum())} pixels in small regions")


def test_edge_labels_without_high_res(ctx):
    sc = h.S.make_scene("c2_small", seed=4)
    _check(ctx, sc.gray[0], 1, high_res_img=False)


def test_edge_labels_full_size(ctx):
    """The benchmark's 1600x1200 views at their three levels."""
    sc = h.S.make_scene("c2", seed=1, device="cuda")
    for v in (0, 5):
        for scale in (2, 1, 0):
            o = _check(ctx, sc.gray[v], scale)
            assert o.max() > 10


def test_edge_labels_device_memory(ctx):
    import torch

    sc = h.S.make_scene("c2_small", seed=2)
    g = ctx.edge_labels(torch.from_numpy(sc.gray[1]).cuda(), 1, memory=D.MEM_DEVICE)
    assert np.array_equal(g.cpu().numpy(), O.edge_labels(sc.gray[1], 1))


def test_scene_device_edges_and_labels_match_host_maps(ctx):
    """dpe_scene_run making each level's edge and label maps itself gives the results of the run fed
    the host preprocessing's maps (which call OpenCV as the reference does)."""
    sc = h.S.make_scene("small_weak", seed=3)
    V, L = sc.n, 2
    edges_l, labels_l = [], []
    for v in range(V):
        ev, lv = zip(*[E.level_inputs(sc.gray[v], 1 << (L - 1 - l)) for l in range(L)])
        edges_l.append([np.ascontiguousarray(e) for e in ev])
        labels_l.append([np.ascontiguousarray(x) for x in lv])
    cams = [h.S.camera_struct(sc, v) for v in range(V)]
    kw = dict(num_levels=L, refine_calls=1, max_iterations=2, fuse_mode=D.FUSE_FP64, seed=23)
    host = ctx.scene_run(list(sc.gray), list(sc.bgr), cams, sc.pairs, edges_l, labels_l, **kw)
    dev = ctx.scene_run(list(sc.gray), list(sc.bgr), cams, sc.pairs, None, None, device_edges=True,
                        device_labels=True, **kw)
    for v in range(V):
        for k in ("depth", "normal", "weak", "views"):
            assert np.array_equal(dev[k][v], host[k][v]), (k, v)
    assert dev["points"] == host["points"] and np.array_equal(dev["xyz"], host["xyz"])
