"""GPU parity of the device edge maps (dpe_edge_map, dpe_schedule.device_edges) against the CPU
restatement of EdgeSegment's mode 0 (oracle/edge_oracle.py, itself pinned to cv2.Canny): bit-exact
maps, and a whole schedule with device-made edge maps identical to one fed the host's maps."""
import numpy as np
import pytest

import dpe_b200 as D
import edge_oracle as EO
import edges as E
import helpers as h
from test_edges import IMAGES

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,img", IMAGES, ids=[n for n, _ in IMAGES])
def test_edge_map_matches_oracle(ctx, name, img):
    g = ctx.edge_map(img)
    o = EO.edge_map(img)
    assert np.array_equal(g, o), (name, int((g != o).sum()))


def test_edge_map_full_size(ctx):
    """A 1600x1200 level image (the benchmark's finest level): piecewise-constant blocks, a ramp
    and noise, so every suppression sector and long hysteresis chains occur."""
    rng = np.random.default_rng(8)
    img = np.kron(rng.integers(0, 256, (60, 80)), np.ones((20, 20))).astype(np.float64)
    img += np.linspace(0, 40, 1600)[None, :] + rng.normal(0, 6, (1200, 1600))
    img = np.clip(np.rint(img), 0, 255).astype(np.uint8)
    g = ctx.edge_map(img)
    o = EO.edge_map(img)
    print(f"full-size edge map: {int((o > 0).sum())} edge pixels")
    assert np.array_equal(g, o)


@pytest.mark.parametrize("shape", [(1, 1), (1, 9), (9, 1), (2, 2), (3, 7), (17, 2)])
def test_edge_map_small_shapes(ctx, shape):
    rng = np.random.default_rng(sum(shape))
    img = rng.integers(0, 256, shape, dtype=np.uint8)
    assert np.array_equal(ctx.edge_map(img), EO.edge_map(img))


def test_edge_map_device_memory(ctx):
    import torch

    img = IMAGES[3][1]
    g = ctx.edge_map(torch.from_numpy(img).cuda(), memory=D.MEM_DEVICE)
    assert np.array_equal(g.cpu().numpy(), EO.edge_map(img))


def test_edge_map_rejects_bad_arguments(ctx):
    with pytest.raises(D.DPEError) as e:
        ctx.edge_map(np.zeros((0, 5), np.uint8))
    assert e.value.status == D.ERR_INVALID_ARGUMENT


def test_scene_device_edges_match_host_edges(ctx):
    """dpe_scene_run making each level's edge map itself (from its own level image) gives the same
    depth maps, states, views and points as the run fed the host's edge maps."""
    sc = h.S.make_scene("small_weak", seed=3)
    V, L = sc.n, 2
    edges_l, labels_l = [], []
    for v in range(V):
        ev, lv = zip(*[E.level_inputs(sc.gray[v], 1 << (L - 1 - l)) for l in range(L)])
        edges_l.append([np.ascontiguousarray(e) for e in ev])
        labels_l.append([np.ascontiguousarray(x) for x in lv])
    cams = [h.S.camera_struct(sc, v) for v in range(V)]
    kw = dict(num_levels=L, refine_calls=1, max_iterations=2, fuse_mode=D.FUSE_FP64, seed=17)
    host = ctx.scene_run(list(sc.gray), list(sc.bgr), cams, sc.pairs, edges_l, labels_l, **kw)
    dev = ctx.scene_run(list(sc.gray), list(sc.bgr), cams, sc.pairs, None, labels_l, device_edges=True, **kw)
    for v in range(V):
        for k in ("depth", "normal", "weak", "views"):
            assert np.array_equal(dev[k][v], host[k][v]), (k, v)
    assert dev["points"] == host["points"] and np.array_equal(dev["xyz"], host["xyz"])
    with pytest.raises(D.DPEError):  # edges given and asked for on the device
        ctx.scene_run(list(sc.gray), list(sc.bgr), cams, sc.pairs, edges_l, labels_l, device_edges=True, **kw)
