"""The batching workload's layout (CPU): 49 reference views of three sizes on the 60-camera ring, each
with its 10 nearest ring neighbours as sources, and renderings whose depth agrees with the camera
struct the kernels receive."""
import numpy as np

import scene as S


def test_c5_layout():
    lay = S.c5_views()
    assert len(lay) == 49
    sizes = [(w, h) for _, w, h, _ in lay]
    assert sizes.count((640, 480)) == 20 and sizes.count((1600, 1200)) == 20 and sizes.count((3200, 2400)) == 9
    refs = [r for r, _, _, _ in lay]
    assert len(set(refs)) == 49 and all(0 <= r < 60 for r in refs)
    for r, _, _, srcs in lay:
        assert len(srcs) == 10 == len(set(srcs)) and r not in srcs
        ring_dist = sorted(min((s - r) % 60, (r - s) % 60) for s in srcs)
        assert ring_dist == [1, 1, 2, 2, 3, 3, 4, 4, 5, 5]


def test_c5_rendering_matches_camera():
    ring = S.RingScene("c5_ring", seed=1)
    W, H = 160, 120
    gray, bgr, depth = ring.render(7, W, H)
    assert gray.shape == (H, W) and bgr.shape == (H, W, 3) and depth.shape == (H, W)
    assert np.isfinite(depth).all() and depth.min() > 0.5 and depth.max() < ring.spec.depth_max
    assert 20 < gray.std() < 80  # textured everywhere (objects and wall)
    cam = ring.camera(7, W, H)
    K = np.asarray(cam["K"], np.float64).reshape(3, 3)
    R = np.asarray(cam["R"], np.float64).reshape(3, 3)
    t = np.asarray(cam["t"], np.float64)
    assert cam["width"] == W and cam["height"] == H
    # multi-view consistency through the camera structs: points of camera 7 back-projected with their
    # ray-cast depth land, in the neighbouring camera 8, on pixels whose ray-cast depth matches
    _, _, depth8 = ring.render(8, W, H)
    c8 = ring.camera(8, W, H)
    K8 = np.asarray(c8["K"], np.float64).reshape(3, 3)
    R8 = np.asarray(c8["R"], np.float64).reshape(3, 3)
    t8 = np.asarray(c8["t"], np.float64)
    ok = 0
    for v in range(20, H - 20, 10):
        for u in range(20, W - 20, 10):
            Xw = R.T @ (depth[v, u] * np.linalg.solve(K, np.array([u, v, 1.0])) - t)
            x = K8 @ (R8 @ Xw + t8)
            u8, v8 = int(round(x[0] / x[2])), int(round(x[1] / x[2]))
            if 0 <= u8 < W and 0 <= v8 < H and abs(depth8[v8, u8] - x[2]) < 0.03 * x[2]:
                ok += 1
    assert ok >= 0.8 * len(range(20, H - 20, 10)) * len(range(20, W - 20, 10))
