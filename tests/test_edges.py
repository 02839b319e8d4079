"""CPU tests of the edge-map restatement (oracle/edge_oracle.py) against OpenCV, the library the
reference calls for it (cv::Canny in EdgeSegment, DPE.cpp:221), bit for bit."""
import numpy as np
import pytest

import edge_oracle as EO
import edges as E
import helpers as h

cv2 = pytest.importorskip("cv2")


def _images():
    """Level images of the synthetic scenes as GetProblemEdges makes them, plus noise, ramps,
    constants and near-saturated content."""
    out = []
    for name, levels in (("tiny", 1), ("small", 2), ("c2_small", 2)):
        sc = h.S.make_scene(name, seed=2)
        for v in range(min(2, sc.n)):
            for lvl in range(levels):
                scale_size = 1 << lvl
                rows, cols = sc.gray[v].shape
                f = 1.0 / float(scale_size)
                lev = cv2.resize(sc.gray[v].astype(np.float32), (int(round(cols * f)), int(round(rows * f))),
                                 interpolation=cv2.INTER_LINEAR)
                out.append((f"{name}/v{v}/s{scale_size}", EO.level_image_u8(lev)))
    rng = np.random.default_rng(5)
    out.append(("noise", rng.integers(0, 256, (97, 131), dtype=np.uint8)))
    out.append(("ramp", np.tile(np.arange(200, dtype=np.uint8), (50, 1))))
    out.append(("zeros", np.zeros((40, 30), np.uint8)))
    out.append(("all255", np.full((33, 47), 255, np.uint8)))  # median -1: thresholds 0 and -1
    sat = np.full((64, 64), 255, np.uint8)
    sat[16:48, 16:48] = rng.integers(200, 256, (32, 32), dtype=np.uint8)
    out.append(("saturated", sat))
    out.append(("blocks", np.kron(rng.integers(0, 256, (8, 10), dtype=np.uint8), np.ones((9, 7), np.uint8))))
    return out


IMAGES = _images()


@pytest.mark.parametrize("name,img", IMAGES, ids=[n for n, _ in IMAGES])
def test_canny_restatement_matches_opencv(name, img):
    t1, t2 = EO.median_thresholds(img)
    mine = EO.canny_l2(img, t1, t2)
    for use_ipp in (True, False):
        cv2.ipp.setUseIPP(use_ipp)
        try:
            ref = cv2.Canny(img, t1, t2, apertureSize=3, L2gradient=True)
        finally:
            cv2.ipp.setUseIPP(True)
        assert np.array_equal(mine, ref), (name, use_ipp, int((mine != ref).sum()))


@pytest.mark.parametrize("name,img", IMAGES, ids=[n for n, _ in IMAGES])
def test_edge_map_matches_host_edge_segment(name, img):
    """The whole mode-0 map against the host preprocessing that feeds the kernels (edges.py, which
    calls cv2 the way EdgeSegment does)."""
    assert np.array_equal(EO.edge_map(img), E.edge_segment(0, img, 0, True))


@pytest.mark.parametrize("shape", [(1, 1), (1, 9), (9, 1), (2, 2), (3, 7), (17, 2), (1200, 1600)])
def test_canny_restatement_small_and_full_shapes(shape):
    rng = np.random.default_rng(sum(shape))
    if shape[0] > 100:  # a full-size level: blocks, a ramp and noise
        img = np.kron(rng.integers(0, 256, (60, 80)), np.ones((20, 20))) + np.linspace(0, 40, 1600)[None, :]
        img = np.clip(np.rint(img + rng.normal(0, 6, shape)), 0, 255).astype(np.uint8)
    else:
        img = rng.integers(0, 256, shape, dtype=np.uint8)
    t1, t2 = EO.median_thresholds(img)
    assert np.array_equal(EO.canny_l2(img, t1, t2), cv2.Canny(img, t1, t2, apertureSize=3, L2gradient=True))


def test_median_thresholds_float_rule():
    # (1 - 0.67f) * median is evaluated in float (DPE.cpp:217-218); in double it would truncate
    # to one less at medians 100 and 200
    for m in range(-1, 255):
        img = np.full(10, max(m, 0), np.uint8) if m >= 0 else np.full(10, 255, np.uint8)
        t1, t2 = EO.median_thresholds(img)
        assert t2 == m
        assert t1 == int((1 - 0.67) * m) + (1 if m in (100, 200) else 0)
    assert EO.median_thresholds(np.full(10, 100, np.uint8)) == (33, 100)


def test_border_rule_order():
    d = np.full((4, 5), 255, np.uint8)
    d[1, 1] = 0  # clears (1, 0) in the row pass, then (0, 0) reads it in the column pass
    r = EO.border_rule(d)
    assert r[1, 0] == 0 and r[0, 1] == 0 and r[0, 0] == 0
    assert r[3, 4] == 255
