"""CPU tests of the reference's region labelling Connect (DPE.cpp:27-134): the oracle's literal C++
restatement against a pure-Python one on small cases, the host preprocessing's row-vectorised form
against the oracle up to full size, and the lossy joins that make it differ from plain connected
components."""
import numpy as np
import pytest

import edges as E
import helpers as h
import oracle_py as O

cv2 = pytest.importorskip("cv2")


def connect_literal(d):
    """Connect, line by line in Python (small images only)."""
    rows, cols = d.shape
    lab = [[0] * cols for _ in range(rows)]
    conn = [0]
    cnt = 1
    for y in range(rows):
        for x in range(cols):
            if d[y, x] == 255:
                continue
            left = x > 0 and d[y, x] == 0 and d[y, x - 1] == 0
            up = y > 0 and d[y, x] == 0 and d[y - 1, x] == 0
            if left:
                lab[y][x] = lab[y][x - 1]
            if up:
                lab[y][x] = lab[y - 1][x]
            if not left and not up:
                lab[y][x] = cnt
                conn.append(cnt)
                cnt += 1
            elif left and up:
                l_, u_ = lab[y][x - 1], lab[y - 1][x]
                if l_ > u_:
                    conn[l_] = u_
                    lab[y][x] = u_
                elif l_ < u_:
                    conn[u_] = l_
                    lab[y][x] = l_
    for i in range(1, len(conn)):
        cur, pre = conn[i], conn[conn[i]]
        while pre != cur:
            cur, pre = pre, conn[pre]
        conn[i] = cur
    num, mapping = 1, [0] * len(conn)
    for i in range(1, len(conn)):
        if conn[i] == i:
            mapping[i] = num
            num += 1
    out = np.array([[mapping[conn[lab[y][x]]] for x in range(cols)] for y in range(rows)], np.int32)
    return out, np.bincount(out.ravel(), minlength=num)


def _random_masks(n, seed, max_side=40):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        hh, ww = rng.integers(1, max_side, 2)
        out.append(np.where(rng.random((hh, ww)) < rng.uniform(0.2, 0.8), 255, 0).astype(np.uint8))
        out.append(rng.choice(np.array([0, 0, 0, 7, 255], np.uint8), (hh, ww)))  # other values open labels
    return out


def _scene_masks():
    """EdgeSegment's first labelling input: Roberts > 4 on the 4x-downsampled view."""
    out = []
    for name in ("small_weak", "c2_small"):
        sc = h.S.make_scene(name, seed=2)
        for v in range(2):
            g = sc.gray[v]
            d = cv2.resize(g, (g.shape[1] // 2, g.shape[0] // 2), interpolation=cv2.INTER_LINEAR)
            d = cv2.resize(d, (d.shape[1] // 2, d.shape[0] // 2), interpolation=cv2.INTER_LINEAR)
            _, d = cv2.threshold(E.roberts(d), 4, 255, cv2.THRESH_BINARY)
            out.append(np.ascontiguousarray(d))
    return out


def test_oracle_matches_literal_restatement():
    for d in _random_masks(15, 1) + _scene_masks()[:2]:
        a, ca = O.connect(d)
        b, cb = connect_literal(d)
        assert np.array_equal(a, b) and np.array_equal(ca, cb)


def test_host_vectorised_form_matches_oracle():
    rng = np.random.default_rng(3)
    big = np.where(rng.random((1200, 1600)) < 0.3, 255, 0).astype(np.uint8)
    for d in _random_masks(20, 2) + _scene_masks() + [big]:
        a, ca = O.connect(d)
        b, cb = E.connect(d)
        assert np.array_equal(a, b) and np.array_equal(ca, cb)


def test_joins_are_lossy():
    """An overwritten join splits a region: fewer plain 4-connected components than labels."""
    from scipy import ndimage

    d = _scene_masks()[2]
    _, counts = O.connect(d)
    _, n_cc = ndimage.label(d != 255, structure=[[0, 1, 0], [1, 1, 1], [0, 1, 0]])
    assert len(counts) - 1 > n_cc
    # and the smallest such case among random 8x8 masks is reproduced by every form
    rng = np.random.default_rng(11)
    for _ in range(5000):
        m = np.where(rng.random((8, 8)) < 0.35, 255, 0).astype(np.uint8)
        lab, c = O.connect(m)
        if len(c) - 1 != ndimage.label(m == 0, structure=[[0, 1, 0], [1, 1, 1], [0, 1, 0]])[1]:
            assert np.array_equal(lab, connect_literal(m)[0]) and np.array_equal(lab, E.connect(m)[0])
            return
    pytest.fail("no lossy 8x8 case found")


# ------------------------------------------------------------------ the OpenCV parts and the whole map
def test_resize_u8_matches_opencv():
    rng = np.random.default_rng(4)
    for (sh, sw, dh, dw) in [(1200, 1600, 600, 800), (600, 800, 300, 400), (75, 100, 300, 400), (37, 51, 150, 200),
                             (300, 400, 1200, 1600), (20, 30, 77, 93), (301, 401, 150, 200), (7, 9, 300, 301),
                             (150, 200, 75, 100), (33, 47, 33, 47)]:
        img = rng.integers(0, 256, (sh, sw), dtype=np.uint8)
        for use_ipp in (True, False):
            cv2.ipp.setUseIPP(use_ipp)
            try:
                ref = cv2.resize(img, (dw, dh), interpolation=cv2.INTER_LINEAR)
            finally:
                cv2.ipp.setUseIPP(True)
            assert np.array_equal(O.resize_u8(img, dw, dh), ref), ((sh, sw, dh, dw), use_ipp)


def _weak_region_borders(gray, scale=0):
    """EdgeSegment's Hough inputs: the outer border of each large weak region (DPE.cpp:164-187)."""
    rows, cols = gray.shape
    weak_tex_num = int(1.0 * rows * cols / (1024 << scale << scale))
    d = cv2.resize(gray, (cols // 2, rows // 2), interpolation=cv2.INTER_LINEAR)
    d = cv2.resize(d, (d.shape[1] // 2, d.shape[0] // 2), interpolation=cv2.INTER_LINEAR)
    thr = int(int(min(d.shape)) / 30.0)
    _, d = cv2.threshold(E.roberts(d), 4, 255, cv2.THRESH_BINARY)
    lab, cnt = E.connect(d)
    out = []
    for k in range(1, len(cnt)):
        if cnt[k] < weak_tex_num:
            continue
        inside = lab == k
        border = np.zeros_like(inside)
        border[:, 1:] |= inside[:, :-1]
        border[:, :-1] |= inside[:, 1:]
        border[1:, :] |= inside[:-1, :]
        border[:-1, :] |= inside[1:, :]
        out.append((np.where(border & ~inside, 255, 0).astype(np.uint8), thr))
    return out


def test_hough_lines_p_matches_opencv():
    import math

    n = 0
    for name in ("small_weak", "c2_small"):
        sc = h.S.make_scene(name, seed=2)
        for v in range(3):
            for img, thr in _weak_region_borders(sc.gray[v]):
                ref = cv2.HoughLinesP(img, 1, math.pi / 180, thr, minLineLength=thr, maxLineGap=thr)
                ref = [] if ref is None else [tuple(int(t) for t in r) for r in ref[:, 0, :]]
                assert O.hough_lines_p(img, thr, thr, thr) == ref
                n += len(ref)
    assert n > 200


@pytest.mark.parametrize("name,scale", [("small_weak", 0), ("c2_small", 0), ("c2_small", 1), ("c2_small", 2)])
def test_edge_labels_match_host_preprocessing(name, scale):
    """The whole label map: the oracle's restatement against edges.py, which runs the same
    sequence with cv2's resize, threshold, HoughLinesP and line."""
    sc = h.S.make_scene(name, seed=2)
    for v in range(2):
        o = O.edge_labels(sc.gray[v], scale)
        ref = E.edge_segment(scale, sc.gray[v], 1, False)
        assert o.shape == ref.shape and np.array_equal(o, ref), (v, int((o != ref).sum()))
