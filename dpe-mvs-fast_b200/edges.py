"""Edge and label maps the PatchMatch kernels read (host preprocessing, OpenCV).

Restates EdgeSegment / Roberts / Connect (DPE.cpp:9-291) and GetProblemEdges (main.cpp:166-221)
with the same OpenCV calls through cv2: Canny with a median-derived threshold for the edge map
(mode 0), and for the label map (mode 1) a Roberts gradient on the 4x-downsampled image,
the reference's region labelling (Connect, whose lossy joins can split a region), Hough-line
closure of large weak regions, a second labelling at the target scale and small regions marked
-1.  The reference caches these per scale as
edges_<scale>.dmb / labels_<scale>.dmb.
"""
from __future__ import annotations

import math

import numpy as np

try:
    import cv2
except ImportError:  # pragma: no cover - cv2 ships with the image
    cv2 = None


def _need_cv2():
    if cv2 is None:
        raise RuntimeError("edge/label precompute needs OpenCV (cv2)")


def roberts(src: np.ndarray) -> np.ndarray:
    """Roberts cross magnitude (DPE.cpp:9-25); border pixels get t1 = t2 = 50."""
    s = src.astype(np.int32)
    out = np.full(s.shape, 50 * 50 * 2, np.int64)
    t1 = s[1:-1, 1:-1] - s[2:, 2:]   # (i, j) - (i+1, j+1) for interior i, j
    t2 = s[2:, 1:-1] - s[1:-1, 2:]   # (i+1, j) - (i, j+1)
    out[1:-1, 1:-1] = t1.astype(np.int64) ** 2 + t2.astype(np.int64) ** 2
    # (uchar)sqrt(int): truncation to int, then the low byte (x86 conversion of values > 255)
    return (np.sqrt(out.astype(np.float64)).astype(np.int64) & 0xFF).astype(np.uint8)


def connect(binary: np.ndarray):
    """Connect (DPE.cpp:27-134): the reference's labelling of the pixels other than 255.

    Not plain connected components.  The reference scans in raster order with provisional labels
    (a pixel joins its left and upper neighbours when both it and they are 0, taking the smaller
    label; otherwise it opens a new label) and records a join of two different labels as
    connection[larger] = smaller, overwriting any earlier join of that label; the final label of a
    provisional label is the end of its connection chain, renumbered in increasing order.  An
    overwritten join is lost, so a region can end up split.  Returns (labels int32, counts per
    label), label 0 being the 255 pixels.

    Evaluated a row at a time: along a run of left-joined pixels the provisional label is the
    running minimum of the run's opening label and the upper labels where the pixel joins upwards
    (a segmented minimum-scan), new labels are numbered by a prefix count of the run openings
    without an upper join, and for each label only the last join in raster order is kept."""
    d = np.asarray(binary)
    rows, cols = d.shape
    lab = np.zeros((rows, cols), np.int64)
    nxt = 1
    last_join = {}  # larger provisional label -> smaller label of its last join
    zero_prev = None
    lab_prev = None
    xs = np.arange(cols)
    BIG = np.int64(1) << 40
    for y in range(rows):
        row = d[y]
        labelled = row != 255
        zero = row == 0
        leftj = np.zeros(cols, bool)
        leftj[1:] = zero[1:] & zero[:-1]
        upj = zero & zero_prev if zero_prev is not None else np.zeros(cols, bool)
        opens = labelled & ~leftj & ~upj
        new_ids = nxt + np.cumsum(opens) - 1
        nxt += int(opens.sum())
        up = lab_prev if lab_prev is not None else np.zeros(cols, np.int64)
        # value contributed at each pixel: its upper label where it joins up, its new label where
        # it opens one, +inf otherwise (a left-joined pixel takes the running value)
        val = np.where(upj, up, np.where(opens, new_ids, BIG))
        run = np.cumsum(~leftj) - 1  # run index; a run restarts wherever there is no left join
        shifted = val - run * (BIG * 4)
        lrow = np.minimum.accumulate(shifted) + run * (BIG * 4)
        lrow = np.where(labelled, lrow, 0)
        # joins: both neighbours joined and their labels differ (the left pixel's final label)
        both = leftj & upj
        if both.any():
            xb = xs[both]
            left_lab = lrow[xb - 1]
            up_lab = up[xb]
            diff = left_lab != up_lab
            big_l = np.maximum(left_lab, up_lab)[diff]
            small_l = np.minimum(left_lab, up_lab)[diff]
            for t, v in zip(big_l.tolist(), small_l.tolist()):
                last_join[t] = v
        lab[y] = lrow
        zero_prev, lab_prev = zero, lrow
    conn = np.arange(nxt, dtype=np.int64)
    if last_join:
        t = np.fromiter(last_join.keys(), np.int64)
        conn[t] = np.fromiter(last_join.values(), np.int64)
    while True:  # chain ends: every join points to a smaller label, so this converges
        nc = conn[conn]
        if np.array_equal(nc, conn):
            break
        conn = nc
    is_root = conn == np.arange(nxt)
    is_root[0] = False
    mapping = np.zeros(nxt, np.int64)
    mapping[is_root] = np.arange(1, int(is_root.sum()) + 1)
    final = mapping[conn]
    out = final[lab]
    counts = np.bincount(out.ravel(), minlength=int(is_root.sum()) + 1)
    return out.astype(np.int32), counts


def _border_fix(d: np.ndarray) -> None:
    """Zero the image border where the adjacent inner pixel is zero (DPE.cpp:239-250)."""
    rows, cols = d.shape
    for y in range(rows):
        if d[y, 1] == 0:
            d[y, 0] = 0
        if d[y, cols - 2] == 0:
            d[y, cols - 1] = 0
    for x in range(cols):
        if d[1, x] == 0:
            d[0, x] = 0
        if d[rows - 2, x] == 0:
            d[rows - 1, x] = 0


def edge_segment(scale: int, src: np.ndarray, mode: int, use_canny: bool, high_res_img: bool = True) -> np.ndarray:
    """EdgeSegment (DPE.cpp:136-291): mode 0 -> uint8 edge map, mode 1 -> int32 label map."""
    _need_cv2()
    robthr = 4 if high_res_img else 6
    rows, cols = src.shape
    weak_tex_num = int(1.0 * rows * cols / (1024 << scale << scale))
    src_down = cv2.resize(src, (cols // 2, rows // 2), interpolation=cv2.INTER_LINEAR) if high_res_img else src.copy()
    if not use_canny:
        src_down = cv2.resize(src_down, (src_down.shape[1] // 2, src_down.shape[0] // 2), interpolation=cv2.INTER_LINEAR)
        m = min(src_down.shape[1], src_down.shape[0])
        houthr = int(int(m) / 30.0)
        min_len = int(int(m) / 30.0)
        max_gap = int(int(m) / 30.0)
        dst = roberts(src_down)
        _, dst = cv2.threshold(dst, robthr, 255, cv2.THRESH_BINARY)
        lab0, cnt0 = connect(dst)
        for k in range(1, len(cnt0)):
            if cnt0[k] < weak_tex_num:
                continue
            inside = lab0 == k
            border = np.zeros_like(inside)
            border[:, 1:] |= inside[:, :-1]
            border[:, :-1] |= inside[:, 1:]
            border[1:, :] |= inside[:-1, :]
            border[:-1, :] |= inside[1:, :]
            img_weak = np.where(border & ~inside, 255, 0).astype(np.uint8)
            lines = cv2.HoughLinesP(img_weak, 1, math.pi / 180, houthr, minLineLength=min_len, maxLineGap=max_gap)
            if lines is not None:
                for ln in lines[:, 0, :]:
                    cv2.line(dst, (int(ln[0]), int(ln[1])), (int(ln[2]), int(ln[3])), 255, 1)
    else:
        hist = np.bincount(src.ravel(), minlength=256)
        half = rows * cols // 2
        median = -1
        acc = 0
        for i in range(255):
            acc += hist[i]
            if acc > half:
                median = i
                break
        # `const float sigma = 0.67; int threshold1 = (1 - sigma) * median_val;` in float (the double
        # form truncates 32.99999 to 32 at median 100, and 65 at 200)
        t1 = int(np.float32(np.float32(1.0) - np.float32(0.67)) * np.float32(median))
        t2 = median
        dst = cv2.Canny(src, t1, t2, apertureSize=3, L2gradient=True)
    if mode == 0:
        dst = cv2.resize(dst, (cols, rows), interpolation=cv2.INTER_LINEAR)
    else:
        f = 1.0 / float(1 << scale)
        dst = cv2.resize(dst, (int(round(cols * f)), int(round(rows * f))), interpolation=cv2.INTER_LINEAR)
    _, dst = cv2.threshold(dst, robthr, 255, cv2.THRESH_BINARY)
    dst = np.ascontiguousarray(dst)
    _border_fix(dst)
    if mode == 0:
        return dst
    lab, cnt = connect(dst)
    small = (cnt <= weak_tex_num)
    small[0] = False
    lab = lab.copy()
    lab[small[lab]] = -1
    return np.ascontiguousarray(lab.astype(np.int32))


def level_inputs(gray_full: np.ndarray, scale_size: int, high_res_img: bool = True):
    """Edge map and label map of one view at one pyramid scale (GetProblemEdges, main.cpp:166-221)."""
    _need_cv2()
    scale = 0
    while (1 << scale) < scale_size:
        scale += 1
    rows, cols = gray_full.shape
    f = 1.0 / float(scale_size)
    new_cols, new_rows = int(round(cols * f)), int(round(rows * f))
    scaled = cv2.resize(gray_full.astype(np.float32), (new_cols, new_rows), interpolation=cv2.INTER_LINEAR)
    scaled_u8 = np.clip(np.round(scaled), 0, 255).astype(np.uint8)  # convertTo(CV_8UC1)
    edge = edge_segment(scale, scaled_u8, 0, True, high_res_img)
    label = edge_segment(scale, gray_full, 1, False, high_res_img)
    return edge, label
