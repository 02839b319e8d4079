"""edge_oracle.py -- CPU restatement of EdgeSegment's edge map (DPE.cpp:136-250, mode 0 with
use_canny), as GetProblemEdges requests it (main.cpp:166-197).

TEST INFRASTRUCTURE ONLY: the checker for the device edge maps (dpe_edge_map and
dpe_schedule.device_edges).  Only tests/ may use it.

The reference calls OpenCV for this map: cv::Canny (apertureSize 3, L2gradient true) on the level
image converted to 8 bits, with thresholds from the image's median.  OpenCV is a third-party
dependency absent from the reference tree; its Canny is the published algorithm (Canny 1986) in
OpenCV's integer form, restated here:
  - 3x3 Sobel derivatives with a replicated border, squared L2 magnitude in integers, thresholds
    squared (each clamped to 32767 first, squared only when positive);
  - non-maximum suppression by gradient sector, chosen with the fixed-point tangent of 22.5
    degrees (round(tan(pi/8) * 2^15) = 13573): the magnitude must exceed the neighbour before the
    pixel and be >= the one after it along the sector (> both on the diagonals), with 0 outside
    the image;
  - hysteresis: the 8-connected components of the surviving pixels above the low threshold that
    contain a pixel above the high threshold.
PINNED against the dependency itself: tests/test_edges.py compares this restatement with cv2.Canny
(OpenCV 4.13.0 in this image, with and without its IPP path) bit for bit.
"""
from __future__ import annotations

import numpy as np

TG22 = 13573


def median_thresholds(img: np.ndarray):
    """(threshold1, threshold2) of EdgeSegment (DPE.cpp:193-219): the first gray value whose
    cumulative histogram exceeds half the pixels (values 0..254; -1 if none), then
    (1 - 0.67f) * median in float, truncated."""
    hist = np.bincount(img.ravel(), minlength=256)
    half = img.size // 2
    median, acc = -1, 0
    for i in range(255):
        acc += int(hist[i])
        if acc > half:
            median = i
            break
    t1 = int(np.float32(np.float32(1.0) - np.float32(0.67)) * np.float32(median))
    return t1, median


def canny_l2(img: np.ndarray, threshold1: float, threshold2: float) -> np.ndarray:
    """cv::Canny(img, edges, threshold1, threshold2, 3, true) for a uint8 image."""
    lo, hi = min(32767.0, float(threshold1)), min(32767.0, float(threshold2))
    if lo > 0:
        lo *= lo
    if hi > 0:
        hi *= hi
    if lo > hi:
        lo, hi = hi, lo
    low, high = int(np.floor(lo)), int(np.floor(hi))
    p = np.pad(img.astype(np.int64), 1, mode="edge")
    dx = (p[:-2, 2:] + 2 * p[1:-1, 2:] + p[2:, 2:]) - (p[:-2, :-2] + 2 * p[1:-1, :-2] + p[2:, :-2])
    dy = (p[2:, :-2] + 2 * p[2:, 1:-1] + p[2:, 2:]) - (p[:-2, :-2] + 2 * p[:-2, 1:-1] + p[:-2, 2:])
    mag = dx * dx + dy * dy
    mp = np.pad(mag, 1)  # 0 outside the image
    ax, ay = np.abs(dx), np.abs(dy) << 15
    tg22x = ax * TG22
    tg67x = tg22x + (ax << 16)
    left, right = mp[1:-1, :-2], mp[1:-1, 2:]
    up, down = mp[:-2, 1:-1], mp[2:, 1:-1]
    s_neg = (dx ^ dy) < 0
    diag_before = np.where(s_neg, mp[:-2, 2:], mp[:-2, :-2])   # row above, column x - s
    diag_after = np.where(s_neg, mp[2:, :-2], mp[2:, 2:])      # row below, column x + s
    horiz = ay < tg22x
    vert = ~horiz & (ay > tg67x)
    diag = ~horiz & ~vert
    keep = ((horiz & (mag > left) & (mag >= right)) | (vert & (mag > up) & (mag >= down)) |
            (diag & (mag > diag_before) & (mag > diag_after)))
    cand = keep & (mag > low)
    strong = cand & (mag > high)
    from scipy import ndimage

    lab, n = ndimage.label(cand, structure=np.ones((3, 3), bool))
    hit = np.zeros(n + 1, bool)
    hit[np.unique(lab[strong])] = True
    hit[0] = False
    return np.where(hit[lab], 255, 0).astype(np.uint8)


def border_rule(d: np.ndarray) -> np.ndarray:
    """DPE.cpp:239-250: rows first, then columns, each in statement order."""
    d = d.copy()
    rows, cols = d.shape
    if cols >= 2:
        for y in range(rows):
            if d[y, 1] == 0:
                d[y, 0] = 0
            if d[y, cols - 2] == 0:
                d[y, cols - 1] = 0
    if rows >= 2:
        for x in range(cols):
            if d[1, x] == 0:
                d[0, x] = 0
            if d[rows - 2, x] == 0:
                d[rows - 1, x] = 0
    return d


def edge_map(img: np.ndarray) -> np.ndarray:
    """EdgeSegment(scale, img, 0, true, high_res_img) for an 8-bit level image."""
    t1, t2 = median_thresholds(img)
    return border_rule(canny_l2(img, t1, t2))


def level_image_u8(level: np.ndarray) -> np.ndarray:
    """convertTo(CV_8UC1) of a float level image: round half to even, saturate (main.cpp:178)."""
    return np.clip(np.rint(level), 0, 255).astype(np.uint8)
