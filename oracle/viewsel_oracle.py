"""CPU restatement of the reference's pair score (calc_score, colmap2mvsnet.py:280-302).

TEST INFRASTRUCTURE ONLY: the checker for the GPU view scores (dpe_view_scores).  Pinned to the
reference itself: tests/golden/viewsel_ring.npz holds the pair.txt that the reference's own
processing_single_scene wrote for the same model (tests/golden/make_viewsel_golden.py).
"""
from __future__ import annotations

import numpy as np


def pair_score(ids_i: np.ndarray, ids_j: np.ndarray, center_i, center_j, xyz_of) -> float:
    """Score of images i < j: image i's observations whose point image j also observes (duplicates
    count), 0 when the 75th-percentile triangulation angle is below 1 degree."""
    present = set(int(x) for x in ids_j)
    score = 0
    angles = []
    for pid in ids_i:
        pid = int(pid)
        if pid not in present or pid == -1:
            continue
        p = xyz_of(pid)
        a, b = center_i - p, center_j - p
        angles.append((180 / np.pi) * np.arccos(np.dot(a, b) / np.linalg.norm(a) / np.linalg.norm(b)))
        score += 1
    if angles and sorted(angles)[int(len(angles) * 0.75)] < 1:
        return 0.0
    return float(score)


def score_matrix(obs: list, centers: np.ndarray, xyz_of) -> np.ndarray:
    n = len(obs)
    s = np.zeros((n, n))
    for i in range(n):
        for j in range(i + 1, n):
            s[i, j] = s[j, i] = pair_score(obs[i], obs[j], centers[i], centers[j], xyz_of)
    return s
