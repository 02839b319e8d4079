"""View selection: each reference view's source views and scores, as pair.txt lists them.

The reference computes them in colmap2mvsnet.py's processing_single_scene: one score per image pair
(calc_score, colmap2mvsnet.py:280-302; here dpe_view_scores on the GPU), then per view the
`min(20, N - 1)` highest-scoring images (colmap2mvsnet.py:405-419) written to pair.txt
(colmap2mvsnet.py:447-453).  The inputs are the sparse model as COLMAP's reader gives it: per image
(in image-id order) its rotation and translation and the 3D point id of each 2D observation (-1 for
none), and the xyz of every point id.
"""
from __future__ import annotations

from typing import Dict, List, Sequence, Tuple

import numpy as np


def camera_centers(rotmats: Sequence[np.ndarray], tvecs: Sequence[np.ndarray]) -> np.ndarray:
    """-R^T t per image, with the reference's expression (colmap2mvsnet.py:285-286)."""
    out = []
    for R, t in zip(rotmats, tvecs):
        e = np.zeros((4, 4))
        e[:3, :3] = R
        e[:3, 3] = t
        e[3, 3] = 1
        out.append(-np.matmul(e[:3, :3].transpose(), e[:3, 3:4])[:, 0])
    return np.stack(out)


def dense_model(obs_ids: Sequence[np.ndarray], point_ids: np.ndarray, point_xyz: np.ndarray):
    """Observation offsets, dense point index per observation (-1: none) and point coordinates."""
    index = {int(p): k for k, p in enumerate(point_ids)}
    offsets = np.zeros(len(obs_ids) + 1, np.int64)
    offsets[1:] = np.cumsum([len(o) for o in obs_ids])
    dense = np.array([index[int(p)] if p != -1 else -1 for o in obs_ids for p in o], np.int32)
    return offsets, dense, np.ascontiguousarray(point_xyz, np.float64)


def select_views(score: np.ndarray, num_view: int | None = None) -> List[List[Tuple[int, float]]]:
    """Per view the num_view (default min(20, N - 1)) best images, by np.argsort of the score row
    reversed, exactly as colmap2mvsnet.py:414-418 ranks them (ties in argsort's order)."""
    n = score.shape[0]
    k = min(20, n - 1) if num_view is None else num_view
    out = []
    for i in range(n):
        order = np.argsort(score[i])[::-1]
        out.append([(int(j), score[i, j]) for j in order[:k]])
    return out


def pair_txt(view_sel: List[List[Tuple[int, float]]]) -> str:
    """pair.txt text (colmap2mvsnet.py:447-453): the view count, then per view its index and
    `n id score ...` with integer scores."""
    lines = ["%d\n" % len(view_sel)]
    for i, sel in enumerate(view_sel):
        lines.append("%d\n%d " % (i, len(sel)))
        lines.append("".join("%d %d " % (j, s) for j, s in sel))
        lines.append("\n")
    return "".join(lines)


def view_selection(ctx, obs_ids, point_ids, point_xyz, rotmats, tvecs) -> Tuple[np.ndarray, str]:
    """Scores on the GPU and the pair.txt text they give."""
    offsets, dense, xyz = dense_model(obs_ids, point_ids, point_xyz)
    scores = ctx.view_scores(camera_centers(rotmats, tvecs), offsets, dense, xyz)
    return scores, pair_txt(select_views(scores))
