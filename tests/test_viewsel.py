"""View selection (pair.txt) against the reference's own output: tests/golden/viewsel_ring.npz holds a
13-camera sparse model and the pair.txt that the reference's processing_single_scene wrote for it
(tests/golden/make_viewsel_golden.py).  CPU: the score restatement plus this repository's ranking and
writer give the same text.  GPU: dpe_view_scores gives the same scores, so the same text."""
import os

import numpy as np
import pytest

import viewsel as VS
import viewsel_oracle as VO

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "viewsel_ring.npz")


def _model():
    z = np.load(GOLDEN)
    off = z["obs_offsets"]
    obs = [z["obs_ids"][off[i]:off[i + 1]] for i in range(len(off) - 1)]
    return z, obs


def test_oracle_scores_reproduce_reference_pair_txt():
    z, obs = _model()
    centers = VS.camera_centers(z["rotmats"], z["tvecs"])
    xyz = {int(p): x for p, x in zip(z["point_ids"], z["point_xyz"])}
    scores = VO.score_matrix(obs, centers, xyz.__getitem__)
    assert (scores == 0).sum() > len(obs)  # the twin cameras' pair triangulates below 1 degree
    assert VS.pair_txt(VS.select_views(scores)) == str(z["pair_txt"])


def test_dense_model_layout():
    z, obs = _model()
    off, dense, xyz = VS.dense_model(obs, z["point_ids"], z["point_xyz"])
    assert off[-1] == len(dense) and (dense >= -1).all() and dense.max() < len(xyz)
    k = int(np.nonzero(dense >= 0)[0][0])
    assert z["point_ids"][dense[k]] == z["obs_ids"][k]


@pytest.mark.gpu
def test_gpu_scores_equal_reference(ctx):
    z, obs = _model()
    scores, text = VS.view_selection(ctx, obs, z["point_ids"], z["point_xyz"], z["rotmats"], z["tvecs"])
    centers = VS.camera_centers(z["rotmats"], z["tvecs"])
    xyz = {int(p): x for p, x in zip(z["point_ids"], z["point_xyz"])}
    assert np.array_equal(scores, VO.score_matrix(obs, centers, xyz.__getitem__))
    assert text == str(z["pair_txt"])


@pytest.mark.gpu
def test_gpu_scores_large_ring(ctx):
    """A 60-camera ring with 200k points (tracks of ~10-30 views): GPU scores against the restatement
    on a sample of pairs."""
    rng = np.random.default_rng(5)
    n_cams, n_pts = 60, 200_000
    pts = rng.uniform(-1, 1, (n_pts, 3))
    ang = 2 * np.pi * np.arange(n_cams) / n_cams
    centers = np.stack([4 * np.sin(ang), 0.3 * np.cos(2 * ang), -4 * np.cos(ang)], 1)
    obs = []
    for c in range(n_cams):
        d = pts - centers[c]
        facing = (d @ -centers[c]) / np.linalg.norm(d, axis=1) / np.linalg.norm(centers[c]) > 0.97
        ids = np.nonzero(facing & (rng.random(n_pts) < 0.7))[0].astype(np.int64)
        ids = np.concatenate([ids, -np.ones(50, np.int64), ids[:7]])
        obs.append(rng.permutation(ids))
    off = np.zeros(n_cams + 1, np.int64)
    off[1:] = np.cumsum([len(o) for o in obs])
    g = ctx.view_scores(centers, off, np.concatenate(obs).astype(np.int32), pts)
    assert np.array_equal(g, g.T)
    for i, j in [(0, 1), (0, 5), (10, 11), (3, 40), (59, 0)]:
        a, b = min(i, j), max(i, j)
        want = VO.pair_score(obs[a], obs[b], centers[a], centers[b], lambda p: pts[p])
        assert g[a, b] == want, (a, b, g[a, b], want)
