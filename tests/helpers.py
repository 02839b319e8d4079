"""Shared helpers of the test-suite: scene -> per-view problem inputs, comparison metrics."""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "dpe-mvs-fast_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

import dpe_b200 as D  # noqa: E402
import scene as S  # noqa: E402


def view_inputs(scene, ref: int, n_src: int | None = None):
    """Images (float32 gray), cameras and source ids of one reference view at full resolution."""
    srcs = scene.pairs[ref][: (n_src if n_src is not None else len(scene.pairs[ref]))]
    ids = [ref] + list(srcs)
    images = [np.ascontiguousarray(scene.gray[i].astype(np.float32)) for i in ids]
    cams = [S.camera_struct(scene, i) for i in ids]
    return images, cams, srcs


def first_init_params(scene, n_images: int, iters: int = 3):
    """Level-0 call of the reference schedule (main.cpp:398-420): FIRST_INIT, no APD/edge, geom off."""
    p = D.default_params()
    p.num_images = n_images
    p.state = D.FIRST_INIT
    p.use_APD = 0
    p.use_edge = 0
    p.use_limit = 0
    p.use_label = 0
    p.geom_consistency = 0
    p.max_iterations = iters
    p.weak_peak_radius = 6
    # DPE::InuputInitialization (DPE.cpp:953-954)
    p.depth_min = np.float32(scene.spec.depth_min) * np.float32(0.6)
    p.depth_max = np.float32(scene.spec.depth_max) * np.float32(1.2)
    return p


def synthetic_edges(gray: np.ndarray, edge_fraction: float = 0.08):
    """Simple stand-ins for the edge / label precompute (EdgeSegment, DPE.cpp:136-291): the
    strongest `edge_fraction` of gradient magnitudes as edges, and connected non-edge labels
    (0 on edges, -1 for small regions)."""
    from scipy import ndimage

    g = gray.astype(np.float32)
    gx = ndimage.sobel(g, axis=1)
    gy = ndimage.sobel(g, axis=0)
    mag = np.hypot(gx, gy)
    edge = (mag > np.quantile(mag, 1.0 - edge_fraction)).astype(np.uint8) * 255
    lab, n = ndimage.label(edge == 0)
    counts = np.bincount(lab.ravel())
    small = counts < 200
    label = lab.astype(np.int32)
    label[(small[lab]) & (lab > 0)] = -1
    low = edge[::4, ::4].copy()
    return np.ascontiguousarray(edge), np.ascontiguousarray(low), np.ascontiguousarray(label)


def post_process(plane: np.ndarray, weak: np.ndarray, dmin: float, dmax: float):
    """ProcessProblem's result assembly (main.cpp:266-279): out-of-range depths -> 0 and UNKNOWN."""
    depth = plane[..., 3].copy()
    weak = weak.copy()
    bad = (depth < dmin) | (depth > dmax)
    depth[bad] = 0.0
    weak[bad] = 2
    state = np.concatenate([plane[..., :3], depth[..., None]], -1).astype(np.float32)
    return np.ascontiguousarray(state), np.ascontiguousarray(weak)


def refine_params(scene, n_images: int, level: int, state: int, geom: bool, j: int = 0):
    """Calls of level >= 1 of the reference schedule (main.cpp:402-445)."""
    p = first_init_params(scene, n_images)
    p.state = state
    p.use_APD = 1
    p.use_edge = 1
    p.use_limit = 1
    p.use_label = 1
    p.use_radius = 1
    p.ransac_threshold = np.float32(0.01 - level * 0.00125)
    p.rotate_time = min(2 ** level, 4)
    p.geom_consistency = 1 if geom else 0
    p.weak_peak_radius = 6 if state == D.REFINE_INIT else max(4 - 2 * j, 2)
    return p


def rel_depth_agreement(d_a: np.ndarray, d_b: np.ndarray, tol: float = 1e-3) -> float:
    """Fraction of pixels whose depths agree within `tol` relative error."""
    a = d_a.astype(np.float64)
    b = d_b.astype(np.float64)
    ok = np.abs(a - b) <= tol * np.maximum(np.abs(b), 1e-12)
    return float(ok.mean())
