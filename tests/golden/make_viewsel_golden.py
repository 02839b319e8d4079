"""Golden fixture of the reference's view selection (tests/golden/viewsel_ring.npz).

Writes a small synthetic COLMAP text model (12 cameras on a ring around random surface points and a
twin of camera 0 a few centimetres away, with
observations of points outside the image dropped, some observations without a 3D point and a few
listed twice) and tiny images, runs the reference's own colmap2mvsnet.processing_single_scene on it
(imported from the reference tree, which must be present), and stores the model's arrays together
with the pair.txt the reference wrote.  The test (tests/test_viewsel.py) rebuilds pair.txt from the
same arrays with this repository's code and compares the text.

    python tests/golden/make_viewsel_golden.py [/path/to/reference]
"""
from __future__ import annotations

import argparse
import importlib.util
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def rotmat_look_at(center, target):
    z = target - center
    z = z / np.linalg.norm(z)
    x = np.cross(np.array([0.0, -1.0, 0.0]), z)
    x = x / np.linalg.norm(x)
    y = np.cross(z, x)
    return np.stack([x, y, z])  # world -> camera rows


def rotmat_to_qvec(R):
    """Unit quaternion (w, x, y, z) of a rotation matrix (Shepperd's method)."""
    t = np.trace(R)
    if t > 0:
        s = 2.0 * np.sqrt(t + 1.0)
        q = [0.25 * s, (R[2, 1] - R[1, 2]) / s, (R[0, 2] - R[2, 0]) / s, (R[1, 0] - R[0, 1]) / s]
    else:
        i = int(np.argmax(np.diag(R)))
        j, k = (i + 1) % 3, (i + 2) % 3
        s = 2.0 * np.sqrt(1.0 + R[i, i] - R[j, j] - R[k, k])
        q = [0.0] * 4
        q[0] = (R[k, j] - R[j, k]) / s
        q[1 + i] = 0.25 * s
        q[1 + j] = (R[j, i] + R[i, j]) / s
        q[1 + k] = (R[k, i] + R[i, k]) / s
    q = np.array(q)
    return q if q[0] >= 0 else -q


def synthetic_model(seed: int = 3, n_cams: int = 12, n_points: int = 1500, width: int = 64, height: int = 48):
    rng = np.random.default_rng(seed)
    f, cx, cy = 60.0, width / 2.0, height / 2.0
    pts = rng.uniform(-0.6, 0.6, (n_points, 3)) * np.array([1.0, 0.6, 1.0])
    point_ids = rng.choice(np.arange(1, 10 * n_points), n_points, replace=False)  # COLMAP ids are sparse
    cams = []
    centers = [np.array([3.0 * np.sin(a), 0.2 * np.cos(3 * a), -3.0 * np.cos(a)])
               for a in (2 * np.pi * c / n_cams for c in range(n_cams))]
    # a twin of camera 0 a few centimetres away: its pairs with camera 0 triangulate below 1 degree,
    # which the reference scores 0
    centers.append(centers[0] + np.array([0.03, 0.01, 0.0]))
    for c, center in enumerate(centers):
        R = rotmat_look_at(center, np.zeros(3))
        t = -R @ center
        Xc = pts @ R.T + t
        u = f * Xc[:, 0] / Xc[:, 2] + cx
        v = f * Xc[:, 1] / Xc[:, 2] + cy
        vis = (Xc[:, 2] > 0) & (u >= 0) & (u < width) & (v >= 0) & (v < height) & (rng.random(n_points) < 0.8)
        idx = np.nonzero(vis)[0]
        ids = list(point_ids[idx])
        xys = [(float(u[k]), float(v[k])) for k in idx]
        # observations without a 3D point, and a few points observed twice
        for _ in range(20):
            ids.append(-1)
            xys.append((float(rng.uniform(0, width)), float(rng.uniform(0, height))))
        for k in idx[:5]:
            ids.append(int(point_ids[k]))
            xys.append((float(u[k]) + 0.25, float(v[k])))
        order = rng.permutation(len(ids))
        cams.append(dict(qvec=rotmat_to_qvec(R), tvec=t, ids=np.array(ids, np.int64)[order],
                         xys=np.array(xys)[order]))
    return dict(f=f, cx=cx, cy=cy, width=width, height=height, points=pts, point_ids=point_ids, cams=cams)


def write_colmap_text(model, dense):
    mdir = os.path.join(dense, "dslr_calibration_undistorted")
    idir = os.path.join(dense, "images")
    os.makedirs(mdir)
    os.makedirs(idir)
    with open(os.path.join(mdir, "cameras.txt"), "w") as fh:
        fh.write(f"1 PINHOLE {model['width']} {model['height']} {model['f']!r} {model['f']!r} {model['cx']!r} "
                 f"{model['cy']!r}\n")
    with open(os.path.join(mdir, "images.txt"), "w") as fh:
        for i, c in enumerate(model["cams"]):
            q, t = c["qvec"], c["tvec"]
            q, t = [float(x) for x in q], [float(x) for x in t]
            fh.write(f"{i + 1} {q[0]!r} {q[1]!r} {q[2]!r} {q[3]!r} {t[0]!r} {t[1]!r} {t[2]!r} 1 img{i:03d}.png\n")
            fh.write(" ".join(f"{float(x)!r} {float(y)!r} {int(p)}" for (x, y), p in zip(c["xys"], c["ids"])) + "\n")
    with open(os.path.join(mdir, "points3D.txt"), "w") as fh:
        for k, (pid, X) in enumerate(zip(model["point_ids"], model["points"])):
            fh.write(f"{int(pid)} {float(X[0])!r} {float(X[1])!r} {float(X[2])!r} 128 128 128 0.5 1 0\n")
    import cv2

    for i in range(len(model["cams"])):
        cv2.imwrite(os.path.join(idir, f"img{i:03d}.png"), np.full((model["height"], model["width"], 3), 100, np.uint8))


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("reference", nargs="?", default="/root/reference")
    args = ap.parse_args()
    spec = importlib.util.spec_from_file_location("colmap2mvsnet", os.path.join(args.reference, "colmap2mvsnet.py"))
    ref = importlib.util.module_from_spec(spec)
    sys.modules["colmap2mvsnet"] = ref  # its worker pool pickles calc_score by module name
    spec.loader.exec_module(ref)
    model = synthetic_model()
    with tempfile.TemporaryDirectory() as tmp:
        dense, save = os.path.join(tmp, "dense"), os.path.join(tmp, "out")
        write_colmap_text(model, dense)
        os.makedirs(save)
        ns = argparse.Namespace(dense_folder=dense, save_folder=save, max_d=192, interval_scale=1.0, scale_factor=1.0,
                                theta0=5.0, sigma1=1.0, sigma2=10.0, model_ext=".txt")
        ref.processing_single_scene(ns)
        pair_txt = open(os.path.join(save, "pair.txt")).read()
        # the model as the reference parsed it: per image (sorted by image id) its point3D_ids and
        # extrinsic, per point id its xyz
        _, images, points3d = ref.read_model(os.path.join(dense, "dslr_calibration_undistorted"), ".txt")
    order = sorted(images.keys())
    obs = [np.asarray(images[k].point3D_ids, np.int64) for k in order]
    qvecs = np.stack([np.asarray(images[k].qvec, np.float64) for k in order])
    tvecs = np.stack([np.asarray(images[k].tvec, np.float64) for k in order])
    pid = np.array(sorted(points3d.keys()), np.int64)
    xyz = np.stack([points3d[p].xyz for p in pid])
    rot = np.stack([ref.qvec2rotmat(q) for q in qvecs])
    out = os.path.join(HERE, "viewsel_ring.npz")
    np.savez_compressed(out, obs_offsets=np.cumsum([0] + [len(o) for o in obs]), obs_ids=np.concatenate(obs),
                        qvecs=qvecs, tvecs=tvecs, rotmats=rot, point_ids=pid, point_xyz=xyz,
                        pair_txt=np.array(pair_txt))
    print(out, os.path.getsize(out), "bytes;", pair_txt.count("\n"), "lines of pair.txt")
    return 0


if __name__ == "__main__":
    sys.exit(main())
