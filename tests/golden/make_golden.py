"""Generate the golden fixtures of tests/golden/ from the CPU oracle.

    python tests/golden/make_golden.py

Each fixture holds its complete inputs (images, cameras, parameters, queries, prior state) and the
oracle's outputs, so the tests rebuild every call from the file alone.  The reference itself has
no tests or known-answer vectors for this path, so these freeze the oracle's restatement: the CPU
tests check that the oracle still reproduces them bit for bit, the GPU tests check the kernels
against them with the parity bars.

Fixtures:
  ncc_small.npz        2,000 strong-NCC queries (near and far hypotheses) on the 160x120 4-view
                       scene, float and FP64 costs
  pm_tiny.npz          FIRST_INIT call, then a REFINE_ITER call with APD, edges, labels and the
                       geometric term, on the 64x48 3-view scene
  fusion_tiny.npz      fusion of noisy ground-truth depth maps, FP64 and float modes
  fusion_tat_tiny.npz  both TAT fusion rules, FP64 and float modes, on the 64x48 3-view scene with
                       depth holes, a source band without depth and a block mask
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "dpe-mvs-fast_b200"), os.path.join(ROOT, "oracle"), os.path.dirname(HERE)):
    if p not in sys.path:
        sys.path.insert(0, p)

import dpe_b200 as D  # noqa: E402
import helpers as h  # noqa: E402
import oracle_py as O  # noqa: E402
import scene as S  # noqa: E402

CAM_KEYS = ("K", "R", "t", "c", "width", "height", "depth_min", "depth_max")


def params_to_json(p) -> str:
    return json.dumps({name: (float(getattr(p, name)) if isinstance(getattr(p, name), float) else int(getattr(p, name)))
                       for name, _ in p._fields_})


def params_from_json(s: str):
    p = D.Params()
    for k, v in json.loads(str(s)).items():
        setattr(p, k, v)
    return p


def cams_to_array(cams) -> np.ndarray:
    """Cameras as one float64 row each: K(9) R(9) t(3) c(3) width height depth_min depth_max."""
    rows = []
    for c in cams:
        rows.append(np.concatenate([np.asarray(c[k], np.float64).reshape(-1) for k in CAM_KEYS]))
    return np.stack(rows)


def cams_from_array(a: np.ndarray):
    out = []
    for r in a:
        out.append(dict(K=r[0:9].astype(np.float32), R=r[9:18].astype(np.float32), t=r[18:21].astype(np.float32),
                        c=r[21:24].astype(np.float32), width=int(r[24]), height=int(r[25]),
                        depth_min=np.float32(r[26]), depth_max=np.float32(r[27])))
    return out


def make_ncc(path: str) -> None:
    from test_oracle import _random_queries

    sc = S.make_scene("small", seed=1)
    images = [np.ascontiguousarray(g.astype(np.float32)) for g in sc.gray]
    cams = [S.camera_struct(sc, i) for i in range(sc.n)]
    p = D.default_params()
    rng = np.random.default_rng(2024)
    a = _random_queries(sc, 1000, rng)
    b = _random_queries(sc, 1000, rng, near_gt=False)
    px, py, src, planes = (np.concatenate([x, y]) for x, y in zip(a, b))
    f32 = O.ncc_strong(images, cams, p, px, py, src, planes, fp64=False)
    f64 = O.ncc_strong(images, cams, p, px, py, src, planes, fp64=True)
    np.savez_compressed(path, gray=np.stack([g.astype(np.uint8) for g in sc.gray]), cams=cams_to_array(cams),
                        params=params_to_json(p), px=px.astype(np.int32), py=py.astype(np.int32),
                        src=src.astype(np.int32), planes=planes.astype(np.float32), cost_f32=f32, cost_f64=f64)


def make_pm(path: str) -> None:
    sc = S.make_scene("tiny", seed=4)
    ref = 1
    images, cams, srcs = h.view_inputs(sc, ref)
    ids = [ref] + list(srcs)
    p0 = h.first_init_params(sc, len(images))
    o0 = O.pm_run(images, cams, p0, seed=4242)
    state, weak = h.post_process(o0["plane"], o0["weak"], p0.depth_min, p0.depth_max)
    edge, low, label = h.synthetic_edges(sc.gray[ref], edge_fraction=0.1)
    depths = [np.ascontiguousarray(sc.depth[i].astype(np.float32)) for i in ids]
    p1 = h.refine_params(sc, len(images), level=1, state=D.REFINE_ITER, geom=True, j=0)
    views = np.ascontiguousarray(o0["views"])
    o1 = O.pm_run(images, cams, p1, plane_in=state, views_in=views, weak_in=weak, edge=edge, edge_low=low,
                  label=label, depths=depths, seed=4343)
    np.savez_compressed(path, gray=np.stack([g.astype(np.uint8) for g in sc.gray[ids]]), cams=cams_to_array(cams),
                        params0=params_to_json(p0), seed0=np.uint64(4242), plane0=o0["plane"], weak0=o0["weak"],
                        views0=o0["views"], cost0=o0["costs"],
                        params1=params_to_json(p1), seed1=np.uint64(4343), state_in=state, weak_in=weak,
                        edge=edge, edge_low=low, label=label, depths=np.stack(depths),
                        plane1=o1["plane"], weak1=o1["weak"], views1=o1["views"], cost1=o1["costs"])


def make_fusion(path: str) -> None:
    from test_oracle import _gt_fusion_views

    sc = S.make_scene("tiny", seed=5)
    views = _gt_fusion_views(sc, noise=0.002, seed=9)
    f64 = O.fuse(views, D.FUSE_FP64)
    f32 = O.fuse(views, D.FUSE_FLOAT)
    m2 = O.fuse(views, D.FUSE_FP64, min_consistent=2)
    out = dict(depth=np.stack([v["depth"] for v in views]), normal=np.stack([v["normal"] for v in views]),
               weak=np.stack([v["weak"] for v in views]), bgr=np.stack([v["bgr"] for v in views]),
               cams=cams_to_array([v["camera"] for v in views]), src=np.array([v["src"] for v in views], np.int32))
    for tag, r in (("fp64", f64), ("float", f32), ("fp64_min2", m2)):
        for k in ("xyz", "bgr", "origin", "num_consistent"):
            out[f"{tag}_{k}"] = r[k]
        out[f"{tag}_count"] = np.int64(r["count"])
    np.savez_compressed(path, **out)


def make_fusion_tat(path: str) -> None:
    from test_fusion_tat import tat_views

    sc = S.make_scene("tiny", seed=5)
    views = tat_views(sc, noise=2e-4, seed=19)
    out = dict(depth=np.stack([v["depth"] for v in views]), normal=np.stack([v["normal"] for v in views]),
               bgr=np.stack([v["bgr"] for v in views]), cams=cams_to_array([v["camera"] for v in views]),
               src=np.array([v["src"] for v in views], np.int32),
               has_block=np.array([v["block"] is not None for v in views]),
               block=np.stack([v["block"] if v["block"] is not None else np.full(v["depth"].shape, 255, np.uint8)
                               for v in views]))
    for vname, variant in (("inter", D.TAT_INTERMEDIATE), ("adv", D.TAT_ADVANCED)):
        for mname, mode in (("fp64", D.FUSE_FP64), ("float", D.FUSE_FLOAT)):
            r = O.fuse_tat(views, variant, mode)
            tag = f"{vname}_{mname}"
            for k in ("xyz", "bgr", "origin", "num_consistent"):
                out[f"{tag}_{k}"] = r[k]
            out[f"{tag}_count"] = np.int64(r["count"])
    np.savez_compressed(path, **out)


def fusion_tat_views_from(z) -> list:
    cams = cams_from_array(z["cams"])
    return [dict(depth=np.ascontiguousarray(z["depth"][v]), normal=np.ascontiguousarray(z["normal"][v]),
                 bgr=np.ascontiguousarray(z["bgr"][v]), camera=cams[v], src=[int(s) for s in z["src"][v]],
                 block=np.ascontiguousarray(z["block"][v]) if z["has_block"][v] else None) for v in range(len(cams))]


def fusion_views_from(z) -> list:
    cams = cams_from_array(z["cams"])
    return [dict(depth=np.ascontiguousarray(z["depth"][v]), normal=np.ascontiguousarray(z["normal"][v]),
                 weak=np.ascontiguousarray(z["weak"][v]), bgr=np.ascontiguousarray(z["bgr"][v]), camera=cams[v],
                 src=[int(s) for s in z["src"][v]]) for v in range(len(cams))]


def main() -> int:
    O.build()
    make_ncc(os.path.join(HERE, "ncc_small.npz"))
    make_pm(os.path.join(HERE, "pm_tiny.npz"))
    make_fusion(os.path.join(HERE, "fusion_tiny.npz"))
    make_fusion_tat(os.path.join(HERE, "fusion_tat_tiny.npz"))
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")
    return 0


if __name__ == "__main__":
    sys.exit(main())
