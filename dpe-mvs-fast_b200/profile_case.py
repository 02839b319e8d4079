"""A small whole-schedule run for kernel profilers (ncu): one seeded synthetic scene, device-resident
inputs, `--repeat` complete schedules (PatchMatch pyramid + fusion) through dpe_scene_run.

    python dpe-mvs-fast_b200/profile_case.py [--scene c2_small] [--levels 2] [--iters 3] [--repeat 2]
                                             [--stats] [--staging 0|1|2] [--gn]

The default scene is the 10-view benchmark layout at 400x300, small enough that a multi-pass
capture of one launch restores little device memory.  Prints one line with the schedule's device
time and the number of library kernel launches per schedule; --stats adds the device time of each
kernel class over the last schedule (event pairs around every launch).
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--scene", default="c2_small")
    ap.add_argument("--levels", type=int, default=2)
    ap.add_argument("--iters", type=int, default=3)
    ap.add_argument("--refine-calls", type=int, default=1)
    ap.add_argument("--repeat", type=int, default=2)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--stats", action="store_true")
    ap.add_argument("--staging", type=int, default=0)
    ap.add_argument("--gn", action="store_true")
    args = ap.parse_args(argv)

    import torch

    import dpe_b200 as D
    import edges as E
    import scene as S

    sc = S.make_scene(args.scene, seed=args.seed, device="cuda")
    V = sc.n
    L = args.levels
    edges_d, labels_d = [], []
    for v in range(V):
        ev, lv = zip(*[E.level_inputs(sc.gray[v], 1 << (L - 1 - lvl)) for lvl in range(L)])
        edges_d.append([torch.from_numpy(np.ascontiguousarray(e)).cuda() for e in ev])
        labels_d.append([torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in lv])
    gray_d = [torch.from_numpy(np.ascontiguousarray(sc.gray[v])).cuda() for v in range(V)]
    bgr_d = [torch.from_numpy(np.ascontiguousarray(sc.bgr[v])).cuda() for v in range(V)]
    cams = [S.camera_struct(sc, v) for v in range(V)]
    ctx = D.Context(0)
    ctx.set_options(staging=args.staging, gn_refine=1 if args.gn else 0)
    lib = D.load_library()
    for r in range(args.repeat):
        if args.stats and r == args.repeat - 1:
            ctx.reset_kernel_stats()
            ctx.set_profiling(True)
        n0 = lib.dpe_launch_count()
        res = ctx.scene_run(gray_d, bgr_d, cams, sc.pairs, edges_d, labels_d, num_levels=L,
                            refine_calls=args.refine_calls, max_iterations=args.iters, fuse_mode=D.FUSE_FP64,
                            seed=7, memory=D.MEM_DEVICE, want_maps=False)
        print(f"schedule {r}: {args.scene} {V} views, {L} levels: {res['gpu_ms']:.1f} ms, {res['points']} points, "
              f"{lib.dpe_launch_count() - n0} launches", flush=True)
    if args.stats:
        for name, st in sorted(ctx.kernel_stats().items(), key=lambda kv: -kv[1]["ms"]):
            print(f"  {name:24s} {st['launches']:6d} launches {st['ms']:10.2f} ms")
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
