"""The view-sharded schedule (dpe-mvs-fast_b200/sharded.py) over two `gloo` ranks on the CPU: views
spread over the ranks, one all-gather of the view states per call, and the result equal bit for bit
to one process running the same (Jacobi-ordered) schedule.  The per-view calls are the CPU oracle's
here; on GPUs they are dpe_pm_run calls and the all-gather runs over NCCL."""
import os
import socket
import sys

import numpy as np
import pytest

import sharded as SH

HERE = os.path.dirname(os.path.abspath(__file__))


def test_assign_views_balances_pixels():
    px = [640 * 480] * 4 + [1600 * 1200] * 3 + [3200 * 2400]
    owners = SH.assign_views(px, 3)
    assert sorted(v for o in owners for v in o) == list(range(len(px)))
    loads = [sum(px[v] for v in o) for o in owners]
    # largest first to the least-loaded rank: no rank exceeds another by more than one view
    assert max(loads) - min(loads) <= max(px)
    assert loads[0] == 3200 * 2400  # the largest view alone
    assert SH.assign_views([5, 5, 5, 5], 2) == [[0, 2], [1, 3]]


def _level(scene_name: str):
    """The call function, sources, pixel counts and depth ranges of a one-level schedule (a FIRST_INIT
    call and one geometric REFINE_ITER call per view) on the oracle."""
    sys.path.insert(0, HERE)
    import dpe_b200 as D
    import helpers as h
    import oracle_py as O

    sc = h.S.make_scene(scene_name, seed=1)
    inputs = [h.view_inputs(sc, v) for v in range(sc.n)]

    def params(v, c):
        p = h.first_init_params(sc, len(inputs[v][0]))
        if c > 0:
            p.state = D.REFINE_ITER
            p.geom_consistency = 1
            p.weak_peak_radius = 4
        return p

    def call(v, c, **kw):
        images, cams, _ = inputs[v]
        return O.pm_run(images, cams, params(v, c), seed=1000 + 10 * c + v, threads=2, **kw)

    p0 = params(0, 0)
    H, W = sc.gray.shape[1:]
    return call, [inputs[v][2] for v in range(sc.n)], [W * H] * sc.n, (lambda v: (p0.depth_min, p0.depth_max)), H, W


def _worker(rank, world, port, out_path):
    for p in (HERE, os.path.join(HERE, "..", "dpe-mvs-fast_b200"), os.path.join(HERE, "..", "oracle")):
        sys.path.insert(0, p)
    import torch.distributed as dist
    import sharded

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        call, sources, pixels, drange, H, W = _level("tiny")
        states = sharded.run_level(call, sources, pixels, drange, H, W, refine_calls=1)
        if rank == 0:
            np.savez(out_path, **{f"{k}_{v}": states[v][k] for v in states for k in ("plane", "weak", "views")})
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_equal_one_process(tmp_path):
    import torch.multiprocessing as mp

    out = str(tmp_path / "rank0.npz")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    call, sources, pixels, drange, H, W = _level("tiny")
    one = SH.run_level(call, sources, pixels, drange, H, W, refine_calls=1)
    got = np.load(out)
    assert len(one) == 3
    for v in one:
        for k in ("plane", "weak", "views"):
            assert np.array_equal(got[f"{k}_{v}"], one[v][k], equal_nan=True), (v, k)
    # the geometric call used every view's depth: the result differs from a FIRST_INIT-only run
    assert (one[0]["plane"][..., 3] > 0).mean() > 0.5
