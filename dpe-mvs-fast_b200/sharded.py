"""View-sharded schedule over several processes (one per GPU).

Within one call of the reference's schedule (main.cpp:390-457) every reference view is
independent of the others given the source views' depth maps, so the views of a call can be
spread over ranks.  The exchange is one all-gather per call: each rank publishes the state it
computed for its views (plane = world normal + depth, pixel state, selected views), and every rank
then holds every view's state for the next call's geometric-consistency term.  Fusion, whose masks
make it order-dependent across views (DPE.cpp:1460-1540), runs on rank 0 after the last call.

The reference runs views one after another inside a call, each reading the depths its predecessors
just wrote (Gauss-Seidel); sharded, every view reads the previous call's depths (Jacobi), the order
of dpe_schedule::batch_views.  So the sharded result equals the single-process Jacobi schedule on
the same seeds, bit for bit, which tests/test_sharded.py checks with `gloo` ranks on the CPU.

Views go to ranks largest first, each to the rank with the fewest pixels so far (ties: lowest
rank), which balances uneven resolutions.  This module covers one pyramid level (a FIRST_INIT call
and `refine_calls` geometric REFINE_ITER calls); the per-view work is a caller-supplied function,
`dpe_b200.Context.pm_run` on a GPU.
"""
from __future__ import annotations

from typing import Callable, Dict, List, Sequence

import numpy as np


def assign_views(pixels: Sequence[int], world: int) -> List[List[int]]:
    """Views per rank: largest first, each to the least-loaded rank (ties: lowest rank)."""
    load = [0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for v in sorted(range(len(pixels)), key=lambda v: (-pixels[v], v)):
        r = min(range(world), key=lambda r: (load[r], r))
        out[r].append(v)
        load[r] += pixels[v]
    for lst in out:
        lst.sort()
    return out


def _pack(states: Dict[int, Dict], views: List[int], slots: int, H: int, W: int):
    import torch

    plane = torch.zeros((slots, H, W, 4), dtype=torch.float32)
    weak = torch.zeros((slots, H, W), dtype=torch.uint8)
    sel = torch.zeros((slots, H, W), dtype=torch.int32)
    for k, v in enumerate(views):
        plane[k] = torch.from_numpy(states[v]["plane"])
        weak[k] = torch.from_numpy(states[v]["weak"])
        sel[k] = torch.from_numpy(states[v]["views"].view(np.int32))
    return plane, weak, sel


def all_gather_states(local: Dict[int, Dict], owners: List[List[int]], H: int, W: int, group=None,
                      device: str = "cpu") -> Dict[int, Dict]:
    """Every rank's view states to every rank: one all-gather per array (slots = the largest
    number of views a rank owns)."""
    import torch
    import torch.distributed as dist

    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    slots = max(len(o) for o in owners)
    mine = _pack(local, owners[rank], slots, H, W)
    out: Dict[int, Dict] = {}
    gathered = []
    for t in mine:
        t = t.to(device)
        parts = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(parts, t, group=group)
        gathered.append([p.cpu() for p in parts])
    for r in range(world):
        for k, v in enumerate(owners[r]):
            out[v] = dict(plane=gathered[0][r][k].numpy().copy(), weak=gathered[1][r][k].numpy().copy(),
                          views=gathered[2][r][k].numpy().view(np.uint32).copy())
    return out


def post_process(plane: np.ndarray, weak: np.ndarray, dmin: float, dmax: float):
    """ProcessProblem's result assembly (main.cpp:266-279): out-of-range depths -> 0 and UNKNOWN."""
    depth = plane[..., 3].copy()
    weak = weak.copy()
    bad = (depth < dmin) | (depth > dmax)
    depth[bad] = 0.0
    weak[bad] = 2
    return np.ascontiguousarray(np.concatenate([plane[..., :3], depth[..., None]], -1).astype(np.float32)), \
        np.ascontiguousarray(weak)


def run_level(call: Callable, sources: Sequence[Sequence[int]], pixels: Sequence[int], depth_range: Callable,
              H: int, W: int, refine_calls: int = 1, group=None, device: str = "cpu") -> Dict[int, Dict]:
    """One pyramid level of the schedule, views sharded over the ranks of `group` (None: the default
    group; without an initialised process group, one process does every view).

    call(v, c, **kw) runs view v's call c (0: FIRST_INIT; 1..refine_calls: geometric REFINE_ITER,
    given plane_in / views_in / weak_in / depths) and returns dict(plane, weak, views);
    depth_range(v) is view v's (depth_min, depth_max) for ProcessProblem's result assembly.
    Returns every view's post-processed state (plane with depth, weak, views) after the last call,
    on every rank."""
    import torch.distributed as dist

    distributed = dist.is_available() and dist.is_initialized()
    rank = dist.get_rank(group) if distributed else 0
    world = dist.get_world_size(group) if distributed else 1
    owners = assign_views(pixels, world)
    states: Dict[int, Dict] = {}
    for c in range(1 + refine_calls):
        local = {}
        for v in owners[rank]:
            kw = {}
            if c > 0:
                kw = dict(plane_in=states[v]["plane"], views_in=states[v]["views"], weak_in=states[v]["weak"],
                          depths=[np.ascontiguousarray(states[u]["plane"][..., 3]) for u in [v] + list(sources[v])])
            o = call(v, c, **kw)
            dmin, dmax = depth_range(v)
            plane, weak = post_process(o["plane"], o["weak"], dmin, dmax)
            local[v] = dict(plane=plane, weak=weak, views=np.ascontiguousarray(o["views"]))
        states = all_gather_states(local, owners, H, W, group=group, device=device) if distributed else local
    return states
