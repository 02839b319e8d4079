"""Benchmark: reference-view Mpix/s of the complete PatchMatch + fusion schedule on one B200.

Workload (the measured configuration): 10 views at 1600x1200 of a seeded synthetic scene (6 planes
+ 2 spheres, half the surface nearly textureless, sigma 3), a 3-level image pyramid with one
FIRST_INIT/REFINE_INIT call and one geom-consistency REFINE_ITER call per view and level (3
red/black iterations each, edge-aware and weak-texture propagation on levels >= 1), then fusion
with a 2-view consistency threshold.  ETH3D, on which the reference is run, is not available; the
synthetic scene stands in for it.

A step is one complete schedule over all views.  `value` is measured with the inputs resident in
device memory (CUDA events on the library's stream around the schedule); `e2e` runs the same
schedule through the public C-ABI entry point with pinned host buffers, including the uploads of
images / edge maps / label maps and the downloads of the depth, normal, state and view maps and
of the fused points.  The scene's working set (10 x 1600 x 1200 images, states and source views)
is far larger than the 126 MB L2, so no flush is needed between steps.

`--impl reference` times the reference's own DPE.cu / DPE.cpp compiled for the host CPU
(oracle/_ref/libref.so; its CUDA build reads past the ends of its device buffers and an
uninitialised radius array, so it is not run on the GPU),
on a bounded sample of the same schedule, on all host cores.

`--case` runs only device-resident schedules of a chosen scene (for profilers):
    python bench.py --case c2 --levels 2 --repeat 1 [--stats] [--staging 0|1|2] [--gn]
`--case c5` measures the batching forms on the 49-view ring workload (one JSON line).

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "dpe-mvs-fast_b200"))

METRIC = "ref-view Mpix/s"
UNIT = "Mpix/s"
STRONG_NCC_FLOP = 1176   # 36 taps x 32 FLOP + 24 finalize (per strong window evaluation)
WEAK_NCC_FLOP = 3672     # 108 taps x 32 FLOP + 9 x 24 finalize (per deformable evaluation)
WORKLOAD = dict(scene="c2", views=10, width=1600, height=1200, levels=3, refine_calls=1, max_iterations=3,
                min_consistent=2)
# the cost kernels the bench reports a roofline fraction for (FP32 issue bound)
COST_KERNELS = ("k_strong_update", "k_depth_to_weak", "k_weak_eval", "k_local_refine", "k_random_init",
                "k_weak_finish")
FUSION_KERNELS = ("k_fuse_entries", "k_fuse_rounds", "k_fuse_emit")
TRAFFIC_TABLE = os.path.join(ROOT, "profiles", "dram_bytes_per_launch.md")


def _env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def _prepare_scene(name: str, seed: int, device: str, levels: int):
    import scene as S
    import edges as E

    sc = S.make_scene(name, seed=seed, device=device)
    V = sc.n
    edges_l, labels_l = [], []
    for v in range(V):
        ev, lv = [], []
        for lvl in range(levels):
            e, lab = E.level_inputs(sc.gray[v], 1 << (levels - 1 - lvl))
            ev.append(np.ascontiguousarray(e))
            lv.append(np.ascontiguousarray(lab))
        edges_l.append(ev)
        labels_l.append(lv)
    cams = [S.camera_struct(sc, v) for v in range(V)]
    srcs = [sc.pairs[v] for v in range(V)]
    return sc, cams, srcs, edges_l, labels_l


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        fd, self.path = tempfile.mkstemp(prefix=f"dpe_clocks_gpu{gpu}_", suffix=".csv")
        os.close(fd)

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        loaded = [x for x in sm if x > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def load_traffic_table(path: str = TRAFFIC_TABLE):
    """DRAM bytes per launch at the finest level (1600x1200), per kernel, from the ncu summary
    profiles/dram_bytes_per_launch.md: the rows of its table `| kernel | read | write | ... |`
    (bytes).  Returns {kernel: bytes} (empty when the summary is absent)."""
    out = {}
    if not os.path.exists(path):
        return out
    for line in open(path):
        m = re.match(r"\|\s*`?(k_\w+)`?\s*\|\s*([\d.e+]+)\s*\|\s*([\d.e+]+)\s*\|", line)
        if m:
            out[m.group(1)] = float(m.group(2)) + float(m.group(3))
    return out


# ----------------------------------------------------------------------------- the CPU reference
def schedule_params(level: int, call: int, n_images: int):
    """PatchMatchParams of call `call` (0: FIRST_INIT / REFINE_INIT, 1: the geom REFINE_ITER call)
    at pyramid level `level` of the measured schedule (main.cpp:390-457, as csrc/scene.cu sets
    them), built without loading the CUDA library."""
    import dpe_b200 as D

    p = D.reference_default_params()
    p.num_images = n_images
    p.max_iterations = WORKLOAD["max_iterations"]
    if call == 0:
        if level == 0:
            p.state, p.use_APD, p.use_edge = D.FIRST_INIT, 0, 0
        else:
            p.state, p.use_APD, p.use_edge = D.REFINE_INIT, 1, 1
            p.ransac_threshold = np.float32(0.01 - level * 0.00125)
            p.rotate_time = min(1 << level, 4)
        p.geom_consistency = 0
        p.weak_peak_radius = 6
    else:
        p.state = D.REFINE_ITER
        p.use_APD = p.use_edge = 1 if level > 0 else 0
        p.ransac_threshold = np.float32(0.01 - level * 0.00125)
        p.rotate_time = min(1 << level, 4)
        p.geom_consistency = 1
        p.weak_peak_radius = max(4 - 2 * (call - 1), 2)
    return p


class RefSampler:
    """The reference's own code compiled for the host (oracle/_ref/libref.so) on a bounded sample of
    the measured schedule: one reference view of the same scene layout rendered at 200x150 (the
    `c2_200` preset, 10 images), running the schedule's call kinds in order --
      0 FIRST_INIT (level-0 parameters), 1 geom REFINE_ITER (level 0), 2 REFINE_INIT with APD,
      edges, labels (level 1), 3 geom REFINE_ITER (level 1), 4 / 5 the same with level-2
      parameters, 6 the fusion of the 10-view depth set --
    each call fed the state the previous one produced (source depths for the geometric term and
    the other views' depth maps for fusion are the scene's ground truth).  Every item is one real
    call of the reference's code, timed alone on all host cores; the schedule time is estimated
    from the measured time per pixel of each kind and the pixel count each kind has in the full
    schedule (10 views x 400x300, 800x600, 1600x1200; fusion of 10 x 1600x1200)."""

    KINDS = ("first_init_L0", "geom_L0", "refine_init_L1", "geom_L1", "refine_init_L2", "geom_L2", "fusion")
    LEVEL_OF = (0, 0, 1, 1, 2, 2, None)

    def __init__(self, threads: int):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import edges as E
        import ref_py as R
        import scene as S

        self.R = R
        self.threads = threads
        self.sc = S.make_scene("c2_200", seed=1)
        self.v = 4
        self.srcs = list(self.sc.pairs[self.v])
        ids = [self.v] + self.srcs
        self.images = [np.ascontiguousarray(self.sc.gray[i].astype(np.float32)) for i in ids]
        self.cams = [S.camera_struct(self.sc, i) for i in ids]
        self.edge, self.label = E.level_inputs(self.sc.gray[self.v], 1)
        self.low = np.ascontiguousarray(E.level_inputs(self.sc.gray[self.v], 4)[0])
        self.edge = np.ascontiguousarray(self.edge)
        self.label = np.ascontiguousarray(self.label)
        self.pixels = self.images[0].size
        self.state = None
        self.times = {k: [] for k in self.KINDS}
        self.first_init_inputs = None

    def _call(self, level: int, call: int):
        p = schedule_params(level, call, len(self.images))
        p.max_scale_size = self.edge.shape[1] // self.low.shape[1]
        kw = dict(seed=1000 + 10 * level + call)
        if p.state != 0:
            plane, weak, views = self.state
            kw.update(plane_in=plane, views_in=views, weak_in=weak)
        if p.use_edge or p.use_limit:
            kw.update(edge=self.edge, edge_low=self.low)
        if p.use_label:
            kw.update(label=self.label)
        if p.geom_consistency:
            kw["depths"] = [np.ascontiguousarray(self.state[0][..., 3])] + \
                [np.ascontiguousarray(self.sc.depth[i].astype(np.float32)) for i in self.srcs]
        t0 = time.perf_counter()
        r = self.R.pm_call(self.images, self.cams, p, threads=self.threads, serial_race=False, **kw)
        dt = time.perf_counter() - t0
        if p.state == 0:
            self.first_init_inputs = (p, kw, r)
        # ProcessProblem's result assembly (main.cpp:266-279)
        depth = r["plane"][..., 3].copy()
        weak = r["weak"].copy()
        bad = (depth < r["params"].depth_min) | (depth > r["params"].depth_max)
        depth[bad] = 0.0
        weak[bad] = 2
        plane = np.ascontiguousarray(np.concatenate([r["plane"][..., :3], depth[..., None]], -1).astype(np.float32))
        self.state = (plane, np.ascontiguousarray(weak), np.ascontiguousarray(r["views"]))
        return dt

    def _fusion(self):
        import scene as S

        views = []
        for i in range(self.sc.n):
            if i == self.v:
                d, n = self.state[0][..., 3], self.state[0][..., :3]
            else:
                d, n = self.sc.depth[i].astype(np.float32), self.sc.normal[i].astype(np.float32)
            views.append(dict(depth=np.ascontiguousarray(d), normal=np.ascontiguousarray(n),
                              weak=np.full(d.shape, 1, np.uint8), bgr=np.ascontiguousarray(self.sc.bgr[i]),
                              camera=S.camera_struct(self.sc, i), src=self.sc.pairs[i]))
        t0 = time.perf_counter()
        r = self.R.fuse(views)
        return time.perf_counter() - t0, r["count"]

    def run(self, item: int) -> float:
        """Runs item `item` (0..6; the chain restarts at 0) and returns its seconds."""
        k = item % len(self.KINDS)
        if k == 6:
            dt, _ = self._fusion()
        else:
            if self.state is None and k > 0:
                self._call(0, 0)  # the chain's first state, untimed
            dt = self._call(self.LEVEL_OF[k], k % 2)
        self.times[self.KINDS[k]].append(dt)
        return dt

    def schedule_seconds(self):
        """Estimated seconds of the full schedule from the measured kinds (None if a kind is missing);
        kinds not measured take the time per pixel of the closest measured kind of the same call."""
        med = {k: statistics.median(v) for k, v in self.times.items() if v}
        if "fusion" not in med or not any(k.startswith("geom") for k in med) or not any(
                not k.startswith("geom") and k != "fusion" for k in med):
            return None
        V, W, H, L = WORKLOAD["views"], WORKLOAD["width"], WORKLOAD["height"], WORKLOAD["levels"]
        total = 0.0
        for lvl in range(L):
            px = (W >> (L - 1 - lvl)) * (H >> (L - 1 - lvl))
            for call, prefix in ((0, "first_init" if lvl == 0 else "refine_init"), (1, "geom")):
                name = f"{prefix}_L{lvl}"
                if name not in med:  # nearest measured level of the same call kind
                    cands = [k for k in med if (k.startswith("geom") if call else not k.startswith("geom") and k != "fusion")]
                    name = min(cands, key=lambda k: abs(int(k[-1]) - lvl))
                total += V * med[name] / self.pixels * px
        total += med["fusion"] / (self.sc.n * self.pixels) * (V * W * H)
        return total


def cpu_reference_line(sampler: RefSampler, n_items: int):
    """Runs `n_items` timed sample items (at least one full cycle of the 7 kinds) and returns
    (value Mpix/s, seconds per item, description)."""
    per = [sampler.run(i) for i in range(max(n_items, len(RefSampler.KINDS)))]
    sched = sampler.schedule_seconds()
    pix = WORKLOAD["views"] * WORKLOAD["width"] * WORKLOAD["height"] / 1e6
    med = {k: round(statistics.median(v), 3) for k, v in sampler.times.items() if v}
    desc = ("the reference's own DPE.cu/DPE.cpp compiled for the host (oracle/_ref/libref.so), all host threads; "
            f"{len(per)} timed items cycling through the schedule's 6 call kinds and fusion on one reference view of "
            "the c2 layout rendered at 200x150 with 10 images (seconds per item: "
            + ", ".join(f"{k} {v}" for k, v in med.items()) +
            "); the full schedule time is each kind's measured time per pixel times its pixel count in the "
            "10-view 400x300/800x600/1600x1200 schedule and the 10 x 1600x1200 fusion (no other scaling)")
    return pix / sched, per, desc, sched


def run_reference(args):
    rank, world, _ = _env_rank()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    sampler = RefSampler(threads)
    if args.warmup > 0:
        sampler.run(0)  # untimed: pages in the library and the scene; the chain restarts below
        sampler.times = {k: [] for k in RefSampler.KINDS}
        sampler.state = None
    value, per, desc, sched = cpu_reference_line(sampler, args.steps)
    line = dict(metric=METRIC, value=round(value, 6), unit=UNIT, impl="reference", n_gpus=args.gpus, steps=len(per),
                warmup=min(args.warmup, 1), ms_per_step=round(statistics.mean(per) * 1e3, 3), higher_is_better=True,
                scaling="weak", vs_baseline=None, dtype="f32", data="synthetic",
                config=dict(workload="c2 full pipeline: 10 views 1600x1200, 3 levels, init + 1 geom call per level, "
                                     "3 iterations, fusion min 2 views", **WORKLOAD),
                schedule_s_estimate=round(sched, 2),
                cpu_baseline=dict(value=round(value, 6), unit=UNIT, cores=threads, kind="reference", sample=desc),
                e2e=dict(value=round(value, 6), unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------- this library
def _measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d.get("hbm_gbs", 6650.0)), "measured (MEASURED_PEAKS.json)"
    return 6650.0, "fallback (6.65 TB/s, no MEASURED_PEAKS.json)"


def _depth_accuracy(res, sc, V):
    rl = np.concatenate([np.abs(res["depth"][v] - sc.depth[v]).ravel() / sc.depth[v].ravel() for v in range(V)])
    ok = np.concatenate([(res["depth"][v] > 0).ravel() for v in range(V)])
    return float((rl[ok] < 0.01).mean()), float((rl[ok] < 0.001).mean()), float(ok.mean())


def _depth_agreement(a, b, V, tol=1e-3):
    """Fraction of pixels whose depths in two schedule results agree within `tol` relative."""
    da = np.concatenate([a["depth"][v].ravel() for v in range(V)]).astype(np.float64)
    db = np.concatenate([b["depth"][v].ravel() for v in range(V)]).astype(np.float64)
    return float((np.abs(da - db) <= tol * np.maximum(np.abs(db), 1e-12)).mean())


def kernel_rooflines(stats, counted, steps, fp32_peak, traffic, levels):
    """FP32 roofline of every cost kernel: algorithmic FLOP per step (NCC evaluations from the
    counting pass x FLOP per evaluation) over its event-timed device time per step, and its DRAM
    bytes per launch (the finest-level ncu figure scaled to the mean launch: the kernels launch
    equally often at every pyramid level, whose pixel counts are 1/4^k of the finest)."""
    mean_px_ratio = statistics.mean(4.0 ** -(levels - 1 - l) for l in range(levels))
    out = {}
    for name in COST_KERNELS:
        st, c = stats.get(name), counted.get(name, {})
        if not st or st["ms"] <= 0:
            continue
        flop = c.get("strong_ncc_evals", 0) * STRONG_NCC_FLOP + c.get("weak_ncc_evals", 0) * WEAK_NCC_FLOP
        ms = st["ms"] / steps
        ach = flop / (ms * 1e-3) / 1e12
        launches = max(1, st["launches"] // steps)
        tb = traffic.get(name)
        out[name] = dict(achieved=round(ach, 3), unit="TFLOP/s", frac=round(ach / fp32_peak, 4) if fp32_peak else None,
                         ms_per_step=round(ms, 3), launches_per_step=launches, flop_per_launch=flop / launches,
                         ms_per_launch=round(ms / launches, 4),
                         traffic=int(tb * mean_px_ratio) if tb else None)
    return out


def fusion_roofline(srcs, width, height, points, num_consistent, fusion_ms, hbm_peak, peak_src):
    """HBM roofline of fusion: algorithmic bytes per step (per reference pixel its depth, normal,
    state and mask, 18 B, plus 17 B per source tested; per point the 3 B colours of the reference
    and every consistent source and the 15 B written) over the measured fusion device time."""
    npix = width * height
    read = sum(npix * (18 + 17 * len(s)) for s in srcs)
    colour = int(3 * (points + int(np.asarray(num_consistent, np.int64).sum())))
    total = read + colour + 15 * points
    ach = total / (fusion_ms * 1e-3) / 1e9
    return dict(bound="hbm", achieved=round(ach, 2), peak=round(hbm_peak, 1), unit="GB/s",
                frac=round(ach / hbm_peak, 5), algorithmic_bytes=total, fusion_ms=round(fusion_ms, 3),
                peak_source=peak_src)


def run_ours(args):
    import torch
    import dpe_b200 as D

    rank, world, local = _env_rank()
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    L = WORKLOAD["levels"]
    sc, cams, srcs, edges_l, labels_l = _prepare_scene(WORKLOAD["scene"], seed=1 + rank, device=dev, levels=L)
    V, H, W = sc.gray.shape
    ctx = D.Context(local)
    fp32_peak = ctx.fp32_peak_tflops()
    hbm_peak, hbm_src = _measured_peaks()

    # device-resident inputs
    gray_d = [torch.from_numpy(sc.gray[v]).to(dev).contiguous() for v in range(V)]
    bgr_d = [torch.from_numpy(sc.bgr[v]).to(dev).contiguous() for v in range(V)]
    edges_d = [[torch.from_numpy(e).to(dev).contiguous() for e in ev] for ev in edges_l]
    labels_d = [[torch.from_numpy(l).to(dev).contiguous() for l in lv] for lv in labels_l]
    torch.cuda.synchronize()
    kw = dict(num_levels=L, refine_calls=WORKLOAD["refine_calls"], max_iterations=WORKLOAD["max_iterations"],
              fuse_mode=D.FUSE_FP64, min_consistent=WORKLOAD["min_consistent"])

    def step_device(seed, want_maps=False, **extra):
        return ctx.scene_run(gray_d, bgr_d, cams, srcs, edges_d, labels_d, seed=seed, memory=D.MEM_DEVICE,
                             want_maps=want_maps, **kw, **extra)

    for i in range(args.warmup):
        step_device(100 + i)
    # one untimed counting pass: NCC evaluations per kernel class (deterministic for the seed)
    ctx.set_eval_counting(True)
    ctx.reset_kernel_stats()
    step_device(7)
    counted = ctx.kernel_stats()
    ctx.set_eval_counting(False)
    evals_strong = sum(k["strong_ncc_evals"] for k in counted.values())
    evals_weak = sum(k["weak_ncc_evals"] for k in counted.values())

    # timed region (per-kernel event timing on)
    ctx.reset_kernel_stats()
    ctx.set_profiling(True)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = D.load_library().dpe_launch_count()
    wall0 = time.perf_counter()
    gpu_ms = 0.0
    last = None
    torch.cuda.nvtx.range_push("timed_steps")
    with ClockSampler(local) as clocks:
        for i in range(args.steps):
            last = step_device(7)
            gpu_ms += last["gpu_ms"]
        torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    wall = time.perf_counter() - wall0
    if dist is not None:
        dist.barrier()
    launches = D.load_library().dpe_launch_count() - launches0
    ctx.set_profiling(False)
    stats = ctx.kernel_stats()
    # the launch tuner's choices at the finest level (made during the warm-up steps): the kept
    # setting and its gain over the first candidate (16x8 blocks / the driver's carveout)
    tuning = ctx.tuning()
    finest = max((e["size_class"] for e in tuning), default=None)
    autotune = {}
    for e in tuning:
        if e["size_class"] != finest or e["chosen"] < 0 or not e["mean_ms"][e["chosen"]]:
            continue
        kept = f"{e['block'][0]}x{e['block'][1]} blocks" if e["block"][0] else f"carveout {e['carveout']}"
        autotune[e["kernel"]] = dict(kept=kept, mean_ms=e["mean_ms"],
                                     gain_vs_first=round(e["mean_ms"][0] / e["mean_ms"][e["chosen"]], 3))
    ms_per_step = gpu_ms / args.steps
    if dist is not None:
        t = torch.tensor([ms_per_step], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_per_step = float(t.item())
    pix_step = V * W * H / 1e6
    value = pix_step * world / (ms_per_step / 1e3)

    # end to end through the C-ABI with pinned host buffers
    pin = lambda a: torch.from_numpy(a).pin_memory().numpy()
    gray_h = [pin(sc.gray[v]) for v in range(V)]
    bgr_h = [pin(sc.bgr[v]) for v in range(V)]
    edges_h = [[pin(e) for e in ev] for ev in edges_l]
    labels_h = [[pin(l) for l in lv] for lv in labels_l]
    h2d = sum(a.nbytes for a in gray_h) + sum(a.nbytes for a in bgr_h) + sum(e.nbytes for ev in edges_h for e in ev) + \
        sum(l.nbytes for lv in labels_h for l in lv)
    e2e_times = []
    res = None
    for i in range(max(1, min(args.steps, 5))):
        t0 = time.perf_counter()
        res = ctx.scene_run(gray_h, bgr_h, cams, srcs, edges_h, labels_h, seed=7, memory=D.MEM_HOST, want_maps=True,
                            want_consistency=True, **kw)
        e2e_times.append(time.perf_counter() - t0)
    d2h = V * H * W * (4 + 12 + 1 + 4) + res["points"] * 15
    e2e_s = statistics.median(e2e_times)
    if dist is not None:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = pix_step * world / e2e_s
    acc1, acc01, valid = _depth_accuracy(res, sc, V)

    # the batched forms on the same scene (device-resident; 1 warm-up + 3 timed schedules each, then
    # one schedule with maps for accuracy and agreement with the plain schedule): all views of a
    # call in one batch (reading the previous call's depths), then additionally FP16-staged sources
    # and the Gauss-Newton plane hypothesis from the NCC adjoint
    forms = {}
    if not args.no_forms:
        for name, staging, gn in (("batched", D.STAGE_FP32, 0), ("batched_fp16_gn", D.STAGE_FP16, 1)):
            ctx.set_options(staging=staging, gn_refine=gn)
            step_device(7, batch_views=True)
            times = []
            with ClockSampler(local) as fclocks:
                for i in range(3):
                    times.append(step_device(7, batch_views=True)["gpu_ms"])
            r = step_device(7, want_maps=True, batch_views=True)
            ctx.set_options()
            fms = statistics.median(times)
            fv = pix_step * world / (fms / 1e3)
            a1, a01, _ = _depth_accuracy(r, sc, V)
            forms[name] = dict(value=round(fv, 4), unit=UNIT, ms_per_step=round(fms, 3),
                               ms_per_step_samples=[round(t, 1) for t in times], vs_plain=round(fv / value, 3),
                               depth_within_1pct=round(a1, 4), depth_within_0_1pct=round(a01, 4),
                               depth_agreement_with_plain_0_1pct=round(_depth_agreement(r, res, V), 4),
                               staging={D.STAGE_FP32: "fp32", D.STAGE_FP16: "fp16"}[staging],
                               gauss_newton=bool(gn), points=int(r["points"]), clocks=fclocks.summary())

    # the same forms on the batching workload (C5), one process only; a failure there leaves the
    # rest of the line intact
    forms_c5 = None
    if not args.no_forms and world == 1:
        try:
            c5 = measure_c5(ctx, 1)
            forms_c5 = dict(workload=c5["config"]["workload"], reference_mpix=c5["config"]["reference_mpix"],
                            fusion=c5["fusion"], **c5["forms"])
        except Exception as e:  # noqa: BLE001 -- reported in the line
            forms_c5 = dict(error=repr(e)[:300])
    traffic = load_traffic_table()
    rooflines = kernel_rooflines(stats, counted, args.steps, fp32_peak, traffic, L)
    dname = max(rooflines, key=lambda k: rooflines[k]["ms_per_step"])
    d = rooflines[dname]
    total_kernel_ms = sum(k["ms"] for k in stats.values())
    roofline = dict(kernel=dname, bound="fp32", achieved=d["achieved"], peak=round(fp32_peak, 3), unit="TFLOP/s",
                    frac=d["frac"], traffic=d["traffic"],
                    peak_source="measured FP32 FMA throughput on this GPU (dpe_fp32_peak); MEASURED_PEAKS.json has no "
                                "FP32 figure",
                    traffic_source="profiles/dram_bytes_per_launch.md (finest level, scaled to the mean launch)",
                    share_of_kernel_time=round(stats[dname]["ms"] / total_kernel_ms, 4),
                    flop_per_launch=d["flop_per_launch"], ms_per_launch=d["ms_per_launch"])
    fusion = fusion_roofline(srcs, W, H, res["points"], res["num_consistent"], last["fusion_ms"], hbm_peak, hbm_src)
    fusion["kernel_ms_per_step"] = {k: round(stats[k]["ms"] / args.steps, 3) for k in FUSION_KERNELS if k in stats}
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sampler = RefSampler(threads)
        cvalue, per, desc, _ = cpu_reference_line(sampler, len(RefSampler.KINDS))
        # the same first-init sample call on this GPU: depth agreement with the reference's own result
        p0, kw0, r0 = sampler.first_init_inputs
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        g0 = ctx.pm_run(sampler.images, sampler.R.camera_dicts(r0["cameras"]), r0["params"], **kw0)
        da, db = g0["plane"][..., 3].astype(np.float64), r0["plane"][..., 3].astype(np.float64)
        agree = float((np.abs(da - db) <= 1e-3 * np.abs(db)).mean())
        cpu = dict(value=round(cvalue, 6), unit=UNIT, cores=threads, kind="reference", sample=desc,
                   gpu_vs_reference_first_init_depth_within_0_1pct=round(agree, 5))
    line = dict(metric=METRIC, value=round(value, 4), unit=UNIT, n_gpus=world, steps=args.steps, warmup=args.warmup,
                ms_per_step=round(ms_per_step, 3), higher_is_better=True, scaling="weak", vs_baseline=None,
                dtype="f32", data="synthetic (seeded ray-cast scene in place of ETH3D)",
                config=dict(workload="c2 full pipeline: 10 views 1600x1200, 3 levels, init + 1 geom call per level, "
                                     "3 iterations, fusion min 2 views", parallelism=f"replicas{world}",
                            l2="inputs and state larger than L2 (no flush)", **WORKLOAD),
                ncc_evals_per_s=round((evals_strong + evals_weak) * world / (ms_per_step / 1e3), 1),
                strong_ncc_evals_per_step=evals_strong, weak_ncc_evals_per_step=evals_weak,
                points=int(last["points"]), fusion_ms=round(last["fusion_ms"], 3), wall_s_timed=round(wall, 3),
                depth_within_1pct=round(acc1, 4), depth_within_0_1pct=round(acc01, 4),
                valid_depth_fraction=round(valid, 4),
                roofline=roofline, rooflines=rooflines, fusion_roofline=fusion, cpu_baseline=cpu,
                clocks=clocks.summary(), gpu_launches=int(launches),
                e2e=dict(value=round(e2e_value, 4), unit=UNIT, h2d_bytes_per_step=int(h2d), d2h_bytes_per_step=int(d2h)),
                kernel_ms_per_step={k: round(v["ms"] / max(1, args.steps), 3) for k, v in
                                    sorted(stats.items(), key=lambda kv: -kv[1]["ms"])},
                forms=forms or None, forms_c5=forms_c5, autotune=autotune or None)
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


# ----------------------------------------------------------------------------- profiling runs
def run_case(args):
    """Device-resident schedules of one scene for kernel profilers: `--repeat` complete schedules
    (PatchMatch pyramid + fusion) through dpe_scene_run; prints each schedule's device time and
    library launches, and with --stats the device time of every kernel class over the last one."""
    import torch
    import dpe_b200 as D

    sc, cams, srcs, edges_l, labels_l = _prepare_scene(args.case, seed=args.seed, device="cuda", levels=args.levels)
    V = sc.n
    gray_d = [torch.from_numpy(np.ascontiguousarray(sc.gray[v])).cuda() for v in range(V)]
    bgr_d = [torch.from_numpy(np.ascontiguousarray(sc.bgr[v])).cuda() for v in range(V)]
    edges_d = [[torch.from_numpy(e).cuda() for e in ev] for ev in edges_l]
    labels_d = [[torch.from_numpy(x).cuda() for x in lv] for lv in labels_l]
    ctx = D.Context(0)
    ctx.set_options(staging=args.staging, gn_refine=1 if args.gn else 0)
    lib = D.load_library()
    for r in range(args.repeat):
        if args.stats and r == args.repeat - 1:
            ctx.reset_kernel_stats()
            ctx.set_profiling(True)
        n0 = lib.dpe_launch_count()
        res = ctx.scene_run(gray_d, bgr_d, cams, srcs, edges_d, labels_d, num_levels=args.levels,
                            refine_calls=WORKLOAD["refine_calls"], max_iterations=args.iters, fuse_mode=D.FUSE_FP64,
                            min_consistent=WORKLOAD["min_consistent"], seed=7, memory=D.MEM_DEVICE, want_maps=False)
        print(f"schedule {r}: {args.case} {V} views, {args.levels} levels: {res['gpu_ms']:.1f} ms "
              f"(fusion {res['fusion_ms']:.1f} ms), {res['points']} points, {lib.dpe_launch_count() - n0} launches",
              flush=True)
    if args.stats:
        for name, st in sorted(ctx.kernel_stats().items(), key=lambda kv: -kv[1]["ms"]):
            print(f"  {name:24s} {st['launches']:6d} launches {st['ms']:10.2f} ms")
    ctx.close()
    return 0


def run_c5(args):
    """The batching workload: 49 reference views of three sizes (20 at 640x480, 20 at 1600x1200, 9 at
    3200x2400) on a 60-camera ring, each with its 10 nearest ring neighbours as sources; one
    FIRST_INIT call per view (3 iterations, geom off).  Forms: per-view FP32 calls (plain), all 49
    problems in one kernel sequence (batched), and batched with FP16-staged sources and the
    Gauss-Newton hypothesis; 1 warm-up + 3 timed runs each (device time of the kernel sequences),
    with clocks; depth agreement with plain and accuracy against ground truth; then fusion of the
    last form's depth maps into one point cloud.  Prints one JSON line."""
    import dpe_b200 as D

    ctx = D.Context(0)
    print(json.dumps(measure_c5(ctx, args.seed)), flush=True)
    ctx.close()
    return 0


def measure_c5(ctx, seed: int) -> dict:
    """The forms of the batching workload (run_c5) on context ctx; returns the line's fields."""
    import dpe_b200 as D
    import scene as S

    t0 = time.perf_counter()
    ring, probs = S.c5_workload(seed=seed, device="cuda")
    gen_s = time.perf_counter() - t0
    p = schedule_params(0, 0, 11)
    p.use_limit = p.use_label = 0  # no edge or label maps: FIRST_INIT as ProcessProblem runs it at level 0
    p.depth_min = np.float32(ring.spec.depth_min) * np.float32(0.6)  # DPE::InuputInitialization (DPE.cpp:953-954)
    p.depth_max = np.float32(ring.spec.depth_max) * np.float32(1.2)
    calls = [dict(images=q["images"], cameras=q["cameras"], params=p, seed=1000 + i) for i, q in enumerate(probs)]
    mpix = sum(q["width"] * q["height"] for q in probs) / 1e6

    def plain():
        out, ms = [], 0.0
        for c in calls:
            r = ctx.pm_run(c["images"], c["cameras"], c["params"], seed=c["seed"])
            ms += r["gpu_ms"]
            out.append(r)
        return out, ms

    def batched():
        out = ctx.pm_run_batch(calls)
        return out, max(r["gpu_ms"] for r in out)

    def depths(res):
        return np.concatenate([r["plane"][..., 3].ravel() for r in res])

    gt = np.concatenate([q["depth"].ravel() for q in probs])
    forms, ref_res, last = {}, None, None
    for name, fn, staging, gn in (("plain", plain, D.STAGE_FP32, 0), ("batched", batched, D.STAGE_FP32, 0),
                                  ("batched_fp16_gn", batched, D.STAGE_FP16, 1)):
        ctx.set_options(staging=staging, gn_refine=gn)
        fn()
        times, walls = [], []
        with ClockSampler(0) as clk:
            for _ in range(3):
                w0 = time.perf_counter()
                res, ms = fn()
                walls.append(time.perf_counter() - w0)
                times.append(ms)
        ctx.set_options()
        ms = statistics.median(times)
        d = depths(res)
        f = dict(value=round(mpix / (ms / 1e3), 4), unit=UNIT, ms=round(ms, 2), ms_samples=[round(t, 1) for t in times],
                 wall_s=round(statistics.median(walls), 3), staging={D.STAGE_FP32: "fp32", D.STAGE_FP16: "fp16"}[staging],
                 gauss_newton=bool(gn), depth_within_1pct_of_gt=round(float((np.abs(d - gt) <= 0.01 * gt).mean()), 4),
                 clocks=clk.summary())
        if ref_res is None:
            ref_res = res
        else:
            dp = depths(ref_res)
            f["depth_agreement_with_plain_0_1pct"] = round(float((np.abs(d - dp) <= 1e-3 * np.abs(dp)).mean()), 4)
            f["vs_plain"] = round(f["value"] / forms["plain"]["value"], 3)
        forms[name] = f
        last = res
    # whole-scene fusion: each view's sources are its ring neighbours that are reference views too
    index = {q["ref"]: i for i, q in enumerate(probs)}
    views = []
    for q, r in zip(probs, last):
        views.append(dict(depth=np.ascontiguousarray(r["plane"][..., 3]), normal=np.ascontiguousarray(r["plane"][..., :3]),
                          weak=r["weak"], bgr=q["bgr"], camera=q["cameras"][0],
                          src=[index[s] for s in q["sources"] if s in index]))
    fu = ctx.fuse(views, D.FUSE_FP64, min_consistent=2)
    line = dict(metric=METRIC, unit=UNIT, data="synthetic (seeded 60-camera ring scene)",
                config=dict(workload="c5 batching: 49 reference views (20 x 640x480, 20 x 1600x1200, 9 x 3200x2400) on a "
                                     "60-camera ring, 10 sources each, FIRST_INIT 3 iterations, then fusion min 2 views",
                            reference_mpix=round(mpix, 3)),
                scene_generation_s=round(gen_s, 1), forms=forms,
                fusion=dict(points=int(fu["count"]), gpu_ms=round(fu["gpu_ms"], 2)))
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the batched / FP16 / Gauss-Newton forms")
    ap.add_argument("--case", default=None, help="profiling run of this scene preset (c2, c2_small, ...)")
    ap.add_argument("--levels", type=int, default=2)
    ap.add_argument("--iters", type=int, default=3)
    ap.add_argument("--repeat", type=int, default=2)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--stats", action="store_true")
    ap.add_argument("--staging", type=int, default=0)
    ap.add_argument("--gn", action="store_true")
    args = ap.parse_args()
    if args.case == "c5":
        return run_c5(args)
    if args.case:
        return run_case(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
