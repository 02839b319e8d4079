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

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
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


def _env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def _prepare_scene(seed: int, device: str):
    import scene as S
    import edges as E

    sc = S.make_scene(WORKLOAD["scene"], seed=seed, device=device)
    V, H, W = sc.gray.shape
    L = WORKLOAD["levels"]
    edges_l, labels_l = [], []
    for v in range(V):
        ev, lv = [], []
        for lvl in range(L):
            e, lab = E.level_inputs(sc.gray[v], 1 << (L - 1 - lvl))
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
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_gpu{gpu}.csv") if os.path.isdir(os.path.join(ROOT, "gpurun_out")) \
            else f"/tmp/dpe_clocks_gpu{gpu}.csv"

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
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        loaded = [x for x in sm if x > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# DRAM bytes per launch of the cost kernels on this workload: ncu dram__bytes_read.sum +
# dram__bytes_write.sum over every launch of one complete schedule (a 1-pass capture of
# `dpe-mvs-fast_b200/profile_case.py --scene c2 --levels 3 --repeat 1`), averaged over the launches
# the way `roofline.achieved` averages FLOP over them.  Measured, not modelled: re-captured when a
# kernel changes.
DRAM_BYTES_PER_LAUNCH = {
    "k_strong_update": 121.3e6,
    "k_depth_to_weak": 73.7e6,
    "k_local_refine": 72.1e6,
}


def _traffic_for(kernel: str):
    v = DRAM_BYTES_PER_LAUNCH.get(kernel)
    return int(v) if v is not None else None


def cpu_sample(threads: int = 0):
    """The oracle (OpenMP C++ restatement, all host threads) on a bounded sample of the workload:
    a FIRST_INIT call and a geom REFINE_ITER call (APD, edge, label on) of one view at the
    coarsest pyramid level (400x300, 10 images, 3 iterations).  Returns seconds per call type and
    the estimated seconds of the whole schedule (per-call time scaled by pixel count per level)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import dpe_b200 as D
    import oracle_py as O
    import scene as S
    import edges as E

    sc = S.make_scene("c2_small", seed=1)
    v = 4
    ids = [v] + sc.pairs[v]
    images = [np.ascontiguousarray(sc.gray[i].astype(np.float32)) for i in ids]
    cams = [S.camera_struct(sc, i) for i in ids]
    p = D.Params()
    D.load_library().dpe_params_default(p) if os.path.exists(D.LIB_PATH) else _defaults(p)
    p.num_images = len(images)
    p.depth_min = np.float32(sc.spec.depth_min) * np.float32(0.6)
    p.depth_max = np.float32(sc.spec.depth_max) * np.float32(1.2)
    p.state = D.FIRST_INIT
    p.use_APD = 0
    p.use_edge = 0
    p.use_limit = 0
    p.use_label = 0
    p.geom_consistency = 0
    p.weak_peak_radius = 6
    t0 = time.perf_counter()
    o = O.pm_run(images, cams, p, threads=threads, seed=11)
    t_init = time.perf_counter() - t0
    depth = o["plane"][..., 3].copy()
    weak = o["weak"].copy()
    bad = (depth < p.depth_min) | (depth > p.depth_max)
    weak[bad] = D.UNKNOWN
    state = np.ascontiguousarray(np.concatenate([o["plane"][..., :3], np.where(bad, 0, depth)[..., None]], -1).astype(np.float32))
    e, lab = E.level_inputs(sc.gray[v], 1)
    q = D.Params.from_buffer_copy(p)
    q.state = D.REFINE_ITER
    q.use_APD = 1
    q.use_edge = 1
    q.use_limit = 1
    q.use_label = 1
    q.use_radius = 1
    q.geom_consistency = 1
    q.ransac_threshold = np.float32(0.01)
    q.rotate_time = 1
    q.weak_peak_radius = 4
    depths = [np.ascontiguousarray(sc.depth[i].astype(np.float32)) for i in ids]
    t0 = time.perf_counter()
    O.pm_run(images, cams, q, threads=threads, plane_in=state, views_in=np.ascontiguousarray(o["views"]),
             weak_in=np.ascontiguousarray(weak), edge=e, edge_low=e, label=lab, depths=depths, seed=12)
    t_refine = time.perf_counter() - t0
    # whole schedule: per level V x (1 init + refine_calls refines), time proportional to pixels
    V, L, rc = WORKLOAD["views"], WORKLOAD["levels"], WORKLOAD["refine_calls"]
    total = 0.0
    for lvl in range(L):
        ratio = 4 ** lvl
        init_t = t_init if lvl == 0 else t_refine
        total += ratio * V * (init_t + rc * t_refine)
    return dict(t_init=t_init, t_refine=t_refine, schedule_s=total, sample_pixels=images[0].size)


def _defaults(p):
    # PatchMatchParams defaults (main.h:81-109), used when the CUDA library is not built
    for k, v in dict(max_iterations=3, num_images=5, sigma_spatial=5.0, sigma_color=3.0, top_k=4, strong_radius=5,
                     strong_increment=2, weak_radius=5, weak_increment=5, use_APD=1, use_edge=1, use_limit=1,
                     use_label=1, use_radius=1, high_res_img=1, max_scale_size=1, scale_size=1, weak_peak_radius=2,
                     rotate_time=4, ransac_threshold=0.005, geom_factor=0.2).items():
        setattr(p, k, v)


def run_reference(args):
    rank, world, _ = _env_rank()
    if rank != 0:
        return 0
    import multiprocessing

    threads = multiprocessing.cpu_count()
    pix = WORKLOAD["views"] * WORKLOAD["width"] * WORKLOAD["height"] / 1e6
    if args.warmup > 0:  # one warm-up sample: the CPU path has no caches worth more
        cpu_sample(threads)
    samples = [cpu_sample(threads) for _ in range(args.steps)]
    sched = statistics.median(s["schedule_s"] for s in samples)
    value = pix / sched
    sample_desc = ("oracle C++/OpenMP restatement (the reference's CUDA path has no CPU implementation); per step one "
                   "FIRST_INIT and one geom REFINE_ITER call of one view at 400x300 with 10 images; the schedule time is "
                   "those call times scaled by pixel count over 3 levels x 10 views x 2 calls")
    line = dict(metric=METRIC, value=round(value, 6), unit=UNIT, impl="reference", n_gpus=args.gpus, steps=args.steps,
                warmup=args.warmup, ms_per_step=round(sched * 1e3, 3), higher_is_better=True, scaling="weak",
                vs_baseline=None, dtype="f32", data="synthetic", config=dict(workload="c2 full pipeline", **WORKLOAD),
                cpu_baseline=dict(value=round(value, 6), unit=UNIT, cores=threads, kind="port", sample=sample_desc),
                e2e=dict(value=round(value, 6), unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)
    return 0


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
    sc, cams, srcs, edges_l, labels_l = _prepare_scene(seed=1 + rank, device=dev)
    V, H, W = sc.gray.shape
    L = WORKLOAD["levels"]
    ctx = D.Context(local)
    fp32_peak = ctx.fp32_peak_tflops()

    # device-resident inputs
    gray_d = [torch.from_numpy(sc.gray[v]).to(dev).contiguous() for v in range(V)]
    bgr_d = [torch.from_numpy(sc.bgr[v]).to(dev).contiguous() for v in range(V)]
    edges_d = [[torch.from_numpy(e).to(dev).contiguous() for e in ev] for ev in edges_l]
    labels_d = [[torch.from_numpy(l).to(dev).contiguous() for l in lv] for lv in labels_l]
    torch.cuda.synchronize()
    kw = dict(num_levels=L, refine_calls=WORKLOAD["refine_calls"], max_iterations=WORKLOAD["max_iterations"],
              fuse_mode=D.FUSE_FP64, min_consistent=WORKLOAD["min_consistent"])

    def step_device(seed):
        return ctx.scene_run(gray_d, bgr_d, cams, srcs, edges_d, labels_d, seed=seed, memory=D.MEM_DEVICE,
                             want_maps=False, **kw)

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
    # an NVTX range around the timed steps, so a profiler can select exactly their launches
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
    for i in range(max(1, args.steps)):
        t0 = time.perf_counter()
        res = ctx.scene_run(gray_h, bgr_h, cams, srcs, edges_h, labels_h, seed=7, memory=D.MEM_HOST, want_maps=True, **kw)
        e2e_times.append(time.perf_counter() - t0)
    d2h = V * H * W * (4 + 12 + 1 + 4) + res["points"] * 15
    e2e_s = statistics.median(e2e_times)
    if dist is not None:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = pix_step * world / e2e_s

    # accuracy of the final depth maps against the scene's ground truth
    rel = np.concatenate([np.abs(res["depth"][v] - sc.depth[v]).ravel() / sc.depth[v].ravel() for v in range(V)])
    valid = np.concatenate([(res["depth"][v] > 0).ravel() for v in range(V)])

    # the batched forms on the same scene (device-resident, 1 warm-up + 1 timed schedule each):
    # all views of a call in one batch (reading the previous call's depths), then additionally
    # FP16-staged sources and the Gauss-Newton plane hypothesis from the NCC adjoint
    def accuracy(r):
        rl = np.concatenate([np.abs(r["depth"][v] - sc.depth[v]).ravel() / sc.depth[v].ravel() for v in range(V)])
        ok = np.concatenate([(r["depth"][v] > 0).ravel() for v in range(V)])
        return float((rl[ok] < 0.01).mean()), float((rl[ok] < 0.001).mean())

    plain_acc = accuracy(res)
    forms = {}
    if not args.no_forms:
        for name, staging, gn in (("batched", D.STAGE_FP32, 0), ("batched_fp16_gn", D.STAGE_FP16, 1)):
            ctx.set_options(staging=staging, gn_refine=gn)
            ctx.scene_run(gray_d, bgr_d, cams, srcs, edges_d, labels_d, seed=7, memory=D.MEM_DEVICE, want_maps=False,
                          batch_views=True, **kw)
            torch.cuda.synchronize()
            r = ctx.scene_run(gray_d, bgr_d, cams, srcs, edges_d, labels_d, seed=7, memory=D.MEM_DEVICE,
                              want_maps=True, batch_views=True, **kw)
            ctx.set_options()
            fms = r["gpu_ms"]
            fv = pix_step * world / (fms / 1e3)
            a1, a01 = accuracy(r)
            forms[name] = dict(value=round(fv, 4), unit=UNIT, ms_per_step=round(fms, 3), vs_plain=round(fv / value, 3),
                               depth_within_1pct=round(a1, 4), depth_within_0_1pct=round(a01, 4),
                               staging={D.STAGE_FP32: "fp32", D.STAGE_FP16: "fp16"}[staging],
                               gauss_newton=bool(gn), points=int(r["points"]))

    # roofline of the dominant kernel (device time share in the timed region)
    dom = max(stats.items(), key=lambda kv: kv[1]["ms"])
    dname, dstat = dom
    c = counted.get(dname, {})
    flop_per_step = c.get("strong_ncc_evals", 0) * STRONG_NCC_FLOP + c.get("weak_ncc_evals", 0) * WEAK_NCC_FLOP
    launches_per_step = max(1, dstat["launches"] // max(1, args.steps))
    ms_per_launch = dstat["ms"] / max(1, dstat["launches"])
    flop_per_launch = flop_per_step / launches_per_step
    achieved = flop_per_launch / (ms_per_launch * 1e-3) / 1e12 if ms_per_launch > 0 else 0.0
    total_kernel_ms = sum(k["ms"] for k in stats.values())
    roofline = dict(kernel=dname, bound="fp32", achieved=round(achieved, 3), peak=round(fp32_peak, 3), unit="TFLOP/s",
                    frac=round(achieved / fp32_peak, 4) if fp32_peak > 0 else None, traffic=_traffic_for(dname),
                    peak_source="measured FP32 FMA throughput on this GPU (dpe_fp32_peak); MEASURED_PEAKS.json has no "
                                "FP32 figure", share_of_kernel_time=round(dstat["ms"] / total_kernel_ms, 4),
                    flop_per_launch=flop_per_launch, ms_per_launch=round(ms_per_launch, 4))
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        import multiprocessing

        threads = multiprocessing.cpu_count()
        s = cpu_sample(threads)
        cpu = dict(value=round(pix_step / s["schedule_s"], 6), unit=UNIT, cores=threads, kind="port",
                   sample=f"oracle FIRST_INIT {s['t_init']:.2f}s + geom REFINE_ITER {s['t_refine']:.2f}s of one view at "
                          f"400x300 x 10 images, scaled by pixels to the 3-level x 10-view x 2-call schedule")
    line = dict(metric=METRIC, value=round(value, 4), unit=UNIT, n_gpus=world, steps=args.steps, warmup=args.warmup,
                ms_per_step=round(ms_per_step, 3), higher_is_better=True, scaling="weak", vs_baseline=None,
                dtype="f32", data="synthetic (seeded ray-cast scene in place of ETH3D)",
                config=dict(workload="c2 full pipeline: 10 views 1600x1200, 3 levels, init + 1 geom call per level, "
                                     "3 iterations, fusion min 2 views", parallelism=f"replicas{world}",
                            l2="inputs and state larger than L2 (no flush)", **WORKLOAD),
                ncc_evals_per_s=round((evals_strong + evals_weak) * world / (ms_per_step / 1e3), 1),
                strong_ncc_evals_per_step=evals_strong, weak_ncc_evals_per_step=evals_weak,
                points=int(last["points"]), fusion_ms=round(last["fusion_ms"], 3), wall_s_timed=round(wall, 3),
                depth_within_1pct=round(float((rel[valid] < 0.01).mean()), 4),
                depth_within_0_1pct=round(float((rel[valid] < 0.001).mean()), 4),
                valid_depth_fraction=round(float(valid.mean()), 4),
                roofline=roofline, cpu_baseline=cpu, clocks=clocks.summary(), gpu_launches=int(launches),
                e2e=dict(value=round(e2e_value, 4), unit=UNIT, h2d_bytes_per_step=int(h2d), d2h_bytes_per_step=int(d2h)),
                kernel_ms_per_step={k: round(v["ms"] / max(1, args.steps), 3) for k, v in
                                    sorted(stats.items(), key=lambda kv: -kv[1]["ms"])},
                forms=forms or None)
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the batched / FP16 / Gauss-Newton forms")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
