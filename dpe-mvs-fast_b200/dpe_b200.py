"""Python binding of the C ABI in include/dpe_b200.h (ctypes; no torch types cross the boundary).

This is the host-side mirror of the reference's per-view interface (class DPE, DPE.h:140-243, and
RunFusion, DPE.h:95-96) used by the tests and the bench.  The library is the in-tree
libdpe_sm100.so; loading fails loudly when it is missing -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# DPE_LIBRARY selects another in-tree build (e.g. the bounds-checked libdpe_sm100_checked.so)
LIB_PATH = os.path.join(HERE, os.environ.get("DPE_LIBRARY", "libdpe_sm100.so"))
# the same kernels built without multiply-add contraction: the CPU oracle's arithmetic, bit for bit
EXACT_LIBRARY = "libdpe_sm100_exact.so"

MAX_IMAGES = 32
NEIGHBOUR_NUM = 9
OK, ERR_INVALID_ARGUMENT, ERR_CUDA, ERR_OUT_OF_MEMORY, ERR_CAPACITY, ERR_NO_DEVICE, ERR_DEVICE_TIMEOUT = range(7)
WEAK, STRONG, UNKNOWN = 0, 1, 2
FIRST_INIT, REFINE_INIT, REFINE_ITER = 0, 1, 2
MEM_HOST, MEM_DEVICE = 0, 1
FUSE_FP64, FUSE_FLOAT = 0, 1
TAT_INTERMEDIATE, TAT_ADVANCED = 0, 1
STAGE_FP32, STAGE_FP16, STAGE_BF16 = 0, 1, 2


class Camera(C.Structure):
    _fields_ = [("K", C.c_float * 9), ("R", C.c_float * 9), ("t", C.c_float * 3), ("c", C.c_float * 3),
                ("height", C.c_int), ("width", C.c_int), ("depth_min", C.c_float), ("depth_max", C.c_float)]


class Params(C.Structure):
    _fields_ = [(n, t) for n, t in [
        ("max_iterations", C.c_int), ("num_images", C.c_int), ("sigma_spatial", C.c_float),
        ("sigma_color", C.c_float), ("top_k", C.c_int), ("depth_min", C.c_float), ("depth_max", C.c_float),
        ("geom_consistency", C.c_int), ("strong_radius", C.c_int), ("strong_increment", C.c_int),
        ("weak_radius", C.c_int), ("weak_increment", C.c_int), ("use_APD", C.c_int), ("use_edge", C.c_int),
        ("use_limit", C.c_int), ("use_label", C.c_int), ("use_radius", C.c_int), ("high_res_img", C.c_int),
        ("max_scale_size", C.c_int), ("scale_size", C.c_int), ("weak_peak_radius", C.c_int),
        ("rotate_time", C.c_int), ("ransac_threshold", C.c_float), ("geom_factor", C.c_float), ("state", C.c_int)]]


class Problem(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("num_images", C.c_int),
                ("images", C.c_void_p * MAX_IMAGES), ("cameras", Camera * MAX_IMAGES), ("params", Params),
                ("plane_in", C.c_void_p), ("selected_views_in", C.c_void_p), ("weak_in", C.c_void_p),
                ("edge", C.c_void_p), ("edge_low_res", C.c_void_p), ("low_width", C.c_int), ("low_height", C.c_int),
                ("label", C.c_void_p), ("depths", C.c_void_p * MAX_IMAGES), ("seed", C.c_uint64), ("memory", C.c_int)]


class PMOut(C.Structure):
    _fields_ = [("plane", C.c_void_p), ("weak", C.c_void_p), ("selected_views", C.c_void_p), ("costs", C.c_void_p),
                ("gpu_ms", C.c_float), ("strong_ncc_evals", C.c_uint64), ("weak_ncc_evals", C.c_uint64)]


class FusionView(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("depth", C.c_void_p), ("normal", C.c_void_p),
                ("weak", C.c_void_p), ("bgr", C.c_void_p), ("block_mask", C.c_void_p), ("camera", Camera),
                ("num_src", C.c_int), ("src_views", C.c_void_p)]


class FusionIn(C.Structure):
    _fields_ = [("num_views", C.c_int), ("views", C.POINTER(FusionView)), ("mode", C.c_int), ("memory", C.c_int),
                ("min_consistent", C.c_int)]


class FusionOut(C.Structure):
    _fields_ = [("capacity", C.c_int64), ("count", C.c_int64), ("xyz", C.c_void_p), ("bgr", C.c_void_p),
                ("origin", C.c_void_p), ("num_consistent", C.c_void_p), ("gpu_ms", C.c_float)]


class NCCQuery(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("num_images", C.c_int),
                ("images", C.c_void_p * MAX_IMAGES), ("cameras", Camera * MAX_IMAGES), ("params", Params),
                ("count", C.c_int64), ("px", C.c_void_p), ("py", C.c_void_p), ("src", C.c_void_p), ("plane", C.c_void_p)]


class SceneView(C.Structure):
    _fields_ = [("gray", C.c_void_p), ("bgr", C.c_void_p), ("camera", Camera), ("num_src", C.c_int),
                ("src_views", C.c_void_p), ("edges", C.POINTER(C.c_void_p)), ("labels", C.POINTER(C.c_void_p))]


class Schedule(C.Structure):
    _fields_ = [("num_levels", C.c_int), ("refine_calls", C.c_int), ("max_iterations", C.c_int),
                ("fuse_mode", C.c_int), ("min_consistent", C.c_int), ("seed", C.c_uint64), ("batch_views", C.c_int),
                ("device_edges", C.c_int), ("device_labels", C.c_int)]


class KernelStat(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("launches", C.c_int64), ("ms", C.c_double),
                ("strong_ncc_evals", C.c_uint64), ("weak_ncc_evals", C.c_uint64)]


class TuningEntry(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("size_class", C.c_int), ("candidates", C.c_int), ("chosen", C.c_int),
                ("block_x", C.c_int), ("block_y", C.c_int), ("carveout", C.c_int), ("mean_ms", C.c_float * 8)]


class SceneIn(C.Structure):
    _fields_ = [("num_views", C.c_int), ("width", C.c_int), ("height", C.c_int), ("views", C.POINTER(SceneView)),
                ("memory", C.c_int)]


class SceneOut(C.Structure):
    _fields_ = [("depth", C.POINTER(C.c_void_p)), ("normal", C.POINTER(C.c_void_p)), ("weak", C.POINTER(C.c_void_p)),
                ("selected_views", C.POINTER(C.c_void_p)), ("out_memory", C.c_int), ("fusion", FusionOut),
                ("gpu_ms", C.c_float), ("fusion_ms", C.c_float), ("num_levels", C.c_int), ("calls", C.c_int)]


class SparseModel(C.Structure):
    _fields_ = [("num_images", C.c_int), ("centers", C.c_void_p), ("obs_offsets", C.c_void_p),
                ("obs_point", C.c_void_p), ("num_points", C.c_int64), ("points", C.c_void_p)]


class Options(C.Structure):
    _fields_ = [("staging", C.c_int), ("gn_refine", C.c_int)]


class Limits(C.Structure):
    _fields_ = [("max_width", C.c_int), ("max_height", C.c_int), ("max_images", C.c_int)]


EXPORTED = ["dpe_status_string", "dpe_last_error", "dpe_params_default", "dpe_ctx_create", "dpe_ctx_destroy", "dpe_pm_run",
            "dpe_fuse", "dpe_ncc_eval", "dpe_ctx_set_eval_counting", "dpe_scene_run", "dpe_ctx_set_profiling",
            "dpe_ctx_reset_kernel_stats", "dpe_ctx_get_kernel_stats", "dpe_launch_count", "dpe_fp32_peak",
            "dpe_ncc_eval_noalloc", "dpe_ncc_grad", "dpe_ctx_set_options", "dpe_pm_run_batch", "dpe_fuse_tat", "dpe_edge_map", "dpe_edge_labels",
            "dpe_view_scores", "dpe_ncc_grad_device", "dpe_ctx_set_autotune", "dpe_ctx_get_tuning"]

_lib = None


def load_library(path: Optional[str] = None) -> C.CDLL:
    """Load libdpe_sm100.so (built by build.py).  Raises when it is missing: no fallback path."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"{p} is missing: build it with `python dpe-mvs-fast_b200/build.py`")
    lib = C.CDLL(p)
    lib.dpe_status_string.restype = C.c_char_p
    lib.dpe_status_string.argtypes = [C.c_int]
    lib.dpe_last_error.restype = C.c_char_p
    lib.dpe_last_error.argtypes = []
    lib.dpe_params_default.argtypes = [C.POINTER(Params)]
    lib.dpe_ctx_create.argtypes = [C.c_int, C.POINTER(Limits), C.POINTER(C.c_void_p)]
    lib.dpe_ctx_destroy.argtypes = [C.c_void_p]
    lib.dpe_pm_run.argtypes = [C.c_void_p, C.POINTER(Problem), C.POINTER(PMOut)]
    lib.dpe_fuse.argtypes = [C.c_void_p, C.POINTER(FusionIn), C.POINTER(FusionOut)]
    lib.dpe_fuse_tat.argtypes = [C.c_void_p, C.POINTER(FusionIn), C.c_int, C.POINTER(FusionOut)]
    lib.dpe_edge_map.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]
    lib.dpe_edge_labels.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
    lib.dpe_ncc_eval.argtypes = [C.c_void_p, C.POINTER(NCCQuery), C.c_void_p]
    lib.dpe_ctx_set_eval_counting.argtypes = [C.c_void_p, C.c_int]
    lib.dpe_scene_run.argtypes = [C.c_void_p, C.POINTER(SceneIn), C.POINTER(Schedule), C.POINTER(SceneOut)]
    lib.dpe_ctx_set_profiling.argtypes = [C.c_void_p, C.c_int]
    lib.dpe_ctx_reset_kernel_stats.argtypes = [C.c_void_p]
    lib.dpe_ctx_get_kernel_stats.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int)]
    lib.dpe_ctx_set_autotune.argtypes = [C.c_void_p, C.c_int]
    lib.dpe_ctx_get_tuning.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int)]
    lib.dpe_launch_count.restype = C.c_uint64
    lib.dpe_launch_count.argtypes = []
    lib.dpe_fp32_peak.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    lib.dpe_ncc_eval_noalloc.argtypes = [C.POINTER(NCCQuery), C.c_void_p, C.c_void_p]
    lib.dpe_view_scores.argtypes = [C.c_void_p, C.POINTER(SparseModel), C.c_void_p]
    lib.dpe_ncc_grad_device.argtypes = [C.c_void_p, C.POINTER(NCCQuery), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p]
    lib.dpe_ctx_set_options.argtypes = [C.c_void_p, C.POINTER(Options)]
    lib.dpe_pm_run_batch.argtypes = [C.c_void_p, C.POINTER(Problem), C.c_int, C.POINTER(PMOut)]
    lib.dpe_ncc_grad.argtypes = [C.c_void_p, C.POINTER(NCCQuery), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    if path is None:
        _lib = lib
    return lib


class DPEError(RuntimeError):
    def __init__(self, status: int, what: str):
        lib = load_library()
        detail = lib.dpe_last_error().decode() if status in (ERR_CUDA, ERR_OUT_OF_MEMORY) else ""
        super().__init__(f"{what}: {lib.dpe_status_string(status).decode()} (status {status}) {detail}".rstrip())
        self.status = status


def default_params(lib: Optional[C.CDLL] = None) -> Params:
    p = Params()
    (lib or load_library()).dpe_params_default(C.byref(p))
    return p


def reference_default_params() -> Params:
    """PatchMatchParams' member defaults (main.h:81-109) without loading the library (what
    dpe_params_default returns; a CPU test holds the two equal)."""
    p = Params()
    for k, v in dict(max_iterations=3, num_images=5, sigma_spatial=5.0, sigma_color=3.0, top_k=4, depth_min=0.0,
                     depth_max=1.0, geom_consistency=0, strong_radius=5, strong_increment=2, weak_radius=5,
                     weak_increment=5, use_APD=1, use_edge=1, use_limit=1, use_label=1, use_radius=1, high_res_img=1,
                     max_scale_size=1, scale_size=1, weak_peak_radius=2, rotate_time=4, ransac_threshold=0.005,
                     geom_factor=0.2, state=FIRST_INIT).items():
        setattr(p, k, v)
    return p


def make_camera(d: Dict) -> Camera:
    cam = Camera()
    for name in ("K", "R", "t", "c"):
        arr = np.asarray(d[name], dtype=np.float32).reshape(-1)
        getattr(cam, name)[:] = arr.tolist()
    cam.height = int(d["height"])
    cam.width = int(d["width"])
    cam.depth_min = float(d["depth_min"])
    cam.depth_max = float(d["depth_max"])
    return cam


def _ptr(x) -> Optional[int]:
    """Raw address of a C-contiguous numpy array or a CUDA tensor (anything with data_ptr())."""
    if x is None:
        return None
    if hasattr(x, "data_ptr"):
        return int(x.data_ptr())
    assert isinstance(x, np.ndarray) and x.flags["C_CONTIGUOUS"], "arrays must be C-contiguous"
    return int(x.ctypes.data)


def build_problem(images: Sequence, cameras: Sequence[Dict], params: Params, *, plane_in=None, views_in=None,
                  weak_in=None, edge=None, edge_low=None, label=None, depths=None, seed: int = 0,
                  memory: int = MEM_HOST) -> Problem:
    n = len(images)
    pr = Problem()
    shape = images[0].shape
    pr.height, pr.width = int(shape[0]), int(shape[1])
    pr.num_images = n
    for i in range(n):
        pr.images[i] = _ptr(images[i])
        pr.cameras[i] = make_camera(cameras[i])
        if depths is not None:
            pr.depths[i] = _ptr(depths[i])
    pr.params = params
    pr.params.num_images = n
    pr.plane_in = _ptr(plane_in)
    pr.selected_views_in = _ptr(views_in)
    pr.weak_in = _ptr(weak_in)
    pr.edge = _ptr(edge)
    if edge_low is not None:
        pr.edge_low_res = _ptr(edge_low)
        pr.low_height, pr.low_width = int(edge_low.shape[0]), int(edge_low.shape[1])
    pr.label = _ptr(label)
    pr.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    pr.memory = memory
    return pr


def fusion_input(views: List[Dict], mode: int, memory: int, min_consistent: int, capacity: Optional[int]):
    """dpe_fusion_in for a list of views (dicts with depth, normal, bgr, camera, src and optional
    weak and block); returns it, the arrays it points into, and the point capacity (default: every
    pixel)."""
    arr = (FusionView * len(views))()
    keep = [arr]
    total = 0
    for i, v in enumerate(views):
        fv = arr[i]
        H, W = v["depth"].shape[:2]
        fv.width, fv.height = W, H
        fv.depth = _ptr(v["depth"])
        fv.normal = _ptr(v["normal"])
        fv.weak = _ptr(v.get("weak"))
        fv.bgr = _ptr(v["bgr"])
        fv.block_mask = _ptr(v.get("block"))
        fv.camera = make_camera(v["camera"])
        src = np.ascontiguousarray(np.asarray(v["src"], dtype=np.int32))
        keep.append(src)
        fv.num_src = len(src)
        fv.src_views = _ptr(src) if len(src) else None
        total += W * H
    cap = total if capacity is None else capacity
    return FusionIn(len(views), arr, mode, memory, min_consistent), keep, cap


def fusion_output(cap: int):
    """dpe_fusion_out with host buffers for `cap` points (xyz, bgr, origin, num_consistent)."""
    arrays = dict(xyz=np.zeros((max(cap, 1), 3), np.float32), bgr=np.zeros((max(cap, 1), 3), np.uint8),
                  origin=np.zeros((max(cap, 1), 2), np.int32), num_consistent=np.zeros(max(cap, 1), np.uint8))
    fo = FusionOut()
    fo.capacity = cap
    fo.xyz, fo.bgr = _ptr(arrays["xyz"]), _ptr(arrays["bgr"])
    fo.origin, fo.num_consistent = _ptr(arrays["origin"]), _ptr(arrays["num_consistent"])
    return fo, arrays


def fusion_result(fo, arrays: Dict, **extra) -> Dict:
    n = int(fo.count)
    k = min(n, int(fo.capacity))
    return dict(count=n, **{name: a[:k] for name, a in arrays.items()}, **extra)


class Context:
    """A dpe_ctx on one device."""

    def __init__(self, device: int = 0, library: Optional[str] = None):
        """library: another in-tree build by file name (e.g. EXACT_LIBRARY), default the main one."""
        self.lib = load_library(os.path.join(HERE, library)) if library else load_library()
        h = C.c_void_p()
        st = self.lib.dpe_ctx_create(device, None, C.byref(h))
        if st != OK:
            raise DPEError(st, "dpe_ctx_create")
        self.handle = h
        # DPE_AUTOTUNE=0 turns the launch tuner off for every context (fixed default settings)
        if os.environ.get("DPE_AUTOTUNE") == "0" and hasattr(self.lib, "dpe_ctx_set_autotune"):
            self.lib.dpe_ctx_set_autotune(self.handle, 0)

    def close(self):
        if getattr(self, "handle", None):
            self.lib.dpe_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_eval_counting(self, on: bool):
        self.lib.dpe_ctx_set_eval_counting(self.handle, 1 if on else 0)

    def set_profiling(self, on: bool):
        self.lib.dpe_ctx_set_profiling(self.handle, 1 if on else 0)

    def reset_kernel_stats(self):
        self.lib.dpe_ctx_reset_kernel_stats(self.handle)

    def kernel_stats(self) -> Dict[str, Dict]:
        arr = (KernelStat * 64)()
        n = C.c_int()
        st = self.lib.dpe_ctx_get_kernel_stats(self.handle, arr, 64, C.byref(n))
        if st not in (OK, ERR_CAPACITY):
            raise DPEError(st, "dpe_ctx_get_kernel_stats")
        return {arr[i].name.decode(): dict(launches=int(arr[i].launches), ms=float(arr[i].ms),
                                           strong_ncc_evals=int(arr[i].strong_ncc_evals),
                                           weak_ncc_evals=int(arr[i].weak_ncc_evals)) for i in range(min(n.value, 64))}

    def set_autotune(self, on: bool):
        """The launch tuner (dpe_ctx_set_autotune): on by default."""
        st = self.lib.dpe_ctx_set_autotune(self.handle, 1 if on else 0)
        if st != OK:
            raise DPEError(st, "dpe_ctx_set_autotune")

    def tuning(self) -> List[Dict]:
        """The tuner's table (dpe_ctx_get_tuning): per kernel and size class the candidates' mean
        times and the kept setting."""
        arr = (TuningEntry * 256)()
        n = C.c_int()
        st = self.lib.dpe_ctx_get_tuning(self.handle, arr, 256, C.byref(n))
        if st not in (OK, ERR_CAPACITY):
            raise DPEError(st, "dpe_ctx_get_tuning")
        out = []
        for i in range(min(n.value, 256)):
            e = arr[i]
            out.append(dict(kernel=e.name.decode(), size_class=e.size_class, candidates=e.candidates, chosen=e.chosen,
                            block=(e.block_x, e.block_y), carveout=e.carveout,
                            mean_ms=[round(float(e.mean_ms[k]), 4) for k in range(e.candidates)]))
        return out

    def fp32_peak_tflops(self) -> float:
        v = C.c_double()
        st = self.lib.dpe_fp32_peak(self.handle, C.byref(v))
        if st != OK:
            raise DPEError(st, "dpe_fp32_peak")
        return float(v.value)

    # ------------------------------------------------------------------ PatchMatch
    def pm_run(self, images, cameras, params: Params, *, out=None, want_costs=True, **kw) -> Dict:
        """One per-view call on host arrays (memory=MEM_HOST) or device tensors (memory=MEM_DEVICE)."""
        memory = kw.get("memory", MEM_HOST)
        pr = build_problem(images, cameras, params, **kw)
        H, W = pr.height, pr.width
        if out is None:
            assert memory == MEM_HOST, "device calls pass preallocated outputs"
            out = dict(plane=np.zeros((H, W, 4), np.float32), weak=np.zeros((H, W), np.uint8),
                       views=np.zeros((H, W), np.uint32), costs=np.zeros((H, W), np.float32) if want_costs else None)
        po = PMOut()
        po.plane = _ptr(out["plane"])
        po.weak = _ptr(out["weak"])
        po.selected_views = _ptr(out["views"])
        po.costs = _ptr(out.get("costs"))
        st = self.lib.dpe_pm_run(self.handle, C.byref(pr), C.byref(po))
        if st != OK:
            raise DPEError(st, "dpe_pm_run")
        out["gpu_ms"] = po.gpu_ms
        out["strong_ncc_evals"] = int(po.strong_ncc_evals)
        out["weak_ncc_evals"] = int(po.weak_ncc_evals)
        return out

    def pm_run_batch(self, calls: List[Dict]) -> List[Dict]:
        """dpe_pm_run_batch on host arrays: each call a dict(images=, cameras=, params=, **pm_run keywords)."""
        n = len(calls)
        probs = (Problem * n)()
        outs = (PMOut * n)()
        results = []
        for b, c in enumerate(calls):
            kw = {k: v for k, v in c.items() if k not in ("images", "cameras", "params")}
            probs[b] = build_problem(c["images"], c["cameras"], c["params"], **kw)
            H, W = probs[b].height, probs[b].width
            o = dict(plane=np.zeros((H, W, 4), np.float32), weak=np.zeros((H, W), np.uint8),
                     views=np.zeros((H, W), np.uint32), costs=np.zeros((H, W), np.float32))
            outs[b].plane, outs[b].weak = _ptr(o["plane"]), _ptr(o["weak"])
            outs[b].selected_views, outs[b].costs = _ptr(o["views"]), _ptr(o["costs"])
            results.append(o)
        st = self.lib.dpe_pm_run_batch(self.handle, probs, n, outs)
        if st != OK:
            raise DPEError(st, "dpe_pm_run_batch")
        for b in range(n):
            results[b]["gpu_ms"] = outs[b].gpu_ms
        return results

    # ------------------------------------------------------------------ fusion
    def fuse(self, views: List[Dict], mode: int = FUSE_FP64, capacity: Optional[int] = None,
             memory: int = MEM_HOST, min_consistent: int = 1) -> Dict:
        """RunFusion (DPE.cpp:1387-1548) through dpe_fuse."""
        fin, keep, cap = fusion_input(views, mode, memory, min_consistent, capacity)
        fo, arrays = fusion_output(cap)
        st = self.lib.dpe_fuse(self.handle, C.byref(fin), C.byref(fo))
        if st != OK:
            raise DPEError(st, "dpe_fuse")
        return fusion_result(fo, arrays, gpu_ms=fo.gpu_ms)

    def fuse_tat(self, views: List[Dict], variant: int = TAT_INTERMEDIATE, mode: int = FUSE_FLOAT,
                 capacity: Optional[int] = None, memory: int = MEM_HOST) -> Dict:
        """RunFusion_TAT_Intermediate / RunFusion_TAT_advanced (DPE.cpp:1550-1867) through
        dpe_fuse_tat; the views' "weak" maps are not needed."""
        fin, keep, cap = fusion_input(views, mode, memory, 1, capacity)
        fo, arrays = fusion_output(cap)
        st = self.lib.dpe_fuse_tat(self.handle, C.byref(fin), variant, C.byref(fo))
        if st != OK:
            raise DPEError(st, "dpe_fuse_tat")
        return fusion_result(fo, arrays, gpu_ms=fo.gpu_ms)

    # ------------------------------------------------------------------ edge maps
    def edge_map(self, image, memory: int = MEM_HOST):
        """EdgeSegment's edge map (mode 0, Canny) of an 8-bit image through dpe_edge_map: a numpy
        uint8 array (memory=MEM_HOST) or a CUDA uint8 tensor (MEM_DEVICE); returns the same kind."""
        H, W = image.shape[:2]
        if memory == MEM_HOST:
            img = np.ascontiguousarray(image, dtype=np.uint8)
            out = np.zeros((H, W), np.uint8)
        else:
            import torch

            img = image.contiguous()
            out = torch.empty((H, W), dtype=torch.uint8, device=image.device)
        st = self.lib.dpe_edge_map(self.handle, _ptr(img), W, H, memory, _ptr(out))
        if st != OK:
            raise DPEError(st, "dpe_edge_map")
        return out

    def edge_labels(self, gray, scale: int, high_res_img: bool = True, memory: int = MEM_HOST):
        """EdgeSegment's label map (mode 1) of a full-resolution 8-bit image through dpe_edge_labels:
        int32 labels at the level size of `scale` (0 edges, -1 small regions), as numpy
        (memory=MEM_HOST) or as a CUDA tensor (MEM_DEVICE)."""
        H, W = gray.shape[:2]
        f = np.float32(1.0) / np.float32(1 << scale)
        w, h = int(np.round(np.float32(W) * f)), int(np.round(np.float32(H) * f))
        if memory == MEM_HOST:
            img = np.ascontiguousarray(gray, dtype=np.uint8)
            out = np.zeros((h, w), np.int32)
        else:
            import torch

            img = gray.contiguous()
            out = torch.empty((h, w), dtype=torch.int32, device=gray.device)
        st = self.lib.dpe_edge_labels(self.handle, _ptr(img), W, H, scale, 1 if high_res_img else 0, memory, _ptr(out))
        if st != OK:
            raise DPEError(st, "dpe_edge_labels")
        return out

    # ------------------------------------------------------------------ whole scene
    def scene_run(self, gray, bgr, cameras, srcs, edges=None, labels=None, *, num_levels=0, refine_calls=3,
                  max_iterations=3, fuse_mode=FUSE_FP64, min_consistent=1, seed=1, memory=MEM_HOST,
                  want_maps=True, point_capacity=None, batch_views=False, device_edges=False,
                  device_labels=False, want_consistency=False) -> Dict:
        """The reference's full schedule over all views (dpe_scene_run).  gray[v]: (H, W) uint8,
        bgr[v]: (H, W, 3) uint8, cameras[v]: full-resolution camera dicts, srcs[v]: source view
        indices, edges[v][level] / labels[v][level]: per-level maps (level 0 = coarsest).
        device_edges=True / device_labels=True: the edge / label maps are made on the device (edges /
        labels must then be None)."""
        V = len(gray)
        H, W = int(gray[0].shape[0]), int(gray[0].shape[1])
        arr = (SceneView * V)()
        keep = []
        for v in range(V):
            sv = arr[v]
            sv.gray = _ptr(gray[v])
            sv.bgr = _ptr(bgr[v]) if bgr is not None else None
            sv.camera = make_camera(cameras[v])
            src = np.ascontiguousarray(np.asarray(srcs[v], dtype=np.int32))
            keep.append(src)
            sv.num_src = len(src)
            sv.src_views = _ptr(src)
            if edges is not None:
                ea = (C.c_void_p * len(edges[v]))(*[_ptr(e) for e in edges[v]])
                keep.append(ea)
                sv.edges = C.cast(ea, C.POINTER(C.c_void_p))
            if labels is not None:
                la = (C.c_void_p * len(labels[v]))(*[_ptr(x) for x in labels[v]])
                keep.append(la)
                sv.labels = C.cast(la, C.POINTER(C.c_void_p))
        sc = SceneIn(V, W, H, arr, memory)
        sch = Schedule(num_levels, refine_calls, max_iterations, fuse_mode if fuse_mode is not None else -1,
                       min_consistent, seed, 1 if batch_views else 0, 1 if device_edges else 0,
                       1 if device_labels else 0)
        so = SceneOut()
        so.out_memory = MEM_HOST
        res = {}
        if want_maps:
            res["depth"] = [np.zeros((H, W), np.float32) for _ in range(V)]
            res["normal"] = [np.zeros((H, W, 3), np.float32) for _ in range(V)]
            res["weak"] = [np.zeros((H, W), np.uint8) for _ in range(V)]
            res["views"] = [np.zeros((H, W), np.uint32) for _ in range(V)]
            for key, field in (("depth", "depth"), ("normal", "normal"), ("weak", "weak"), ("views", "selected_views")):
                pa = (C.c_void_p * V)(*[_ptr(x) for x in res[key]])
                keep.append(pa)
                setattr(so, field, C.cast(pa, C.POINTER(C.c_void_p)))
        cap = V * H * W if point_capacity is None else point_capacity
        xyz = np.zeros((max(cap, 1), 3), np.float32)
        rgb = np.zeros((max(cap, 1), 3), np.uint8)
        so.fusion.capacity = cap
        so.fusion.xyz, so.fusion.bgr = _ptr(xyz), _ptr(rgb)
        ncons = np.zeros(max(cap, 1), np.uint8) if want_consistency else None
        so.fusion.num_consistent = _ptr(ncons)
        st = self.lib.dpe_scene_run(self.handle, C.byref(sc), C.byref(sch), C.byref(so))
        if st != OK:
            raise DPEError(st, "dpe_scene_run")
        n = int(so.fusion.count)
        res.update(points=n, xyz=xyz[:n], bgr=rgb[:n], gpu_ms=so.gpu_ms, fusion_ms=so.fusion_ms,
                   num_levels=so.num_levels, calls=so.calls)
        if want_consistency:
            res["num_consistent"] = ncons[:n]
        return res

    # ------------------------------------------------------------------ view selection
    def view_scores(self, centers, obs_offsets, obs_point, points) -> np.ndarray:
        """dpe_view_scores: the pair score matrix (N, N) of calc_score (colmap2mvsnet.py:280-302)."""
        centers = np.ascontiguousarray(centers, np.float64).reshape(-1, 3)
        obs_offsets = np.ascontiguousarray(obs_offsets, np.int64)
        obs_point = np.ascontiguousarray(obs_point, np.int32)
        points = np.ascontiguousarray(points, np.float64).reshape(-1, 3)
        n = centers.shape[0]
        m = SparseModel(n, _ptr(centers), _ptr(obs_offsets), _ptr(obs_point) if obs_point.size else None,
                        points.shape[0], _ptr(points) if points.size else None)
        out = np.zeros((n, n), np.float64)
        st = self.lib.dpe_view_scores(self.handle, C.byref(m), _ptr(out))
        if st != OK:
            raise DPEError(st, "dpe_view_scores")
        return out

    # ------------------------------------------------------------------ NCC queries
    def set_options(self, staging: int = STAGE_FP32, gn_refine: int = 0) -> None:
        """dpe_ctx_set_options: source-image staging (STAGE_*) and the Gauss-Newton hypothesis."""
        st = self.lib.dpe_ctx_set_options(self.handle, C.byref(Options(staging, gn_refine)))
        if st != OK:
            raise DPEError(st, "dpe_ctx_set_options")

    def ncc_grad(self, images, cameras, params: Params, px, py, src, planes, want_images: bool = False):
        """dpe_ncc_grad: (cost (n,), dC/d(n, w) (n, 4), dC/d(depth, n) (n, 4), image gradients or None)."""
        q = make_query(images, cameras, params, px, py, src, planes)
        n = len(q.keep[0])
        cost = np.zeros(n, np.float32)
        gp = np.zeros((n, 4), np.float32)
        gd = np.zeros((n, 4), np.float32)
        gimg, ptrs = None, None
        if want_images:
            H, W = images[0].shape
            gimg = [None] + [np.zeros((H, W), np.float32) for _ in images[1:]]
            ptrs = (C.c_void_p * len(images))(*([None] + [g.ctypes.data for g in gimg[1:]]))
        st = self.lib.dpe_ncc_grad(self.handle, C.byref(q.struct), _ptr(cost), _ptr(gp), _ptr(gd), ptrs)
        if st != OK:
            raise DPEError(st, "dpe_ncc_grad")
        return cost, gp, gd, gimg

    def ncc_eval(self, images, cameras, params: Params, px, py, src, planes) -> np.ndarray:
        q = make_query(images, cameras, params, px, py, src, planes)
        out = np.zeros(len(q.keep[0]), np.float32)
        st = self.lib.dpe_ncc_eval(self.handle, C.byref(q.struct), _ptr(out))
        if st != OK:
            raise DPEError(st, "dpe_ncc_eval")
        return out


def ncc_eval_noalloc(images, cameras, params: Params, px, py, src, planes, costs_out, stream=None, lib=None):
    """dpe_ncc_eval_noalloc: every array a CUDA tensor on the current device (images float32 (H, W),
    px/py/src int32 (n,), planes float32 (n, 4), costs_out float32 (n,)).  The work is enqueued on
    `stream` (a torch.cuda.Stream, default: torch's current stream) and not waited for."""
    import torch

    lib = lib or load_library()
    if not 2 <= len(images) <= MAX_IMAGES or len(cameras) != len(images):
        raise ValueError(f"need 2..{MAX_IMAGES} images and one camera per image")
    if images[0].dim() != 2:
        raise ValueError("images must be 2-D (H, W) tensors")
    shape, device = tuple(images[0].shape), images[0].device
    q = NCCQuery()
    q.height, q.width = int(shape[0]), int(shape[1])
    q.num_images = len(images)
    for i, im in enumerate(images):
        if not (im.is_cuda and im.dtype == torch.float32 and im.is_contiguous()):
            raise ValueError("images must be contiguous float32 CUDA tensors")
        if tuple(im.shape) != shape or im.device != device:
            raise ValueError(f"image {i} has shape {tuple(im.shape)} on {im.device}; every image must be "
                             f"{shape} on {device}")
        q.images[i] = im.data_ptr()
        q.cameras[i] = make_camera(cameras[i])
    q.params = params
    n = int(px.numel())
    for name, t, dt, want in (("px", px, torch.int32, (n,)), ("py", py, torch.int32, (n,)),
                              ("src", src, torch.int32, (n,)), ("planes", planes, torch.float32, (n, 4)),
                              ("costs_out", costs_out, torch.float32, (n,))):
        if not (t.is_cuda and t.dtype == dt and t.is_contiguous()):
            raise ValueError("queries and output must be contiguous CUDA tensors of the documented types")
        if tuple(t.shape) != want:
            raise ValueError(f"{name} has shape {tuple(t.shape)}, expected {want}")
        if t.device != device:
            raise ValueError(f"{name} is on {t.device}, the images on {device}")
    if device != torch.device("cuda", torch.cuda.current_device()):
        raise ValueError(f"the tensors are on {device}, the current device is cuda:{torch.cuda.current_device()}")
    q.count = n
    q.px, q.py, q.src, q.plane = px.data_ptr(), py.data_ptr(), src.data_ptr(), planes.data_ptr()
    s = (stream or torch.cuda.current_stream()).cuda_stream
    st = lib.dpe_ncc_eval_noalloc(C.byref(q), C.c_void_p(costs_out.data_ptr()), C.c_void_p(s))
    if st != OK:
        raise DPEError(st, "dpe_ncc_eval_noalloc")


class _Query:
    def __init__(self, struct, keep):
        self.struct = struct
        self.keep = keep


def make_query(images, cameras, params: Params, px, py, src, planes) -> _Query:
    q = NCCQuery()
    q.height, q.width = int(images[0].shape[0]), int(images[0].shape[1])
    q.num_images = len(images)
    for i, im in enumerate(images):
        q.images[i] = _ptr(im)
        q.cameras[i] = make_camera(cameras[i])
    q.params = params
    px = np.ascontiguousarray(px, dtype=np.int32)
    py = np.ascontiguousarray(py, dtype=np.int32)
    src = np.ascontiguousarray(src, dtype=np.int32)
    planes = np.ascontiguousarray(planes, dtype=np.float32).reshape(-1, 4)
    q.count = len(px)
    q.px, q.py, q.src, q.plane = _ptr(px), _ptr(py), _ptr(src), _ptr(planes)
    return _Query(q, [px, py, src, planes, images])
