"""ctypes binding of the reference's own code compiled for the CPU (oracle/_ref/libref.so).

TEST INFRASTRUCTURE ONLY: the reference-pinned oracle.  oracle/Makefile compiles the reference's
DPE.cu and DPE.cpp where they lie (they are never copied) behind the host stand-ins of
oracle/refshim/, and oracle/ref_harness.cpp drives them: `pm_call` runs one per-view call the way
ProcessProblem does (main.cpp:241-264), `fuse` runs RunFusion (DPE.cpp:1387-1548).  Tests compare
the restatement in oracle/ (oracle_py) with this on identical inputs and random streams; bench.py's
reference arm times it.  The library is built only where the reference sources are present; the
built file travels with the repository tree to machines without them.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
import tempfile
from typing import Dict, List

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "dpe-mvs-fast_b200"))
import dpe_b200 as D  # noqa: E402  (struct layouts of the shared ABI header; loads no library)

LIB_PATH = os.path.join(HERE, "_ref", "libref.so")
REFERENCE_DIR = os.environ.get("DPE_REFERENCE_DIR", "/root/reference")
_lib = None
ETH, TAT_INTERMEDIATE, TAT_ADVANCED = 0, 1, 2  # ref_fuse variants


def available() -> bool:
    return os.path.exists(LIB_PATH) or os.path.exists(os.path.join(REFERENCE_DIR, "DPE.cu"))


def build() -> str:
    if os.path.exists(os.path.join(REFERENCE_DIR, "DPE.cu")):
        subprocess.run(["make", "-s", "-C", HERE, f"REF={REFERENCE_DIR}", "_ref/libref.so"], check=True)
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH}: the reference sources are not here and no built library travelled")
    return LIB_PATH


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    lib.ref_last_error.restype = C.c_char_p
    lib.ref_pm_call.argtypes = [C.POINTER(D.Problem), C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                C.c_void_p, C.c_void_p, C.POINTER(D.Camera), C.POINTER(D.Params), C.POINTER(C.c_longlong)]
    lib.ref_fuse.argtypes = [C.POINTER(D.FusionIn), C.c_int, C.c_char_p, C.c_void_p, C.c_void_p, C.c_int64,
                             C.POINTER(C.c_int64)]
    lib.ref_set_texture_8bit_weights.argtypes = [C.c_int]
    lib.ref_connect.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    lib.ref_roberts.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    _lib = lib
    return lib


class _Quiet:
    """The reference prints its progress to stdout (std::cout); while it runs, file descriptor 1 goes
    to /dev/null so a caller's own output (a bench line) stays the only output."""

    def __enter__(self):
        sys.stdout.flush()
        self.libc = C.CDLL(None)
        self.libc.fflush(None)
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *exc):
        self.libc.fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


QUIET = os.environ.get("DPE_REFERENCE_VERBOSE", "0") != "1"


def _maybe_quiet():
    return _Quiet() if QUIET else _NoOp()


class _NoOp:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


def set_texture_8bit_weights(on: bool) -> None:
    """Bilinear weights rounded to 8 fractional bits, as the texture unit interpolates (default:
    exact float weights, the CUDA kernels' and the oracle's interpolation)."""
    load().ref_set_texture_8bit_weights(1 if on else 0)


def pm_call(images, cameras, params, *, seed: int, threads: int = 0, radius_init: bool = True,
            serial_race: bool = True, work_dir: str | None = None, **kw) -> Dict:
    """One per-view call of the reference (images: float32 arrays of integer grey levels; cameras:
    dicts with the cam-file depth range; params.scale_size 1).  Returns plane / weak / views /
    costs, the cameras and params the reference derived (`cameras`, `params`, ctypes structs), and
    `guard_writes` (bytes the reference wrote just outside its buffers; 0 expected).
    serial_race False runs the edge-aware strong update's blocks in parallel too (timing runs:
    its same-colour read race then resolves by thread timing, as on a GPU)."""
    lib = load()
    pr = D.build_problem(images, cameras, params, seed=seed, **kw)
    H, W, N = pr.height, pr.width, pr.num_images
    out = dict(plane=np.zeros((H, W, 4), np.float32), weak=np.zeros((H, W), np.uint8),
               views=np.zeros((H, W), np.uint32), costs=np.zeros((H, W), np.float32))
    cams = (D.Camera * N)()
    used = D.Params()
    guard = C.c_longlong(0)
    nthreads = threads if threads > 0 else (os.cpu_count() or 1)
    with tempfile.TemporaryDirectory(prefix="dpe_ref_", dir=work_dir) as tmp, _maybe_quiet():
        st = lib.ref_pm_call(C.byref(pr), tmp.encode(), nthreads, 1 if radius_init else 0, 1 if serial_race else 0,
                             out["plane"].ctypes.data,
                             out["weak"].ctypes.data, out["views"].ctypes.data, out["costs"].ctypes.data, cams,
                             C.byref(used), C.byref(guard))
    if st != 0:
        raise RuntimeError(lib.ref_last_error().decode())
    out["cameras"] = list(cams)
    out["params"] = used
    out["guard_writes"] = int(guard.value)
    return out


def camera_dicts(cams) -> List[Dict]:
    """ctypes Camera structs -> the dicts dpe_b200.make_camera takes."""
    return [dict(K=np.array(c.K, np.float32), R=np.array(c.R, np.float32), t=np.array(c.t, np.float32),
                 c=np.array(c.c, np.float32), height=c.height, width=c.width, depth_min=c.depth_min,
                 depth_max=c.depth_max) for c in cams]


def fuse(views: List[Dict], variant: int = 0, work_dir: str | None = None) -> Dict:
    """The reference's fusion over `views` (dicts as for oracle_py.fuse; colour at depth size):
    variant ETH (RunFusion), TAT_INTERMEDIATE (RunFusion_TAT_Intermediate) or TAT_ADVANCED
    (RunFusion_TAT_advanced).  Returns count, xyz (n, 3) float32 and bgr (n, 3) uint8 in PLY order."""
    lib = load()
    fin, keep, cap = D.fusion_input(views, D.FUSE_FLOAT, D.MEM_HOST, 1, None)
    xyz = np.zeros((max(cap, 1), 3), np.float32)
    bgr = np.zeros((max(cap, 1), 3), np.uint8)
    n = C.c_int64(0)
    with tempfile.TemporaryDirectory(prefix="dpe_ref_fuse_", dir=work_dir) as tmp, _maybe_quiet():
        st = lib.ref_fuse(C.byref(fin), variant, tmp.encode(), xyz.ctypes.data, bgr.ctypes.data, cap, C.byref(n))
    if st != 0:
        raise RuntimeError(lib.ref_last_error().decode())
    k = min(int(n.value), cap)
    return dict(count=int(n.value), xyz=xyz[:k], bgr=bgr[:k])


def connect(img: np.ndarray):
    """The reference's Connect (DPE.cpp:27-134): (labels int32, counts per label)."""
    img = np.ascontiguousarray(img, dtype=np.uint8)
    rows, cols = img.shape
    labels = np.zeros((rows, cols), np.int32)
    cap = rows * cols + 1
    counts = np.zeros(cap, np.int32)
    n = C.c_int(0)
    if load().ref_connect(img.ctypes.data, cols, rows, labels.ctypes.data, counts.ctypes.data, cap, C.byref(n)) != 0:
        raise RuntimeError("ref_connect: label count beyond capacity")
    return labels, counts[: n.value].copy()


def roberts(img: np.ndarray) -> np.ndarray:
    """The reference's Roberts cross (DPE.cpp:9-25)."""
    img = np.ascontiguousarray(img, dtype=np.uint8)
    out = np.zeros_like(img)
    load().ref_roberts(img.ctypes.data, img.shape[1], img.shape[0], out.ctypes.data)
    return out
