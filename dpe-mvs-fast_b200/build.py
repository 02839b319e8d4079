"""Build the sm_100a shared library libdpe_sm100.so in-tree (nvcc, no torch extension machinery).

Usage: python dpe-mvs-fast_b200/build.py [--force] [--checked]

Builds the default library and the exact build (libdpe_sm100_exact.so: no multiply-add
contraction, IEEE division); --checked builds the bounds-checked debug library instead.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdpe_sm100.so")
LIB_CHECKED = os.path.join(HERE, "libdpe_sm100_checked.so")
# The exact build: IEEE division at every tap as well, so the device computes the CPU oracle's
# arithmetic bit for bit (the default build takes the hardware reciprocal for a tap's
# perspective divide, and differs from the oracle by that rounding only).
EXACT_FLAGS = ("-fmad=false", "-DDPE_EXACT")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2"]
# per-source extra flags.  No multiply-add contraction in the PatchMatch units (capi.cu, scene.cu)
# and fusion: the decisions between near-equal hypotheses then fall as in the reference's own
# arithmetic (measured: contraction moves 0.6 % of a C1 call's depths by more than 0.1 % against
# the reference, without it 0.45 %, the oracle's figure; it costs 6 % of the C2 schedule).
UNITS = {
    "capi.cu": ["-fmad=false"],
    "scene.cu": ["-fmad=false"],
    "fusion.cu": ["-fmad=false"],
    "edges.cu": [],
    "views.cu": ["-fmad=false"],
}


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _deps() -> list:
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    files.append(os.path.join(HERE, "..", "include", "dpe_b200.h"))
    files.append(os.path.abspath(__file__))
    return files


def build(force: bool = False, verbose: bool = False, checked: bool = False, variant: str = "",
          defines: tuple = ()) -> str:
    """Compile csrc/*.cu for sm_100a and link libdpe_sm100.so (checked=True: the bounds-checked
    debug variant libdpe_sm100_checked.so, built with -DDPE_CHECKED; variant: a named build with
    extra flags, here the exact build)."""
    os.makedirs(OBJ, exist_ok=True)
    lib = LIB_CHECKED if checked else LIB
    if variant:
        lib = os.path.join(HERE, f"libdpe_sm100_{variant}.so")
    newest = max(os.path.getmtime(f) for f in _deps())
    if not force and os.path.exists(lib) and os.path.getmtime(lib) >= newest:
        return lib
    nvcc = _nvcc()
    procs = []
    objs = []
    for src, extra in UNITS.items():
        suffix = f"_{variant}.o" if variant else ("_checked.o" if checked else ".o")
        obj = os.path.join(OBJ, src.replace(".cu", suffix))
        objs.append(obj)
        flags = (["-DDPE_CHECKED"] if checked else []) + list(defines)
        cmd = [nvcc, *ARCH, *COMMON, *extra, *flags, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed: {' '.join(cmd)}\n{out.decode(errors='replace')}")
    link = [nvcc, *ARCH, "-shared", *objs, "-o", lib + ".tmp", "-lcudart"]
    subprocess.run(link, check=True, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    os.replace(lib + ".tmp", lib)
    return lib


def build_all(force: bool = False, verbose: bool = False) -> list:
    """The default library and the exact build (libdpe_sm100_exact.so)."""
    return [build(force=force, verbose=verbose), build(force=force, verbose=verbose, variant="exact", defines=EXACT_FLAGS)]


if __name__ == "__main__":
    args = sys.argv[1:]
    if "--checked" in args:
        print(build(force="--force" in args, verbose=True, checked=True))
    else:
        print("\n".join(build_all(force="--force" in args, verbose=True)))
