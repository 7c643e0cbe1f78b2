"""Build the sm_100a library and the `fsmeld` command in-tree.

Outputs (git-ignored, shipped with the source tree):
  fsmeld_b200/lib/libfsmeld_cuda.so   kernels + C ABI (include/fsmeld_cuda.h)
  fsmeld_b200/bin/fsmeld              the reference-compatible CLI

    python -m fsmeld_b200.build          # incremental
    python -m fsmeld_b200.build --force
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")
INCLUDE = os.path.join(ROOT, "include")
OBJ = os.path.join(PKG, "_obj")
LIBDIR = os.path.join(PKG, "lib")
BINDIR = os.path.join(PKG, "bin")
LIB = os.path.join(LIBDIR, "libfsmeld_cuda.so")
CLI = os.path.join(BINDIR, "fsmeld")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

def _cutlass_include():
    """CUTLASS / CuTe headers (header-only; the sm100 UMMA descriptor unions).
    $FSMELD_CUTLASS_INCLUDE, else the copy vendored with flashinfer."""
    env = os.environ.get("FSMELD_CUTLASS_INCLUDE")
    if env:
        return env
    try:
        import importlib.util
        spec = importlib.util.find_spec("flashinfer")
        if spec and spec.submodule_search_locations:
            cand = os.path.join(list(spec.submodule_search_locations)[0], "data", "cutlass", "include")
            if os.path.isdir(cand):
                return cand
    except Exception:
        pass
    raise RuntimeError("CUTLASS headers not found: set FSMELD_CUTLASS_INCLUDE")


CUTLASS_INC = None
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-static-global-template-stub=false",
                  "-Xcompiler", "-fPIC,-ffp-contract=off", f"-I{INCLUDE}"]

CU = ["k_stats", "k_envelope", "k_threshold", "k_lbip", "k_glb", "k_dp", "k_dpw", "k_lbgemm", "k_select", "engine", "noalloc"]


def _newer(src_files, out):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in src_files)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    return hs + [os.path.join(INCLUDE, "fsmeld_cuda.h")]


def _run(cmd):
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + p.stdout + p.stderr)
    return p


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(BINDIR, exist_ok=True)
    hdrs = _headers()
    jobs = []
    objs = []
    for name in CU:
        src = os.path.join(CSRC, name + ".cu")
        obj = os.path.join(OBJ, name + ".o")
        objs.append(obj)
        if force or _newer([src] + hdrs, obj):
            extra = [f"-I{_cutlass_include()}"] if name == "k_lbgemm" else []
            jobs.append([NVCC] + NVFLAGS + extra + ["-c", src, "-o", obj])
    drv_src = os.path.join(HOST, "cli_driver.cpp")
    drv_obj = os.path.join(OBJ, "cli_driver.o")
    objs.append(drv_obj)
    if force or _newer([drv_src] + hdrs, drv_obj):
        jobs.append(["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", f"-I{INCLUDE}", "-c", drv_src,
                     "-o", drv_obj])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
            for p in ex.map(_run, jobs):
                if verbose and (p.stdout or p.stderr):
                    print(p.stdout + p.stderr)
    if force or _newer(objs, LIB):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"])
    main_src = os.path.join(HOST, "fsmeld_main.cpp")
    if force or _newer([main_src, LIB], CLI):
        _run(["g++", "-O2", "-std=c++17", f"-I{INCLUDE}", main_src, "-o", CLI, f"-L{LIBDIR}", "-lfsmeld_cuda",
              "-Wl,-rpath,$ORIGIN/../lib"])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
