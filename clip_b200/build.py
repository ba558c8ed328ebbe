"""Build libclipb.so (the sm_100a kernels and the C ABI of include/clipb.h) in-tree.

nvcc compiles each translation unit for sm_100a only; the FP64 unit is compiled without
FMA contraction (-fmad=false) so that it rounds like the reference's arithmetic done one
operation at a time.  The FP32 and FP16 units are compiled without contraction as well:
their fused multiply-adds are written out (fmaf), so that every launch shape of the step
rounds the same way whatever the compiler's scheduling.  Static libstdc++ symbols are kept private to the library
(--exclude-libs) so that it can be loaded into processes that already carry another
libstdc++ (Python with numpy, torch).
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(REPO, "_build", "clipb")
LIB = os.path.join(HERE, "libclipb.so")
DRIVER = os.path.join(HERE, "clipb_run")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-I", os.path.join(REPO, "include"), "-I", SRC]
UNITS = {
    "kernels_fp64.cu": ["-fmad=false"],
    "kernels_fp32.cu": ["-fmad=false", "-ftz=true", "-prec-div=false", "-prec-sqrt=false"],
    "kernels_fp16.cu": ["-fmad=false", "-ftz=true", "-prec-div=false", "-prec-sqrt=false"],
    "capi.cu": [],
    "config.cpp": [],
    "noalloc.cu": [],
    "batch.cu": [],
    "checkpoint.cu": [],
    "adjoint.cu": ["-fmad=false"],
    "adjoint_rev.cu": [],
    "vts.cu": [],
    "slab.cu": [],
}
HEADERS = ["lattice.cuh", "kernels.cuh", "kernels_tma.cuh", "tma.cuh", "launch.cuh", "engine.hpp", "config.hpp",
           "solver.hpp", "dual.cuh", "adjoint.cuh"]


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return exe


def _stale(obj, src):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [src] + [os.path.join(SRC, h) for h in HEADERS] + [os.path.join(REPO, "include", "clipb.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    jobs = []
    objs = []
    for unit, flags in UNITS.items():
        src = os.path.join(SRC, unit)
        obj = os.path.join(BUILD, unit + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            extra = ["-Xptxas", "-v"] if ptxas_info and unit.endswith(".cu") else []
            lang = ["-x", "cu"] if unit.endswith(".cu") else []
            jobs.append([nvcc()] + COMMON + ARCH + flags + extra + lang + ["-c", src, "-o", obj])
    outputs = []
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=len(jobs)) as ex:
            for cmd, res in zip(jobs, ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), jobs)):
                if verbose:
                    print(" ".join(cmd))
                outputs.append(res.stdout + res.stderr)
                if res.returncode != 0:
                    sys.stderr.write(res.stdout + res.stderr)
                    raise RuntimeError("nvcc failed: " + " ".join(cmd))
    if jobs or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        link = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xlinker", "--exclude-libs,ALL", "-lcudart_static"]
        res = subprocess.run(link, capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError("link failed")
    # host driver (C++ main loop over the C ABI)
    main_src = os.path.join(SRC, "clipb_main.cpp")
    if force or not os.path.exists(DRIVER) or os.path.getmtime(DRIVER) < max(os.path.getmtime(main_src),
                                                                           os.path.getmtime(LIB)):
        cmd = [shutil.which("g++") or "g++", "-std=c++17", "-O2", "-I", os.path.join(REPO, "include"), main_src,
               "-o", DRIVER, "-L", HERE, "-l:libclipb.so", "-Wl,-rpath,$ORIGIN"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError("driver build failed")
    return "\n".join(outputs)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-v", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print register/spill usage of every kernel")
    a = ap.parse_args()
    out = build(a.v, a.force, a.ptxas)
    if a.ptxas:
        print(out)
    print(LIB)
