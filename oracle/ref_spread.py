"""Spread of the reference's own FP64 builds on the 3D rising bubble (128x256x128 interior),
beside the FP32 and FP16 storage of this library, all against this library's FP64 path.

The whole-field difference between two runs of the 3D bubble is set by chaotic fluctuations
of c in the bulk of each phase: the reference's FMA build differs from itself run to run,
because its periodic ghost kernel writes edge cells from several threads
(src/solver/Solver.cu:96-136).  So the reduced-precision errors are compared on what that
noise does not reach, the interface band and the height of the bubble, with the reference's
own spread on the same case printed beside them.

usage: python oracle/ref_spread.py [STEP ...]     (default: 2000 10000; one JSON line out)

Runs oracle/_ref/ref_harness_3d (the reference's sources as shipped) twice and
oracle/_ref/ref_harness_3d_nofma (built with -fmad=false) once -- both built by
oracle/Makefile -- dumping c at each STEP, then this library's FP64, FP32 and FP16 paths.
Test infrastructure (needs a GPU and the built reference harness); it is not part of the
library.
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, REPO)
WORKLOAD = os.path.join(REPO, "clip_b200", "workloads", "bubble3d_128x256x128.txt")
EXT = (130, 258, 130)


def bubble_y(c):
    """Height of the bubble: mean y of 1 - c over nodes with c < 0.5 (1-based like the grid)."""
    w = np.where(c < 0.5, 1.0 - c, 0.0)
    ys = np.arange(c.shape[1], dtype=np.float64)[None, :, None]
    return float((w * ys).sum() / w.sum()) + 1.0


def reference_run(exe, steps, out):
    os.makedirs(out, exist_ok=True)
    args = [exe, WORKLOAD, out, str(max(steps)), "--dump", ",".join(map(str, steps))]
    res = subprocess.run(args, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if res.returncode != 0:
        raise SystemExit(f"{exe} failed (rc {res.returncode}): {res.stdout[-2000:]}")
    fields = {}
    for k in steps:
        a = np.fromfile(os.path.join(out, f"c_{k:06d}.bin"), dtype=np.float64).reshape(EXT)
        fields[k] = np.ascontiguousarray(a[1:-1, 1:-1, 1:-1])
        for fn in os.listdir(out):
            if fn.endswith(f"_{k:06d}.bin"):
                os.remove(os.path.join(out, fn))
    return fields


def library_run(prec, steps):
    import clip_b200 as cb

    fields = {}
    with cb.Solver(WORKLOAD, prec) as s:
        s.init(on_device=True)
        done = 0
        for k in steps:
            s.solve(k - done)
            done = k
            fields[k] = s.interior_field("c")[..., 0].astype(np.float64)
    return fields


def compare(a, ref):
    band = (ref >= 0.01) & (ref <= 0.99)
    d = np.abs(a - ref)
    return {"max": float(d.max()), "band_max": float(d[band].max()),
            "bubble_y_diff": abs(bubble_y(a) - bubble_y(ref)),
            "sum_c_rel": float(abs(a.sum() - ref.sum()) / ref.sum())}


def main():
    steps = sorted(int(a) for a in sys.argv[1:]) or [2000, 10000]
    exe = os.path.join(HERE, "_ref", "ref_harness_3d")
    runs = {"fp64": library_run("fp64", steps), "fp32": library_run("fp32", steps),
            "fp16": library_run("fp16", steps)}
    with tempfile.TemporaryDirectory() as tmp:
        runs["reference_fma_a"] = reference_run(exe, steps, os.path.join(tmp, "a"))
        runs["reference_fma_b"] = reference_run(exe, steps, os.path.join(tmp, "b"))
        runs["reference_nofma"] = reference_run(exe + "_nofma", steps, os.path.join(tmp, "n"))
    out = {"workload": "bubble3d_128x256x128", "steps": steps,
           "band": "nodes with 0.01 <= c <= 0.99 in the FP64 run of this library",
           "bubble_y": "mean y of 1 - c over nodes with c < 0.5, lattice units"}
    for k in steps:
        ref = runs["fp64"][k]
        row = {name: compare(runs[name][k], ref)
               for name in ("reference_fma_a", "reference_nofma", "fp32", "fp16")}
        row["reference_fma_a_vs_b"] = compare(runs["reference_fma_a"][k], runs["reference_fma_b"][k])
        out[str(k)] = row
    print(json.dumps(out))


if __name__ == "__main__":
    main()
