#!/usr/bin/env python3
"""Golden fixtures from the reference's own FP64 CUDA build.

The reference (mshadkhah/CLIP) has no tests, no golden vectors and no CPU path, so its
results can only be pinned by running its unmodified CUDA solver.  oracle/Makefile
compiles the reference sources with a small harness (oracle/ref_harness.cu) into
oracle/_ref/ref_harness_{2d,3d}; this script

  --write-configs   writes the config.txt files of every golden case into configs/
  --run RAW         runs the harness for every case on a GPU and leaves raw dumps in RAW/
  --pack RAW        converts the raw dumps into compact .npz fixtures (--out DIR)
  --trim DIR        selects the committed subset of packed fixtures into this folder
  --vts RAW         runs the -fmad=false harness with the reference's own VTSwriter for the
                    VTS cases and gzips the kept .vts files into vts/ (--out DIR/vts)

Raw dumps are the reference's own layout: ghosted extent, x slowest, component fastest
(Domain.cuh:63-68).  Packed fixtures keep that layout (ghosted, [X][Y][Z][comp]) as
float64 arrays named <field>_<step>; "full" cases also keep f, g, f_post, g_post, mu, dc,
normal.  Large cases keep c/p/rho/vel only.
"""
import argparse
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CONFIGS = os.path.join(HERE, "configs")
REPO = os.path.dirname(os.path.dirname(HERE))


def _boundary(sides):
    out = ["boundary = ["]
    for side, typ, val in sides:
        out.append("  {")
        out.append(f'    side = "{side}"')
        out.append(f'    type = "{typ}"')
        if val is not None:
            out.append("    value = [" + ", ".join(repr(v) for v in val) + "]")
        out.append("  },")
    out.append("]")
    return "\n".join(out)


def _geometry(geoms):
    out = ["geometry = ["]
    for g in geoms:
        out.append("  {")
        for k, v in g.items():
            if isinstance(v, str):
                out.append(f'    {k} = "{v}"')
            elif isinstance(v, (list, tuple)):
                out.append(f"    {k} = [" + ", ".join(repr(x) for x in v) + "]")
            else:
                out.append(f"    {k} = {v!r}")
        out.append("  }")
    out.append("]")
    return "\n".join(out)


def _config(case, N, scalars, geoms, sides):
    lines = [f"case = {case}", "", "finalStep = 1000", "outputInterval = 1000", "reportInterval = 1000",
             "checkpointInterval = 1000", "checkpointCopy = 0", "",
             "N = [" + ", ".join(repr(v) for v in N) + "]"]
    for k, v in scalars.items():
        if isinstance(v, (list, tuple)):
            lines.append(f"{k} = [" + ", ".join(repr(x) for x in v) + "]")
        else:
            lines.append(f"{k} = {v!r}")
    lines += ["", _geometry(geoms), "", _boundary(sides), ""]
    return "\n".join(lines)


PW = [("x-", "periodic", None), ("x+", "periodic", None), ("y-", "wall", None), ("y+", "wall", None)]
PW3 = PW + [("z-", "periodic", None), ("z+", "periodic", None)]

# name -> (dim, config text, nsteps, dump steps, full dumps)
CASES = {
    # the 2D drop workload (64x128 interior, periodic x / walls y, 1000 steps)
    "drop2d_64x128": (2, _config("drop", [64, 128, 1], dict(
        referenceLength=25, We=5, Re=100, gravity=[0, -1e-6, 0], mobility=0.02, interfaceWidth=4,
        muRatio=100, rhoRatio=1000), [dict(type="circle", center=[32.5, 64.5, 0], radius=12.5, id=0)], PW),
        1000, [0, 1, 2, 10, 100, 1000], [0, 1, 2]),
    # small full-state cases: every field at a few steps
    "drop2d_small": (2, _config("drop", [24, 32, 1], dict(
        referenceLength=12, We=2, Re=20, gravity=[0, -1e-5, 0], mobility=0.05, interfaceWidth=4,
        muRatio=10, rhoRatio=50), [dict(type="circle", center=[12.5, 14.0, 0], radius=6, id=0)], PW),
        50, [0, 1, 2, 3, 10, 50], [0, 1, 2, 3, 10, 50]),
    "bubble2d_walls": (2, _config("bubble", [20, 28, 1], dict(
        referenceLength=10, We=3, Re=30, gravity=[0, -2e-5, 0], mobility=0.03, interfaceWidth=3,
        muRatio=5, rhoRatio=20), [dict(type="square", center=[10.0, 12.0, 0], length=[9, 8, 0], id=0)],
        [("x-", "wall", None), ("x+", "wall", None), ("y-", "wall", None), ("y+", "wall", None)]),
        40, [0, 1, 2, 5, 40], [0, 1, 2, 5, 40]),
    "rti2d_small": (2, _config("RTI", [32, 64, 1], dict(
        referenceLength=32, Re=300, Pe=100, Ca=0.3, gravity=[0, -1e-5, 0], interfaceWidth=5,
        muRatio=1, rhoRatio=3), [dict(type="perturbation", center=[0, 32.5, 0], amplitude=0.1,
                                      length=[32, 0, 0], id=0)], PW),
        60, [0, 1, 2, 10, 60], [0, 1, 2, 10, 60]),
    "inlet2d_small": (2, _config("drop", [24, 30, 1], dict(
        referenceLength=10, We=4, Re=40, gravity=[0, -1e-5, 0], mobility=0.02, interfaceWidth=4,
        muRatio=4, rhoRatio=10), [dict(type="circle", center=[12.5, 31.0, 0], radius=5, id=0)],
        [("x-", "periodic", None), ("x+", "periodic", None), ("y-", "wall", None),
         ("y+", "velocity", [0.0, -0.01, 0.0])]),
        30, [0, 1, 2, 5, 30], [0, 1, 2, 5, 30]),
    # inlet on x-; the reference takes every inlet velocity from the y+ entry (Solver.cu:587-588)
    "inlet2d_side": (2, _config("bubble", [22, 26, 1], dict(
        referenceLength=8, We=4, Re=40, gravity=[0, -1e-5, 0], mobility=0.02, interfaceWidth=4,
        muRatio=4, rhoRatio=10), [dict(type="circle", center=[0.0, 13.5, 0], radius=5, id=0)],
        [("x-", "velocity", None), ("x+", "wall", None), ("y-", "wall", None),
         ("y+", "wall", [0.01, 0.002, 0.0])]),
        20, [0, 1, 2, 5, 20], [0, 1, 2, 5, 20]),
    "rti2d_256x1024": (2, _config("RTI", [256, 1024, 1], dict(
        referenceLength=256, Re=3000, Pe=409.6, Ca=0.26, gravity=[0, -1e-6, 0], interfaceWidth=5,
        muRatio=1, rhoRatio=3), [dict(type="perturbation", center=[0, 512.5, 0], amplitude=0.1,
                                      length=[256, 0, 0], id=0)], PW),
        2000, [2000], []),
    # 3D: extents include the ghost layer (Domain.cu:57-59)
    "drop3d_small": (3, _config("drop", [18, 22, 16], dict(
        referenceLength=10, We=3, Re=30, gravity=[0, -1e-5, 0], mobility=0.03, interfaceWidth=3,
        muRatio=10, rhoRatio=40), [dict(type="sphere", center=[8.5, 10.0, 7.5], radius=5, id=0)],
        PW + [("z-", "wall", None), ("z+", "wall", None)]),
        20, [0, 1, 2, 5, 20], [0, 1, 2, 5, 20]),
    "bubble3d_walls": (3, _config("bubble", [14, 16, 12], dict(
        referenceLength=8, We=3, Re=30, gravity=[0, -1e-5, 0], mobility=0.03, interfaceWidth=3,
        muRatio=10, rhoRatio=40), [dict(type="cube", center=[6.5, 7.0, 5.5], length=[6, 7, 5], id=0)],
        [("x-", "wall", None), ("x+", "wall", None), ("y-", "wall", None), ("y+", "wall", None),
         ("z-", "wall", None), ("z+", "wall", None)]),
        15, [0, 1, 2, 15], [0, 1, 2, 15]),
    "rti3d_small": (3, _config("RTI", [18, 34, 18], dict(
        referenceLength=16, Re=200, Pe=80, Ca=0.3, gravity=[0, 1e-5, 0], interfaceWidth=4,
        muRatio=1, rhoRatio=3), [dict(type="perturbation", center=[0, 16.5, 0], amplitude=0.1,
                                      length=[16, 0, 0], id=0)], PW3),
        20, [0, 1, 2, 20], [0, 1, 2, 20]),
    "rti3d_small_repeat": None,
    "inlet3d_small": (3, _config("drop", [16, 20, 16], dict(
        referenceLength=8, We=4, Re=40, gravity=[0, -1e-5, 0], mobility=0.02, interfaceWidth=4,
        muRatio=4, rhoRatio=10), [dict(type="sphere", center=[7.5, 19.5, 7.5], radius=4, id=0)],
        [("x-", "periodic", None), ("x+", "periodic", None), ("y-", "wall", None),
         ("y+", "velocity", [0.0, -0.01, 0.0]), ("z-", "periodic", None), ("z+", "periodic", None)]),
        12, [0, 1, 2, 12], [0, 1, 2, 12]),
    "bubble3d_64": (3, _config("bubble", [66, 98, 66], dict(
        referenceLength=16, We=10, Re=35, gravity=[0, -1e-6, 0], mobility=0.02, interfaceWidth=4,
        muRatio=100, rhoRatio=1000), [dict(type="sphere", center=[32.5, 24.5, 32.5], radius=8, id=0)], PW3),
        200, [200], []),
}
CASES["rti3d_small_repeat"] = CASES["rti3d_small"]

# Free-convect, Neumann and slip-wall sides (Solver.cu:248-542).  "free convect" and
# "slip wall" are written as the configs spell them; the reference's parser cannot reach
# them (it strips the space), so the harness sets those sides after parsing (--bc).
_JET_SIDES = [("x-", "periodic", None), ("x+", "periodic", None), ("y-", "free convect", None),
              ("y+", "velocity", [0.0, -0.01, 0.0])]
_JET2 = dict(referenceLength=10, We=4, Re=40, gravity=[0, -1e-5, 0], mobility=0.02, interfaceWidth=4,
             muRatio=4, rhoRatio=10)
CASES.update({
    "neumann2d_small": (2, _config("drop", [24, 30, 1], _JET2, [dict(type="circle", center=[12.5, 12.0, 0],
                                                                  radius=5, id=0)],
                                   [("x-", "periodic", None), ("x+", "periodic", None), ("y-", "wall", None),
                                    ("y+", "neumann", None)]),
                        30, [0, 1, 2, 5, 30], [0, 1, 2, 5, 30]),
    "outflow2d_small": (2, _config("drop", [24, 30, 1], _JET2, [dict(type="circle", center=[12.5, 31.0, 0],
                                                                  radius=5, id=0)], _JET_SIDES),
                        30, [0, 1, 2, 5, 30], [0, 1, 2, 5, 30]),
    "mixed2d_small": (2, _config("drop", [22, 28, 1], _JET2, [dict(type="circle", center=[11.5, 29.0, 0],
                                                                radius=5, id=0)],
                                 [("x-", "neumann", None), ("x+", "neumann", None), ("y-", "free convect", None),
                                  ("y+", "velocity", [0.0, -0.01, 0.0])]),
                      30, [0, 1, 2, 5, 30], [0, 1, 2, 5, 30]),
    "slip2d_walls": (2, _config("bubble", [20, 28, 1], dict(
        referenceLength=10, We=3, Re=30, gravity=[0, -2e-5, 0], mobility=0.03, interfaceWidth=3,
        muRatio=5, rhoRatio=20), [dict(type="square", center=[10.0, 12.0, 0], length=[9, 8, 0], id=0)],
        [("x-", "wall", None), ("x+", "slip wall", None), ("y-", "wall", None), ("y+", "wall", None)]),
        40, [0, 1, 2, 5, 40], [0, 1, 2, 5, 40]),
    "outflow3d_small": (3, _config("drop", [16, 20, 16], dict(
        referenceLength=8, We=4, Re=40, gravity=[0, -1e-5, 0], mobility=0.02, interfaceWidth=4,
        muRatio=4, rhoRatio=10), [dict(type="sphere", center=[7.5, 19.5, 7.5], radius=4, id=0)],
        [("x-", "periodic", None), ("x+", "periodic", None), ("y-", "free convect", None),
         ("y+", "velocity", [0.0, -0.01, 0.0]), ("z-", "wall", None), ("z+", "wall", None)]),
        12, [0, 1, 2, 12], [0, 1, 2, 12]),
    "neumann3d_small": (3, _config("drop", [18, 22, 16], dict(
        referenceLength=10, We=3, Re=30, gravity=[0, -1e-5, 0], mobility=0.03, interfaceWidth=3,
        muRatio=10, rhoRatio=40), [dict(type="sphere", center=[8.5, 10.0, 7.5], radius=5, id=0)],
        PW + [("z-", "wall", None), ("z+", "neumann", None)]),
        15, [0, 1, 2, 15], [0, 1, 2, 15]),
    "mixed3d_small": (3, _config("drop", [14, 18, 14], dict(
        referenceLength=8, We=4, Re=40, gravity=[0, -1e-5, 0], mobility=0.02, interfaceWidth=4,
        muRatio=4, rhoRatio=10), [dict(type="sphere", center=[6.5, 17.5, 6.5], radius=4, id=0)],
        [("x-", "neumann", None), ("x+", "neumann", None), ("y-", "free convect", None),
         ("y+", "velocity", [0.0, -0.01, 0.0]), ("z-", "wall", None), ("z+", "slip wall", None)]),
        12, [0, 1, 2, 12], [0, 1, 2, 12]),
})
# harness --bc settings of the cases whose side types the reference's parser cannot reach
BC_OVERRIDE = {"outflow2d_small": "y-=freeconvect", "mixed2d_small": "y-=freeconvect",
               "slip2d_walls": "x+=slipwall", "outflow3d_small": "y-=freeconvect",
               "mixed3d_small": "y-=freeconvect,z+=slipwall"}


def write_configs():
    os.makedirs(CONFIGS, exist_ok=True)
    for name, (dim, text, *_rest) in CASES.items():
        with open(os.path.join(CONFIGS, name + ".txt"), "w") as fp:
            fp.write(text)


def run(raw, only=None, variant=""):
    """Run the reference harness for every case; variant "nofma" uses the -fmad=false build."""
    for name, (dim, _text, nsteps, dumps, full) in CASES.items():
        if only and name not in only:
            continue
        if variant:
            full = []
        out = os.path.join(raw, name)
        os.makedirs(out, exist_ok=True)
        exe = os.path.join(REPO, "oracle", "_ref", f"ref_harness_{dim}d" + (f"_{variant}" if variant else ""))
        cfg = os.path.join(CONFIGS, name + ".txt")
        dumps_all = sorted(set(dumps) | set(full))
        args = [exe, cfg, out, str(nsteps), "--dump", ",".join(map(str, dumps_all))]
        if full:
            args.append("--full")
        if name in BC_OVERRIDE:
            args += ["--bc", BC_OVERRIDE[name]]
        print("running", " ".join(args), flush=True)
        res = subprocess.run(args, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        with open(os.path.join(out, "harness.log"), "w") as fp:
            fp.write(res.stdout)
        if res.returncode != 0:
            print(res.stdout[-3000:])
            raise SystemExit(f"reference harness failed for {name}: rc={res.returncode}")
        # Only the 'full' steps keep the big arrays.
        for fn in os.listdir(out):
            if not fn.endswith(".bin"):
                continue
            field, step = fn[:-4].rsplit("_", 1)
            if field in ("f", "g", "f_post", "g_post", "mu", "dc", "normal") and int(step) not in full:
                os.remove(os.path.join(out, fn))


def pack(raw, out=HERE, only=None, variant=""):
    """Pack raw dumps into <out>/<case>.npz.

    Small ("full") cases keep every dumped field on the whole ghosted grid.  Large cases
    keep the interior c, p and vel subsampled with stride 2 (2D) or 4 (3D) per axis, plus
    global moments of the full interior fields (sum c, sum c^2, sum |u|^2, max |u|, sum p).
    """
    Q = {2: 9, 3: 19}
    os.makedirs(out, exist_ok=True)
    for name, (dim, text, nsteps, dumps, full) in CASES.items():
        if only and name not in only:
            continue
        d = os.path.join(raw, name)
        if not os.path.isdir(d):
            print("missing raw dumps for", name)
            continue
        N = [float(x) for x in text.split("N = [")[1].split("]")[0].split(",")]
        ext = [int(N[0]) + 2, int(N[1]) + 2, 1] if dim == 2 else [int(N[0]), int(N[1]), int(N[2])]
        ncomp = {"c": 1, "p": 1, "rho": 1, "mu": 1, "vel": dim, "dc": dim, "normal": dim,
                 "f": Q[dim], "g": Q[dim], "f_post": Q[dim], "g_post": Q[dim]}
        if variant:
            full = []
        big = not full and not variant
        stride = 2 if dim == 2 else 4
        if variant and np.prod(ext) > 100000:
            big = True
        interior = (slice(1, ext[0] - 1), slice(1, ext[1] - 1), slice(1, ext[2] - 1) if dim == 3 else slice(0, 1))
        arrays = {}
        for fn in sorted(os.listdir(d)):
            if not fn.endswith(".bin"):
                continue
            field, step = fn[:-4].rsplit("_", 1)
            a = np.fromfile(os.path.join(d, fn), dtype=np.float64).reshape(ext + [ncomp[field]])
            key = f"{field}_{int(step)}"
            if not big:
                arrays[key] = a
                continue
            if field == "rho":
                continue
            ai = a[interior]
            sub = ai[::stride, ::stride, ::stride if dim == 3 else 1]
            arrays[key + "_sub"] = np.ascontiguousarray(sub)
            if field == "c":
                arrays[key + "_sum"] = np.array([ai.sum(), (ai * ai).sum(), ai.max(), ai.min()])
            elif field == "vel":
                u2 = (ai * ai).sum(axis=-1)
                arrays[key + "_sum"] = np.array([u2.sum(), np.sqrt(u2.max())])
            elif field == "p":
                arrays[key + "_sum"] = np.array([ai.sum(), np.abs(ai).max()])
        meta = dict(name=name, dim=dim, extent=ext, nsteps=nsteps, dumps=dumps, full=full,
                    subsample_stride=stride if big else 1,
                    source="reference FP64 CUDA build (oracle/_ref/ref_harness_%dd) on NVIDIA B200" % dim)
        arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
        if variant:
            meta["variant"] = variant
            meta["source"] += " built with -fmad=false" if variant == "nofma" else ""
            arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
        fn = os.path.join(out, name + (f"_{variant}" if variant else "") + ".npz")
        np.savez_compressed(fn, **arrays)
        print("packed", os.path.basename(fn), round(os.path.getsize(fn) / 1e6, 3), "MB")


# Steps whose full state (populations, mu, dc, normal) is kept in the committed fixture;
# every other dumped step keeps c, p, rho and vel only.
KEEP_FULL = {"drop2d_64x128": [1], "drop2d_small": [0, 1], "rti2d_small": [1], "inlet2d_small": [1],
             "inlet2d_side": [1], "bubble2d_walls": [1], "drop3d_small": [0, 1], "bubble3d_walls": [1],
             "rti3d_small": [], "rti3d_small_repeat": [], "inlet3d_small": [1],
             "neumann2d_small": [1, 2], "outflow2d_small": [1, 2], "mixed2d_small": [1, 2], "slip2d_walls": [1],
             "outflow3d_small": [1, 2], "neumann3d_small": [1], "mixed3d_small": [1, 2]}


def trim(src, out=HERE, only=None):
    """Select the committed subset of packed fixtures (src/<case>.npz -> out/<case>.npz)."""
    scal = ("c", "p", "rho", "vel")
    for name in CASES:
        if only and name not in only:
            continue
        fn = os.path.join(src, name + ".npz")
        if not os.path.exists(fn):
            continue
        a = np.load(fn)
        keep = {}
        for k in a.files:
            if k == "meta" or k.endswith("_sub") or k.endswith("_sum"):
                keep[k] = a[k]
                continue
            field, step = k.rsplit("_", 1)
            if field in scal or name not in KEEP_FULL or int(step) in KEEP_FULL[name]:
                keep[k] = a[k]
        if name == "rti3d_small_repeat":
            keep = {k: v for k, v in keep.items() if k == "meta" or k.rsplit("_", 1)[0] in ("c", "vel", "p")}
        np.savez_compressed(os.path.join(out, name + ".npz"), **keep)
        print("trimmed", name, round(os.path.getsize(os.path.join(out, name + ".npz")) / 1e6, 3), "MB")


# .vts files written by the reference's VTSwriter (src/io/VTSwriter.cu) through the harness
# (main.cu's call sequence), with the case's outputInterval set to `interval`:
# name -> (interval, steps run, steps kept)
VTS_CASES = {"drop2d_small": (10, 50, [0, 10, 50]), "inlet2d_small": (5, 30, [0, 30]),
             "drop3d_small": (5, 20, [0, 20])}


def run_vts(raw, out=HERE):
    import gzip
    dest = os.path.join(out, "vts")
    os.makedirs(dest, exist_ok=True)
    for name, (interval, nsteps, keep) in VTS_CASES.items():
        dim, text = CASES[name][0], CASES[name][1]
        assert "outputInterval = 1000" in text
        d = os.path.join(raw, name + "_vts")
        os.makedirs(d, exist_ok=True)
        cfg = os.path.join(d, "config.txt")
        with open(cfg, "w") as fp:
            fp.write(text.replace("outputInterval = 1000", f"outputInterval = {interval}"))
        exe = os.path.join(REPO, "oracle", "_ref", f"ref_harness_{dim}d_nofma")
        args = [exe, cfg, d, str(nsteps), "--vts", os.path.join(d, "results")]
        print("running", " ".join(args), flush=True)
        res = subprocess.run(args, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if res.returncode != 0:
            print(res.stdout[-3000:])
            raise SystemExit(f"reference harness failed for {name}: rc={res.returncode}")
        for step in keep:
            src = os.path.join(d, "results", f"results_t{step}.vts")
            with open(src, "rb") as fp:
                data = fp.read()
            fn = os.path.join(dest, f"{name}_t{step}.vts.gz")
            with open(fn, "wb") as raw_fp, gzip.GzipFile(fileobj=raw_fp, mode="wb", mtime=0) as gz:
                gz.write(data)
            print("packed", os.path.basename(fn), len(data), "bytes,", os.path.getsize(fn), "gzipped")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--write-configs", action="store_true")
    ap.add_argument("--run")
    ap.add_argument("--pack")
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--variant", default="", help="'nofma': the reference built with -fmad=false")
    ap.add_argument("--trim", help="directory of packed fixtures to select the committed subset from")
    ap.add_argument("--only", nargs="*")
    ap.add_argument("--vts", help="directory for the raw VTS runs")
    a = ap.parse_args()
    if a.write_configs:
        write_configs()
    if a.run:
        run(a.run, a.only, a.variant)
    if a.pack:
        pack(a.pack, a.out, a.only, a.variant)
    if a.trim:
        trim(a.trim, a.out, a.only)
    if a.vts:
        run_vts(a.vts, a.out)


if __name__ == "__main__":
    sys.exit(main())
