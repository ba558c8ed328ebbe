#!/usr/bin/env python3
"""Throughput of the CLIP lattice update on B200 (MLUPS and fraction of the HBM roofline).

Workload: 3D rising bubble, D3Q19 + D3Q19 phase field, 256x512x256 interior nodes
(clip_b200/workloads/bubble3d_256x512x256.txt; the vertical axis is y as in the
reference's config semantics), synthetic initial state from the config (no dataset).
A step is one time step of the whole grid: one fused kernel launch.

Our arm (default): FP32 population storage (the production precision); FP64 and FP16
storage are timed on the same workload and reported as extra keys.  The timed region
holds exactly K steps between barrier + device synchronise on both sides, timed with CUDA
events on the launching stream (max over ranks).  The state (11.5 GB in FP32) is far
larger than L2, so no flush is needed between steps.

--impl reference: the reference's own FP64 CUDA build (oracle/_ref/ref_harness_3d, built
from its unmodified sources) timing NSAllen::solve() on the same workload.

Multi-GPU (--gpus N, N > 1, under torchrun): by default the case is split into N z slabs,
one per rank, whose boundary planes are exchanged every step with NCCL point-to-point
messages (strong scaling: the same 33.5 M nodes over N GPUs).  --decomp replicas runs N
independent copies of the case instead (weak scaling).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

WORKLOAD = os.path.join(REPO, "clip_b200", "workloads", "bubble3d_256x512x256.txt")
WORKLOAD_NAME = "3d_rising_bubble_256x512x256"
METRIC = "MLUPS"
# Algorithmic bytes per lattice update: f and g read + written once (2 * 2Q values) and
# u, c read + written once (2 * (DIM + 1) values).
Q, DIM = 19, 3
B_LU = {"f32": 2 * 2 * Q * 4 + 2 * (DIM + 1) * 4,
        "f64": 2 * 2 * Q * 8 + 2 * (DIM + 1) * 8,
        "f16": 2 * 2 * Q * 2 + 2 * (DIM + 1) * 4}


def _peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as fp:
            d = json.load(fp)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _profile_traffic(dtype):
    """DRAM bytes per lattice update of the fused kernel from the committed ncu summary."""
    try:
        with open(os.path.join(REPO, "profiles", "ncu_traffic.json")) as fp:
            d = json.load(fp)
        return d.get(f"step3d_{dtype}", {}).get("dram_bytes_per_lu")
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi samples (every 200 ms) while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(v, world, device="cuda"):
    """Largest value over the ranks (the job's time is its slowest rank's)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def upload_bytes(extent):
    """Bytes of the initial c field as clipb_device_initializer copies it: FP64 over the
    ghosted extent in the device layout (rows padded to 32 values after a 31-value lead)."""
    sy = -(-(31 + extent[0]) // 32) * 32
    return -(-(sy * extent[1] * extent[2]) // 32) * 32 * 8


def aggregate_mlups(nodes_per_rank, steps, world, max_ms):
    """Whole-job throughput: every rank's lattice updates over the slowest rank's time."""
    return nodes_per_rank * steps * world / (max_ms * 1e-3) * 1e-6


def cpu_baseline(seconds=12.0):
    """The CPU oracle (FP64 restatement of the reference step) on the host cores, on a
    64x128x64 crop of the workload with the same physics (bounded sample)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O  # noqa: E402  (CPU baseline leg only)
    import tempfile

    text = open(WORKLOAD).read()
    text = text.replace("N = [258, 514, 258]", "N = [66, 130, 66]")
    text = text.replace("center = [128.5, 96.5, 128.5]", "center = [32.5, 24.5, 32.5]")
    text = text.replace("radius = 32", "radius = 8")
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as fp:
        fp.write(text)
        path = fp.name
    o = O.Oracle(path)
    o.init()
    o.solve(1)  # warm-up
    n = 64 * 128 * 64
    steps, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        o.solve(1)
        steps += 1
    dt = time.perf_counter() - t0
    os.unlink(path)
    return {"value": n * steps / dt * 1e-6, "unit": METRIC, "cores": O.threads(), "kind": "port",
            "sample": f"CPU oracle (FP64, {O.threads()} host threads) on a 64x128x64 crop of the workload "
                      f"with the same physics, {steps} steps after 1 warm-up step"}


def precision_errors(steps, block, workload=WORKLOAD):
    """FP64, FP32 and FP16 storage of the workload stepped side by side (all three states
    stay on the GPU: 23 + 11.5 + 6 GB); after every `block` steps the FP32 and FP16 c
    fields are compared with FP64's (max |dc| over the interior), with the kinetic energy's
    relative error and each run's mass drift."""
    import clip_b200 as cb

    precs = ("fp64", "fp32", "fp16")
    sol = {p: cb.Solver(workload, p) for p in precs}
    m0 = {}
    for p, s in sol.items():
        s.init(on_device=True)
        m0[p] = s.monitors()[0]
    out = {"steps": steps, "block": block, "at_step": [],
           "band": "interface band: nodes with 0.01 <= c <= 0.99 in the FP64 run",
           "bubble_y": "height of the bubble: mean y of 1 - c over nodes with c < 0.5"}
    for p in ("fp32", "fp16"):
        for k in ("max_c_err", "max_c_err_band", "bubble_y_err", "kinetic_err_rel"):
            out[f"{p}_{k}"] = []
    out["fp64_bubble_y"] = []

    def bubble_y(c):
        m = c < 0.5
        w = np.where(m, 1.0 - c, 0.0)
        ys = np.arange(c.shape[1], dtype=np.float64)[None, :, None]
        return float((w * ys).sum() / w.sum()) + 1.0

    done = 0
    while done < steps:
        n = min(block, steps - done)
        for s in sol.values():
            s.solve(n)
        done += n
        c64 = sol["fp64"].interior_field("c")[..., 0]
        band = (c64 >= 0.01) & (c64 <= 0.99)
        y64 = bubble_y(c64)
        ke64 = sol["fp64"].monitors()[1]
        out["at_step"].append(done)
        out["fp64_bubble_y"].append(y64)
        for p in ("fp32", "fp16"):
            c = sol[p].interior_field("c")[..., 0]
            d = np.abs(c - c64)
            out[f"{p}_max_c_err"].append(float(d.max()))
            out[f"{p}_max_c_err_band"].append(float(d[band].max()))
            out[f"{p}_bubble_y_err"].append(abs(bubble_y(c) - y64))
            out[f"{p}_kinetic_err_rel"].append(abs(sol[p].monitors()[1] - ke64) / abs(ke64))
            del c, d
        del c64, band
    for p, s in sol.items():
        out[f"{p}_mass_drift_rel"] = abs(s.monitors()[0] - m0[p]) / abs(m0[p])
        s.close()
    return out


def run_ours(args, world, rank, local):
    import torch
    import clip_b200 as cb

    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    interior = 256 * 512 * 256
    stream = torch.cuda.Stream()
    results = {}

    def timed(prec, steps, warmup, sample_clocks=False):
        s = cb.Solver(WORKLOAD, prec)
        s.set_stream(stream.cuda_stream)
        s.init()
        # launch shape picked by the library's autotuner (it rebuilds the initial state)
        variant, seg, _ = s.autotune(3)
        results.setdefault("launch", {})[prec] = {"variant": variant, "planes_per_cta": seg}
        s.solve(warmup)
        torch.cuda.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        clocks = None
        sampler = ClockSampler(local) if sample_clocks else None
        if sampler:
            sampler.__enter__()
        with torch.cuda.stream(stream):
            e0.record(stream)
            s.solve(steps)
            e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        barrier(world)
        if sampler:
            sampler.__exit__(None, None, None)
            clocks = sampler.summary()
        ms = max_over_ranks(e0.elapsed_time(e1), world)
        return s, ms, clocks

    # headline: FP32 storage
    s32, ms32, clocks = timed("fp32", args.steps, args.warmup, sample_clocks=True)
    mlups = aggregate_mlups(interior, args.steps, world, ms32)
    per_launch_ms = ms32 / args.steps
    peak, peak_kind = _peaks()
    achieved = B_LU["f32"] * interior / (per_launch_ms * 1e-3) / 1e9
    traffic_lu = _profile_traffic("f32")
    results.update(value=mlups, ms_per_step=per_launch_ms, clocks=clocks,
                   roofline={"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "peak_source": f"{peak_kind} MEASURED_PEAKS.json hbm_gbs"
                             if peak_kind == "measured" else "fallback 6650 GB/s",
                             "traffic": traffic_lu * interior if traffic_lu else None,
                             "algorithmic_bytes_per_lu": B_LU["f32"]})

    # end to end through the public API: initial field evaluated on the host and uploaded
    # (H2D), then every step solve() + monitors() (device reduction, D2H of the step's mass
    # and kinetic energy); the same with the initial field evaluated on the GPU
    def end_to_end(on_device):
        torch.cuda.synchronize()
        barrier(world)
        t0 = time.perf_counter()
        with torch.cuda.stream(stream):
            s32.init(on_device=on_device)
            for _ in range(args.steps):
                s32.solve_monitored(1)
        torch.cuda.synchronize()
        return max_over_ranks(time.perf_counter() - t0, world)

    # one untimed pass of each path first (the device path's first call loads its kernels)
    end_to_end(False)
    end_to_end(True)
    e2e_s = end_to_end(False)
    # the initial c field, uploaded once per run: the bytes clipb_init sent (its non-uniform
    # rows and a per-plane table; the whole field would be upload_bytes((258, 514, 258)))
    h2d = s32.upload_bytes()
    results["e2e"] = {"value": interior * args.steps * world / e2e_s * 1e-6, "unit": METRIC,
                      "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": 16,
                      "h2d_bytes_whole_field": upload_bytes((258, 514, 258)),
                      "timed": "initial field on the host (clipb_init: host threads, pinned staging, upload "
                               "overlapped in chunks of planes, uniform rows filled on the device) + device "
                               "init, then per step solve_monitored(1): one step whose kernel also sums the FP64 "
                               "mass and kinetic energy, read back to the host"}
    e2e_dev_s = end_to_end(True)
    results["e2e_device_init"] = {"value": interior * args.steps * world / e2e_dev_s * 1e-6, "unit": METRIC,
                                  "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 16,
                                  "timed": "the same with the initial field evaluated on the GPU (clipb_init_device)"}
    s32.close()

    # FP64 and FP16 storage on the same workload
    for prec, key in (("fp64", "f64"), ("fp16", "f16")):
        s, ms, _ = timed(prec, args.steps, args.warmup)
        results[f"{key}_mlups"] = aggregate_mlups(interior, args.steps, world, ms)
        results[f"{key}_frac_hbm"] = B_LU[key] * interior / (ms / args.steps * 1e-3) / 1e9 / peak
        s.close()

    # FP32 and FP16 against FP64 on the same workload, side by side, after every block of
    # steps up to err_steps (c max abs error, kinetic energy relative error, mass drift)
    if rank == 0 and args.err_steps > 0:
        results["precision_vs_fp64"] = precision_errors(args.err_steps, args.err_block)
    barrier(world)
    launches = args.steps  # one fused kernel per step, no inlet on this workload
    return results, launches


def run_slabs(k=4, steps=20, check_steps=10, ms_whole=None):
    """The workload split into k z slabs on this one GPU (clip_b200.slabs.SlabGroup): the
    cost of the decomposition (its boundary-plane exchange) per step, and whether the slabs
    reproduce the whole case bit for bit (FP32 storage)."""
    import torch
    import clip_b200 as cb
    from clip_b200.slabs import SlabGroup

    whole = cb.Solver(WORKLOAD, "fp32")
    whole.set_launch(8, 8)
    whole.init()
    whole.set_graphs(False)
    whole.solve(check_steps)
    c_whole = whole.interior_field("c")
    whole.close()
    out = {}
    for overlap in (False, True):
        with SlabGroup(WORKLOAD, "fp32", k, variant=8, seg=8, overlap=overlap) as grp:
            grp.init()
            grp.solve(check_steps)
            exact = bool(np.array_equal(grp.field("c"), c_whole))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(grp.stream)
            grp.solve(steps)
            e1.record(grp.stream)
            e1.synchronize()
            key = "overlap" if overlap else "serial"
            out[key] = (e0.elapsed_time(e1) / steps, exact)
            packet = grp.slabs[0].packet_bytes
    del c_whole
    return {"slabs": k, "planes_per_slab": 256 // k, "ms_per_step": out["serial"][0],
            "ms_per_step_overlap": out["overlap"][0], "ms_per_step_whole": ms_whole,
            "exchange_bytes_per_step": 2 * 2 * k * packet,
            "bit_exact_vs_whole_after_steps": check_steps if out["serial"][1] and out["overlap"][1] else None,
            "timed": f"{steps} steps of k slabs on one GPU, CUDA events on the slabs' stream: serial = k fused "
                     "steps then 2k pack and 2k unpack launches; overlap = the face planes of each slab first, "
                     "then the packs and unpacks on a second stream while the other planes update"}


def run_slab_ranks(args, world, rank, local):
    """--decomp slab: the workload split into z slabs, one per rank, boundary planes
    exchanged every step with NCCL point-to-point messages (strong scaling)."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    from clip_b200.slabs import DistributedSlab

    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    interior = 256 * 512 * 256
    ds = DistributedSlab(WORKLOAD, "fp32", variant=8, seg=8, overlap=True)
    ds.init()
    ds.solve(args.warmup)
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(local)
    sampler.__enter__()
    e0.record(ds.compute)
    ds.solve(args.steps)
    e1.record(ds.compute)
    torch.cuda.synchronize()
    barrier(world)
    sampler.__exit__(None, None, None)
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    # per step and rank: the two parts of the step, one pack per send and one unpack per receive
    sends = sum(1 for phase in ds._plan for op in phase if op[0] == "send")
    recvs = sum(1 for phase in ds._plan for op in phase if op[0] == "recv")
    launches = args.steps * (2 + sends + recvs)
    nodes_rank = 256 * 512 * (ds.slab.zhi - ds.slab.zlo + 1)
    peak, peak_kind = _peaks()
    per_rank_gbs = B_LU["f32"] * nodes_rank * args.steps / (ms * 1e-3) / 1e9
    # end to end: initial state from the host, then per step the step, the exchange and the
    # monitors summed over the slabs (all-reduce) read back
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    ds.init()
    for _ in range(args.steps):
        ds.solve(1)
        m = torch.tensor(ds.slab.monitors(), dtype=torch.float64, device="cuda")
        dist.all_reduce(m)
        m.cpu()
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    up = torch.tensor([float(ds.slab.upload_bytes())], dtype=torch.float64, device="cuda")
    dist.all_reduce(up)  # the bytes every slab's clipb_init sent
    h2d = up.item()
    ds.close()
    dist.destroy_process_group()
    return {"value": interior * args.steps / (ms * 1e-3) * 1e-6, "ms_per_step": ms / args.steps,
            "clocks": sampler.summary(), "launches": launches,
            "roofline": {"bound": "hbm", "achieved": per_rank_gbs, "peak": peak, "unit": "GB/s",
                         "frac": per_rank_gbs / peak, "traffic": None,
                         "peak_source": f"{peak_kind} MEASURED_PEAKS.json hbm_gbs, per GPU (rank 0's slab)"},
            "e2e": {"value": interior * args.steps / e2e_s * 1e-6, "unit": METRIC,
                    "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": 16 * world,
                    "timed": "host initial condition + upload + init of every slab, then per step the slab "
                             "step, the boundary exchange and the all-reduced monitors read back"}}


def run_rti(steps=20000, block=2000):
    """The 2D Rayleigh-Taylor workload (256 x 1024, 20000 steps) in FP64, FP32 and FP16
    storage side by side: c and u errors of FP32/FP16 against FP64 after every block of
    steps, the kinetic energy's relative error, mass drift, and each precision's MLUPS
    (autotuned launch shape, CUDA events per block).  The flow is unstable: pointwise
    differences grow from rounding alone (the reference's own FP64 builds with and without
    FMA contraction differ by 9e-3 in c at step 2000), global quantities stay close."""
    import clip_b200 as cb

    cfg = os.path.join(REPO, "clip_b200", "workloads", "rti2d_256x1024.txt")
    precs = ("fp64", "fp32", "fp16")
    sol = {p: cb.Solver(cfg, p) for p in precs}
    ms = {p: 0.0 for p in precs}
    m0 = {}
    for p, s in sol.items():
        s.init()
        s.autotune(3)  # rebuilds the initial state
        m0[p] = s.monitors()[0]
    out = {"steps": steps, "block": block, "nodes": 256 * 1024}
    for p in ("fp32", "fp16"):
        out[f"{p}_max_c_err"] = []
        out[f"{p}_max_u_err_rel"] = []
        out[f"{p}_kinetic_err_rel"] = []
    for _ in range(steps // block):
        for p, s in sol.items():
            ms[p] += s.time_steps(block)
        c64, u64 = sol["fp64"].interior_field("c"), sol["fp64"].interior_field("vel")
        umax = float(np.abs(u64).max())
        ke64 = sol["fp64"].monitors()[1]
        for p in ("fp32", "fp16"):
            out[f"{p}_kinetic_err_rel"].append(abs(sol[p].monitors()[1] - ke64) / abs(ke64))
            out[f"{p}_max_c_err"].append(float(np.abs(sol[p].interior_field("c") - c64).max()))
            out[f"{p}_max_u_err_rel"].append(float(np.abs(sol[p].interior_field("vel") - u64).max()) / umax)
    for p, s in sol.items():
        out[f"{p}_mlups"] = 256 * 1024 * steps / (ms[p] * 1e-3) * 1e-6
        out[f"{p}_mass_drift_rel"] = abs(s.monitors()[0] - m0[p]) / abs(m0[p])
        s.close()
    out["timed"] = "time_steps(block) per precision (CUDA events; graph replay), fields read between blocks"
    return out


def run_batch(steps=100, seq_steps=20, ncases=512, seed=12345):
    """The seeded batch workload (512 uneven 2D drop/bubble cases, FP32 storage): batched
    persistent launches (autotuned, CUDA graph) against plain per-case launches."""
    import clip_b200 as cb

    with cb.Batch.seeded(seed, ncases, "fp32") as b:
        b.init()
        nodes = 0
        for i in range(b.size):
            s = b.case(i)
            nodes += s.interior[0] * s.interior[1]
        variant, rows, bps, _ = b.autotune(3)
        b.solve(3)
        ms_b = b.time_steps(steps) / steps
        b.solve_sequential(2)
        ms_s = b.time_steps(seq_steps, sequential=True) / seq_steps
        _, _, _, nitems = b.get_launch()
    per_case_steps = 5000
    return {"cases": ncases, "seed": seed, "interior_nodes": nodes, "case_steps": per_case_steps,
            "ms_per_step_batched": ms_b, "ms_per_step_sequential": ms_s,
            "cases_per_s": ncases / (ms_b * 1e-3 * per_case_steps),
            "cases_per_s_sequential": ncases / (ms_s * 1e-3 * per_case_steps),
            "speedup_vs_sequential": ms_s / ms_b, "mlups_batched": nodes / (ms_b * 1e-3) * 1e-6,
            "launch": {"variant": variant, "rows_per_item": rows, "blocks_per_sm": bps, "work_items": nitems},
            "timed": f"{steps} batched steps (graph replay) and {seq_steps} sequential steps "
                     f"({ncases} plain launches per step), CUDA events, after autotune and warm-up"}


def run_batch_ranks(world, steps=100, ncases=512, seed=12345):
    """The seeded batch workload split over the ranks (replicas only: each rank advances its
    share of the case table, balanced by nodes; the final monitor gather is the only
    collective).  Every rank calls it; the job's time is the slowest rank's."""
    import torch
    import torch.distributed as dist
    from clip_b200.batches import DistributedBatch

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    with DistributedBatch.seeded(seed, ncases, "fp32") as b:
        b.init()
        tuned = b.autotune(3)
        b.solve(3)
        barrier(world)
        torch.cuda.synchronize()
        ms = max_over_ranks(b.time_steps(steps), world, dev) / steps
        mass, _ = b.monitors()
        nodes = torch.tensor([float(b.nodes)], dtype=torch.float64, device=dev)
        dist.all_reduce(nodes)
        per_rank = [len(p) for p in b.parts]
    per_case_steps = 5000
    return {"cases": ncases, "seed": seed, "ranks": world, "cases_per_rank": per_rank,
            "interior_nodes": int(nodes.item()), "case_steps": per_case_steps, "ms_per_step_batched": ms,
            "cases_per_s": ncases / (ms * 1e-3 * per_case_steps), "mlups_batched": nodes.item() / (ms * 1e-3) * 1e-6,
            "mass_sum": float(np.sum(mass)), "launch_rank0": list(tuned) if tuned else None,
            "timed": f"{steps} batched steps of each rank's share (graph replay, CUDA events), max over ranks; "
                     f"cases split by nodes, monitors gathered at the end"}


def run_adjoint(steps=2000, checkpoint_every=100):
    """The adjoint workload: 256x256 2D drop, FP64, objective |centroid(c_2000) - target|^2
    with target = the unperturbed centroid + (3, 5); gradient with respect to the initial c
    field and (g_y, sigma, M) by the adjoint (checkpoints every 100 steps), its cost
    against the forward, and the agreement with the tangent-linear model and with central
    finite differences of the forward."""
    import clip_b200 as cb

    cfg = os.path.join(REPO, "clip_b200", "workloads", "drop2d_256x256_adjoint.txt")
    s = cb.Solver(cfg, "fp64")
    c0 = s.initial_condition()
    s.objective(steps, np.zeros(2), c0)
    c = s.interior_field("c")[..., 0, 0]
    x = np.arange(1, c.shape[0] + 1)[:, None]
    y = np.arange(1, c.shape[1] + 1)[None, :]
    target = np.array([(x * c).sum() / c.sum() + 3.0, (y * c).sum() / c.sum() + 5.0])
    p = s.params()
    theta = np.array([p["gy"], p["sigma"], p["mobility"]])
    # warm-up: the first adjoint call allocates its workspace (tapes, checkpoints), which
    # later calls on the same solver reuse
    s.adjoint(steps, target, c0, checkpoint_every)
    s.objective(steps, target, c0)

    def median_time(fn, reps=3):
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            out = fn()
            ts.append(time.perf_counter() - t0)
        return float(np.median(ts)), out

    t_fwd, _ = median_time(lambda: s.objective(steps, target, c0))
    t_ck, (J, gc0, gp) = median_time(lambda: s.adjoint(steps, target, c0, checkpoint_every))
    # every state of the run in one tape (2001 states, 22 GB of HBM): no recomputation
    s.adjoint(steps, target, c0, steps)
    t_full, _ = median_time(lambda: s.adjoint(steps, target, c0, steps))
    # the library's own choice (checkpoint_every = 0): one tape when it takes at most half
    # of the free device memory, which holds here
    t_adj, _ = median_time(lambda: s.adjoint(steps, target, c0, 0))
    t0 = time.perf_counter()
    _, dJ = s.tangent(steps, target, c0, None, theta)
    t_tlm = time.perf_counter() - t0
    # noise floor of J: its change when one parameter moves by a few ulps, where the
    # derivative predicts a change far below one ulp of J -- the rounding of 2000 steps,
    # amplified by the flow.  A central difference with step h carries an error of about
    # J_noise / (2 h |dJ/dtheta|) from it.
    J0 = s.objective(steps, target, c0)
    noise = [0.0, 0.0, 0.0]
    for i in range(3):
        for k in (1, 2, 3, 5):
            t = theta.copy()
            t[i] = theta[i] * (1 + k * 2.0 ** -52)
            s.set_params(*t)
            noise[i] = max(noise[i], abs(s.objective(steps, target, c0) - J0))
    s.set_params(*theta)
    fd_val = {}
    fd = {}
    fd_noise = {}
    for eps in (1e-7, 1e-6, 1e-5, 1e-4, 1e-3, 1e-2):
        fd_noise[f"eps_{eps:g}"] = [noise[i] / (2 * eps * abs(theta[i]) * abs(gp[i])) for i in range(3)]
        rel = []
        for i in range(3):
            h = eps * abs(theta[i])
            tp, tm = theta.copy(), theta.copy()
            tp[i] += h
            tm[i] -= h
            s.set_params(*tp)
            Jp = s.objective(steps, target, c0)
            s.set_params(*tm)
            Jm = s.objective(steps, target, c0)
            s.set_params(*theta)
            rel.append(abs((Jp - Jm) / (2 * h) - gp[i]) / abs(gp[i]))
            fd_val.setdefault(("gy", "sigma", "mobility")[i], []).append((Jp - Jm) / (2 * h))
        fd[f"eps_{eps:g}"] = rel
    s.close()
    return {"workload": "2d_drop_256x256_fp64", "steps": steps, "checkpoint_every": checkpoint_every,
            "J": J, "grad_params": {"gy": gp[0], "sigma": gp[1], "mobility": gp[2]},
            "grad_c0_norm": float(np.linalg.norm(gc0)),
            "forward_s": t_fwd, "adjoint_s": t_adj, "adjoint_over_forward": t_adj / t_fwd,
            "adjoint_policy": "checkpoint_every = 0: one tape when it fits in half the free device memory",
            "adjoint_checkpointed_s": t_ck, "adjoint_checkpointed_over_forward": t_ck / t_fwd,
            "reverse_over_forward": (t_ck - t_fwd) / t_fwd,
            "adjoint_one_tape_s": t_full, "adjoint_one_tape_over_forward": t_full / t_fwd, "tangent_s": t_tlm,
            "tangent_vs_adjoint_rel": abs(dJ - float(np.dot(gp, theta))) / abs(dJ),
            "fd_rel_err": fd, "fd_eps": [1e-7, 1e-6, 1e-5, 1e-4, 1e-3, 1e-2],
            "fd_values": fd_val,
            "fd_spread_rel": {k: (max(v) - min(v)) / abs(np.median(v)) for k, v in fd_val.items()},
            "J_noise": {"gy": noise[0], "sigma": noise[1], "mobility": noise[2]},
            "fd_noise_rel": fd_noise,
            "timed": "wall clock of one host call each, median of 3 after a warm-up call (init + steps + "
                     "objective); adjoint: the library's default policy (every state in one tape here); "
                     "adjoint_checkpointed: its forward run with checkpoints every 100 steps, the recomputed "
                     "segments and the reverse sweep; reverse_over_forward: the checkpointed adjoint's time "
                     "beyond one forward run over the forward run's; adjoint_one_tape: all 2001 states kept"}


def run_reference(args, world, rank):
    if rank != 0:
        return None
    exe = os.path.join(REPO, "oracle", "_ref", "ref_harness_3d")
    if not os.path.exists(exe):
        return {"impl": "reference", "unavailable": "oracle/_ref/ref_harness_3d was not built (needs the reference sources)"}
    res = subprocess.run([exe, WORKLOAD, "-", "0", "--time", str(args.warmup), str(args.steps)],
                         stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    line = [l for l in res.stdout.splitlines() if l.startswith("{")]
    if res.returncode != 0 or not line:
        return {"impl": "reference", "unavailable": "reference harness failed: " + res.stdout[-300:].replace("\n", " ")}
    r = json.loads(line[-1])
    v = r["mlups"]
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (initial state from the config)",
            "config": {"workload": WORKLOAD_NAME, "interior_nodes": 256 * 512 * 256, "lattice": "D3Q19 + D3Q19",
                       "parallelism": "single GPU", "l2": "state (24 GB) larger than L2"},
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": 1, "kind": "reference",
                             "sample": f"reference FP64 CUDA build (its own sources, oracle/_ref/ref_harness_3d): "
                                       f"NSAllen::solve() timed alone over {args.steps} steps of the full "
                                       f"workload on the B200 after {args.warmup} warm-up steps"},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def summary_of(line):
    """Compact figures of the detail sections, placed early in the JSON line."""
    out = {"f64_mlups": line.get("f64_mlups"), "f16_mlups": line.get("f16_mlups")}
    if line.get("roofline"):
        out["hbm_frac"] = line["roofline"].get("frac")
    if line.get("e2e"):
        out["e2e_mlups"] = line["e2e"]["value"]
    pe = line.get("precision_vs_fp64")
    if pe and pe.get("at_step"):
        out["err_vs_fp64_at_step"] = pe["at_step"][-1]
        out["fp32_max_c_err_vs_fp64"] = pe["fp32_max_c_err"][-1]
        out["fp32_max_c_err_band_vs_fp64"] = pe["fp32_max_c_err_band"][-1]
        out["fp32_bubble_y_err"] = pe["fp32_bubble_y_err"][-1]
        out["fp16_max_c_err_vs_fp64"] = pe["fp16_max_c_err"][-1]
        out["fp32_max_c_err_vs_fp64_first_block"] = pe["fp32_max_c_err"][0]
    if line.get("e2e_device_init"):
        out["e2e_device_init_mlups"] = line["e2e_device_init"]["value"]
    b = line.get("batch")
    if b:
        out["batch_speedup_vs_sequential"] = b.get("speedup_vs_sequential")
        out["batch_cases_per_s"] = b.get("cases_per_s")
    a = line.get("adjoint")
    if a:
        out["adjoint_over_forward"] = a.get("adjoint_over_forward")
        out["adjoint_checkpointed_over_forward"] = a.get("adjoint_checkpointed_over_forward")
        out["adjoint_fd_rel_err"] = a.get("fd_rel_err")
        out["adjoint_J_noise"] = a.get("J_noise")
    sl = line.get("slabs")
    if sl:
        out["slabs_ms_per_step"] = sl.get("ms_per_step")
    r = line.get("rti2d")
    if r:
        out["rti2d_fp32_mlups"] = r.get("fp32_mlups")
    return {k: v for k, v in out.items() if v is not None}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--err-steps", type=int, default=10000,
                    help="FP32/FP16 against FP64 on the workload up to this step (0: skip)")
    ap.add_argument("--err-block", type=int, default=1000, help="steps between two error readings")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched 2D workload")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint workload")
    ap.add_argument("--no-slabs", action="store_true", help="skip the one-GPU z-slab measurement")
    ap.add_argument("--no-rti", action="store_true", help="skip the 2D Rayleigh-Taylor precision run")
    ap.add_argument("--decomp", default="slab", choices=["replicas", "slab"],
                    help="N > 1: one z slab of the case per rank, boundary planes exchanged every step "
                         "(strong scaling; default), or independent replicas (weak scaling)")
    args = ap.parse_args()
    world, rank, local = _dist()
    if args.impl == "reference":
        line = run_reference(args, world, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        return 0

    if args.decomp == "slab" and world > 1:
        res = run_slab_ranks(args, world, rank, local)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": res["value"], "unit": METRIC, "n_gpus": world,
                              "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
                              "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
                              "data": "synthetic (initial state from the config: sphere of radius 32, tanh profile)",
                              "config": {"workload": WORKLOAD_NAME, "interior_nodes": 256 * 512 * 256,
                                         "lattice": "D3Q19 + D3Q19", "parallelism": f"z slabs x{world}",
                                         "l2": "no flush: the state is far larger than L2"},
                              "roofline": res["roofline"], "clocks": res["clocks"], "e2e": res["e2e"],
                              "gpu_launches": res["launches"], "cpu_baseline": None}), flush=True)
        return 0

    results, launches = run_ours(args, world, rank, local)
    batch_ranks = run_batch_ranks(world) if world > 1 and not args.no_batch else None
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    if rank != 0:
        return 0
    detail = {}
    for k in ("f64_mlups", "f64_frac_hbm", "f16_mlups", "f16_frac_hbm", "precision_vs_fp64", "e2e_device_init"):
        if k in results:
            detail[k] = results[k]
    if world == 1 and not args.no_batch:
        detail["batch"] = run_batch()
    elif batch_ranks is not None:
        detail["batch"] = batch_ranks
    if world == 1 and not args.no_adjoint:
        detail["adjoint"] = run_adjoint()
    if world == 1 and not args.no_slabs:
        detail["slabs"] = run_slabs(ms_whole=results["ms_per_step"])
    if world == 1 and not args.no_rti:
        detail["rti2d"] = run_rti()
    cpu = cpu_baseline() if not args.no_cpu_baseline and world == 1 else None
    line = {"metric": METRIC, "value": results["value"], "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": results["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (initial state from the config: sphere of radius 32, tanh profile)",
            "summary": summary_of({**detail, "roofline": results.get("roofline"), "e2e": results.get("e2e")}),
            "config": {"workload": WORKLOAD_NAME, "interior_nodes": 256 * 512 * 256, "lattice": "D3Q19 + D3Q19",
                       "precision": "f32 population storage (g as g - w c), FP32 arithmetic, c kept as "
                                    "(stored, remainder) pairs in the stencils",
                       "launch": results.get("launch"),
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "no flush: the state (11.5 GB) is far larger than L2"},
            "roofline": results["roofline"], "clocks": results["clocks"], "e2e": results["e2e"],
            "gpu_launches": launches, "cpu_baseline": cpu}
    line.update(detail)
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
