"""Batches of independent 2D cases over several GPUs, one process per GPU.

The cases share nothing, so the case table is partitioned.  Each rank advances its own
cases in one libclipb batch (clipb_batch_*: one persistent launch per step), and the only
collective is the gather of the per-case monitors at the end.  The partition balances the
interior nodes per rank: the largest case goes first onto the least loaded rank, so the
ranks finish a step at about the same time.  No counterpart in the reference, which runs
one case per process.
"""
import re

import numpy as np

from . import Batch, seeded_case_config


def case_nodes(config_text):
    """Interior nodes of a 2D case from its config text (N = [nx, ny, 1])."""
    m = re.search(r"^\s*N\s*=\s*\[\s*(\d+)\s*,\s*(\d+)", config_text, re.M)
    if not m:
        raise ValueError("the config has no N = [..] line")
    return int(m.group(1)) * int(m.group(2))


def partition(sizes, k):
    """Case indices of each of k ranks, each list ascending.  Cases in decreasing size
    (lower index first among equals) go to the rank with the fewest nodes so far (lower
    rank first among equals); the result depends on the sizes and k alone."""
    if k < 1:
        raise ValueError("need at least one rank")
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i], i))
    load = [0] * k
    parts = [[] for _ in range(k)]
    for i in order:
        r = min(range(k), key=lambda j: (load[j], j))
        parts[r].append(i)
        load[r] += sizes[i]
    return [sorted(p) for p in parts]


def gather_cases(dist, group, ncases, mine, *values):
    """Every rank's per-case values (arrays over its cases `mine`) in case order, on every
    rank: one all_gather of (indices, values) over the group."""
    local = (list(mine), [np.asarray(v, dtype=float).tolist() for v in values])
    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, local, group=group)
    out = [np.full(ncases, np.nan) for _ in values]
    seen = np.zeros(ncases, dtype=int)
    for idx, vals in parts:
        for a, v in zip(out, vals):
            a[idx] = v
        seen[idx] += 1
    if not (seen == 1).all():
        raise RuntimeError("the ranks' case lists do not partition the table")
    return out


class DistributedBatch:
    """This rank's share of a table of 2D cases (config texts), as one Batch."""

    def __init__(self, configs, precision="fp32", group=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.rank, self.k = dist.get_rank(group), dist.get_world_size(group)
        self.ncases = len(configs)
        sizes = [case_nodes(t) for t in configs]
        self.parts = partition(sizes, self.k)
        self.mine = self.parts[self.rank]
        self.nodes = sum(sizes[i] for i in self.mine)
        self.batch = Batch([configs[i] for i in self.mine], precision, texts=True) if self.mine else None

    @classmethod
    def seeded(cls, seed, ncases, precision="fp32", group=None):
        """The seeded case table of clipb_seeded_case_config."""
        return cls([seeded_case_config(seed, i) for i in range(ncases)], precision, group)

    def close(self):
        if self.batch is not None:
            self.batch.close()
            self.batch = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def init(self):
        if self.batch is not None:
            self.batch.init()

    def autotune(self, trial_steps=4):
        return self.batch.autotune(trial_steps) if self.batch is not None else None

    def solve(self, nsteps=1):
        if self.batch is not None:
            self.batch.solve(nsteps)

    def time_steps(self, nsteps):
        """Device time (ms) of nsteps of this rank's batch (0 without cases)."""
        return self.batch.time_steps(nsteps) if self.batch is not None else 0.0

    def monitors(self):
        """Mass and kinetic energy of every case of the table, in case order, on every
        rank (the gather; every rank must call it)."""
        if self.batch is not None:
            m, ke = self.batch.monitors()
        else:
            m, ke = np.empty(0), np.empty(0)
        return gather_cases(self.dist, self.group, self.ncases, self.mine, m, ke)
