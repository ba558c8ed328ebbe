"""A batch split over ranks (clip_b200/batches.py) on the GPU: two gloo ranks share the one
GPU of the test box, each advancing its own cases (no kernel of one rank waits on the
other), and the gathered monitors equal those of the whole table run as one batch, bit
for bit (a case's result does not depend on the batch that holds it)."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)

pytestmark = pytest.mark.gpu

SEED, NCASES, STEPS = 12345, 12, 25


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, REPO)
    from datetime import timedelta

    import torch.distributed as dist

    from clip_b200.batches import DistributedBatch

    dist.init_process_group("gloo", timeout=timedelta(seconds=120))
    with DistributedBatch.seeded(SEED, NCASES, "fp32") as b:
        b.init()
        b.solve(STEPS)
        m, ke = b.monitors()
        mine = b.mine
    dist.destroy_process_group()
    q.put((rank, mine, m.tolist(), ke.tolist()))


def test_ranks_gather_the_monitors_of_the_whole_table():
    import clip_b200 as cb

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    with cb.Batch.seeded(SEED, NCASES, "fp32") as whole:
        whole.init()
        whole.solve(STEPS)
        m_ref, ke_ref = whole.monitors()
    assert sorted(out[0][1] + out[1][1]) == list(range(NCASES))
    assert out[0][1] and out[1][1]
    for rank, _, m, ke in out:
        np.testing.assert_array_equal(np.array(m), m_ref, err_msg=f"mass, rank {rank}")
        np.testing.assert_array_equal(np.array(ke), ke_ref, err_msg=f"kinetic energy, rank {rank}")


def _bench_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, REPO)
    from datetime import timedelta

    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", timeout=timedelta(seconds=120))
    res = bench.run_batch_ranks(world, steps=6, ncases=24)
    dist.destroy_process_group()
    q.put((rank, res))


def test_bench_batch_section_over_ranks():
    """bench.py's batch key at N > 1, run by two gloo ranks: the ranks agree on the
    slowest rank's time and the table's nodes."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_bench_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    a, b = out[0][1], out[1][1]
    assert a["ms_per_step_batched"] == b["ms_per_step_batched"] > 0
    assert a["interior_nodes"] == b["interior_nodes"] > 0
    assert a["cases_per_rank"] == b["cases_per_rank"] and sum(a["cases_per_rank"]) == 24
    assert a["mass_sum"] == b["mass_sum"]
