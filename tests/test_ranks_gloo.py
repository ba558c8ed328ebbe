"""The multi-rank path of bench.py on CPU: two gloo ranks (the GPU run uses NCCL with the
same calls).  Each rank runs an independent replica; the job's time is the slowest
rank's, and the throughput counts every rank's lattice updates over that time.  The
reference arm prints from rank 0 only."""
import os
import socket
import sys

import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, REPO)
    import torch.distributed as dist
    from datetime import timedelta

    import bench

    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    w, r, _ = bench._dist()
    local_ms = 10.0 + 5.0 * r  # rank 1 is slower
    bench.barrier(w)
    ms = bench.max_over_ranks(local_ms, w, device="cpu")
    value = bench.aggregate_mlups(1000, 20, w, ms)
    ref_line = bench.run_reference(type("A", (), {"warmup": 1, "steps": 2})(), w, r) if r != 0 else "rank0"
    dist.destroy_process_group()
    q.put((r, w, ms, value, ref_line))


def test_two_ranks_take_the_slowest_time_and_sum_the_work():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, w, ms, value, ref_line in out:
        assert w == 2
        assert ms == 15.0  # the slowest rank
        assert abs(value - 1000 * 20 * 2 / 15e-3 * 1e-6) < 1e-9
    assert out[1][4] is None  # only rank 0 runs the reference arm
