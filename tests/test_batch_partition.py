"""The case table of a batch split over ranks (clip_b200/batches.py) on CPU: the
partition covers every case once and balances the nodes, and the final gather of the
per-case monitors over gloo ranks returns the whole table in case order on every rank."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)

from clip_b200 import seeded_case_config  # noqa: E402
from clip_b200.batches import case_nodes, partition  # noqa: E402


def test_case_nodes_reads_the_interior_extent():
    assert case_nodes("case = drop\nN = [96, 416, 1]\n") == 96 * 416
    assert case_nodes("  N = [32,64,1]") == 32 * 64
    with pytest.raises(ValueError):
        case_nodes("case = drop\n")


@pytest.mark.parametrize("k", [1, 2, 3, 4, 8])
def test_partition_of_the_seeded_table(k):
    sizes = [case_nodes(seeded_case_config(12345, i)) for i in range(512)]
    parts = partition(sizes, k)
    assert len(parts) == k
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(512))
    assert all(p == sorted(p) for p in parts)
    loads = [sum(sizes[i] for i in p) for p in parts]
    # greedy largest-first: no rank exceeds another by more than one case
    assert max(loads) - min(loads) <= max(sizes)
    if k > 1:
        assert max(loads) / (sum(sizes) / k) < 1.01
    assert partition(sizes, k) == parts  # deterministic


def test_partition_edge_cases():
    assert partition([], 3) == [[], [], []]
    assert partition([5], 3) == [[0], [], []]
    assert partition([1, 1, 1, 1], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        partition([1], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, parts, overlap, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, REPO)
    from datetime import timedelta

    import torch.distributed as dist

    from clip_b200.batches import gather_cases

    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    mine = parts[rank] + ([parts[0][0]] if overlap and rank == 1 else [])
    mass = [1000.0 + i for i in mine]
    ke = [0.5 * i for i in mine]
    try:
        out = gather_cases(dist, None, 10, mine, mass, ke)
        res = [a.tolist() for a in out]
    except RuntimeError as e:
        res = str(e)
    dist.destroy_process_group()
    q.put((rank, res))


def _run(world, parts, overlap=False):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, parts, overlap, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return out


def test_gather_returns_the_table_in_case_order_on_every_rank():
    parts = partition([3, 9, 1, 4, 4, 7, 2, 8, 5, 6], 2)
    for rank, res in _run(2, parts):
        assert res[0] == [1000.0 + i for i in range(10)], rank
        assert res[1] == [0.5 * i for i in range(10)], rank


def test_gather_rejects_lists_that_do_not_partition_the_table():
    parts = partition([3, 9, 1, 4, 4, 7, 2, 8, 5, 6], 2)
    for _, res in _run(2, parts, overlap=True):
        assert isinstance(res, str) and "partition" in res
