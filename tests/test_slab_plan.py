"""The communication plan of the z-slab decomposition on CPU (gloo ranks; on GPUs the
same calls go over NCCL): every face receives the planes of the right neighbour, in a
fixed order of two phases that stays unambiguous when both neighbours are one rank."""
import os
import socket
import sys

import pytest
import torch
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)

from clip_b200.slabs import exchange_faces, exchange_plan, neighbours, slab_ranges  # noqa: E402


def test_ranges_cover_the_axis_with_balanced_slabs():
    assert slab_ranges(14, 3) == [(1, 5), (6, 10), (11, 14)]
    assert slab_ranges(256, 8)[-1] == (225, 256)
    for nz, k in [(4, 2), (17, 4), (256, 7)]:
        r = slab_ranges(nz, k)
        assert r[0][0] == 1 and r[-1][1] == nz
        assert all(b[0] == a[1] + 1 for a, b in zip(r, r[1:]))
        assert all(e - s + 1 >= 2 for s, e in r)
    with pytest.raises(ValueError):
        slab_ranges(5, 3)  # slabs of at least two planes


def test_neighbours_and_faces():
    assert neighbours(0, 3, False) == (None, 1) and exchange_faces(0, 3, False) == 2
    assert neighbours(2, 3, False) == (1, None) and exchange_faces(2, 3, False) == 1
    assert neighbours(0, 3, True) == (2, 1) and exchange_faces(0, 3, True) == 3
    assert neighbours(0, 1, True) == (None, None) and exchange_faces(0, 1, True) == 0
    assert neighbours(1, 2, True) == (0, 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, periodic, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, REPO)
    from datetime import timedelta

    import torch.distributed as dist

    from clip_b200.slabs import exchange_plan, neighbours, run_exchange

    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    plan = exchange_plan(rank, world, periodic)
    send = [torch.zeros(3, dtype=torch.int64) for _ in range(2)]
    recv = [torch.full((3,), -1, dtype=torch.int64) for _ in range(2)]
    got = {}

    def pack(face, buf):  # the packet names its sender and the side it was packed for
        buf.copy_(torch.tensor([rank, face, 7]))

    def unpack(face, buf):
        got[face] = buf.tolist()

    for _ in range(2):  # two exchanges in a row
        got.clear()
        run_exchange(dist, None, plan, send, recv, pack, unpack)
    dist.destroy_process_group()
    q.put((rank, neighbours(rank, world, periodic), got))


@pytest.mark.parametrize("world,periodic", [(2, False), (2, True), (3, False), (3, True)])
def test_each_face_receives_its_neighbours_planes(world, periodic):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, periodic, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, (down, up), got in out:
        # the z- face holds the top planes of the slab below, the z+ face the bottom planes
        # of the slab above
        assert got.get(0) == ([down, 1, 7] if down is not None else None)
        assert got.get(1) == ([up, 0, 7] if up is not None else None)
