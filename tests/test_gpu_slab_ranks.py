"""z slabs on separate processes (clip_b200.slabs.DistributedSlab): each rank owns one slab
of a small 3D case and the boundary planes move between the processes every step as real
packets, through a gloo process group with host staging (pack on the GPU, copy to pinned
host memory, send / receive, copy back, unpack).  The two or three ranks share the test
box's one GPU; no kernel of one rank waits on another (the exchange is host-side), so the
ranks may run in any order.  The owned planes must equal the whole case bit for bit."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)

pytestmark = pytest.mark.gpu

STEPS = 10


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, cfg, prec, overlap, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, REPO)
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    from clip_b200.slabs import DistributedSlab

    torch.cuda.set_device(0)
    dist.init_process_group("gloo", timeout=timedelta(seconds=120))
    ds = DistributedSlab(cfg, prec, overlap=overlap)
    assert ds.staging == "host"
    ds.init()
    ds.solve(STEPS)
    torch.cuda.synchronize()
    out = {f: ds.slab.own_field(f) for f in ("c", "vel", "p")}
    mon = ds.slab.monitors()
    z = (ds.slab.z_begin, ds.slab.z_end)
    ds.close()
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, z, out, mon))


def _run(cfg, prec, world, overlap):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, cfg, prec, overlap, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=300) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    return out


@pytest.mark.parametrize("name,world,prec,overlap", [("drop3d_small", 2, "fp64", False),
                                                     ("drop3d_small", 2, "fp32", True),
                                                     ("rti3d_small", 2, "fp32", False),
                                                     ("rti3d_small", 3, "fp16", True)])
def test_slab_ranks_equal_the_whole_case(name, world, prec, overlap):
    """drop3d_small: walls in z; rti3d_small: periodic z (first and last rank exchange)."""
    from conftest import golden_config

    import clip_b200 as cb

    cfg = golden_config(name)
    parts = _run(cfg, prec, world, overlap)
    with cb.Solver(cfg, prec) as s:
        s.init()
        s.set_graphs(False)
        s.solve(STEPS)
        want = {f: s.interior_field(f) for f in ("c", "vel", "p")}
        m_want, _ = s.monitors()
    for f in ("c", "vel", "p"):
        got = np.concatenate([p[2][f] for p in parts], axis=2)
        bad = np.argwhere(got != want[f])
        assert bad.size == 0, f"{name} {prec} {f}: {len(bad)} nodes differ, first {tuple(bad[0])}"
    zs = [p[1] for p in parts]
    assert zs[0][0] == 1 and all(zs[i][1] + 1 == zs[i + 1][0] for i in range(world - 1))
    m = sum(p[3][0] for p in parts)
    assert abs(m - m_want) <= 1e-12 * abs(m_want)
