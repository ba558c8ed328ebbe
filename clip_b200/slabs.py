"""Slab decomposition of a 3D case along z (libclipb's clipb_slab_* entry points).

A case of N interior z planes is split into k slabs of whole planes; slab r is an
ordinary solver for its planes (``Slab``) that keeps, on each face bordering another slab,
the neighbour's boundary plane and the plane beyond it.  Before every step each such face
receives one packet from the neighbour (``Slab.pack`` there, ``Slab.unpack`` here), after
which the owned planes evolve exactly as in the whole case.

* ``SlabGroup``: k slabs on the current GPU, packets in device memory.  It proves the
  decomposition (results equal the whole case bit for bit) on one GPU.
* ``DistributedSlab``: one slab per rank of a ``torch.distributed`` process group (one GPU
  per rank), packets sent with point-to-point messages (NCCL over NVLink on GPUs).

The exchange runs in two phases, each with at most one message between two ranks in
each direction: (A) every slab sends its top planes to the slab above and receives from
the slab below into its z- face; (B) the reverse.  On a periodic z axis the slab above the
last one is the first one, so with two slabs both neighbours are the same rank and the
phases keep the two messages apart.
"""
import ctypes
import os

import numpy as np

from . import PRECISIONS, Solver, _check, config_summary, load_library

PERIODIC = 3  # side code of config_summary


def slab_ranges(nz, k):
    """Global plane ranges (1-based, inclusive) of k balanced slabs of nz planes."""
    if k < 1 or nz < 2 * k:
        raise ValueError(f"{nz} planes cannot make {k} slabs of at least two planes")
    out, start = [], 1
    for r in range(k):
        n = nz // k + (1 if r < nz % k else 0)
        out.append((start, start + n - 1))
        start += n
    return out


def neighbours(r, k, periodic):
    """(rank below, rank above) of slab r, None where the face is the case's boundary."""
    down = r - 1 if r > 0 else (k - 1 if periodic and k > 1 else None)
    up = r + 1 if r < k - 1 else (0 if periodic and k > 1 else None)
    return down, up


def exchange_faces(r, k, periodic):
    """clipb_slab_create's exchange_faces bits for slab r."""
    down, up = neighbours(r, k, periodic)
    return (1 if down is not None else 0) | (2 if up is not None else 0)


def exchange_plan(r, k, periodic):
    """The two phases of the exchange for slab r: lists of (op, peer, face) with op
    'send' (face = the side whose planes are packed: 1 = top, 0 = bottom) or 'recv' (face =
    the side that is unpacked)."""
    down, up = neighbours(r, k, periodic)
    phase_a, phase_b = [], []
    if up is not None:
        phase_a.append(("send", up, 1))
        phase_b.append(("recv", up, 1))
    if down is not None:
        phase_a.append(("recv", down, 0))
        phase_b.append(("send", down, 0))
    return [phase_a, phase_b]


class Slab(Solver):
    """Solver of global planes z_begin .. z_end of a 3D case (clipb_slab_create)."""

    def __init__(self, config_path, precision, z_begin, z_end, faces):
        L = load_library()
        self._h = ctypes.c_void_p()
        self._owned = True
        prec = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        _check(L.clipb_slab_create(os.fsencode(config_path), prec, int(z_begin), int(z_end), int(faces),
                                   ctypes.byref(self._h)))
        self.config_path = config_path
        self._describe()
        zb, ze, lo, hi = (ctypes.c_int() for _ in range(4))
        pb = ctypes.c_longlong()
        _check(L.clipb_slab_info(self._h, ctypes.byref(zb), ctypes.byref(ze), ctypes.byref(lo), ctypes.byref(hi),
                                 ctypes.byref(pb)))
        self.z_begin, self.z_end, self.zlo, self.zhi = zb.value, ze.value, lo.value, hi.value
        self.packet_bytes = pb.value
        self.faces = int(faces)

    def pack(self, toward, dev_ptr, stream=None):
        """Packet for the neighbour on side `toward`, on `stream` (a cudaStream_t as int;
        None: the slab's stream)."""
        _check(load_library().clipb_slab_pack(self._h, int(toward), ctypes.c_void_p(dev_ptr),
                                              ctypes.c_void_p(stream or 0)))

    def unpack(self, face, dev_ptr, stream=None):
        _check(load_library().clipb_slab_unpack(self._h, int(face), ctypes.c_void_p(dev_ptr),
                                                ctypes.c_void_p(stream or 0)))

    def step_part(self, part):
        """Part 1 (the planes packed for the neighbours) or part 2 (the rest) of a step."""
        _check(load_library().clipb_slab_step_part(self._h, int(part)))

    def own_field(self, name):
        """Interior nodes of the owned planes, reference layout [x][y][z][component]."""
        a = self.field(name)
        return a[1:-1, 1:-1, self.zlo:self.zhi + 1, :]


def _packets(k, nbytes, device):
    import torch
    return [torch.empty(nbytes, dtype=torch.uint8, device=device) for _ in range(k)]


class SlabGroup:
    """k slabs of one case on the current GPU, exchanging through device packets.
    overlap: each step updates the slabs' face planes first, then packs and unpacks on a
    second stream while the remaining planes update (clipb_slab_step_part)."""

    def __init__(self, config_path, precision="fp32", k=2, variant=None, seg=0, overlap=False):
        import torch
        summary = config_summary(config_path)
        if summary["dim"] != 3:
            raise ValueError("slabs split 3D cases")
        nz = summary["extent"][2] - 2
        self.periodic = summary["sides"][4] == PERIODIC
        self.k = k
        self.stream = torch.cuda.Stream()
        self.comm = torch.cuda.Stream() if overlap else None
        self.slabs = []
        for r, (zb, ze) in enumerate(slab_ranges(nz, k)):
            s = Slab(config_path, precision, zb, ze, exchange_faces(r, k, self.periodic))
            s.set_stream(self.stream.cuda_stream)
            if variant is not None:
                s.set_launch(variant, seg)
            self.slabs.append(s)
        nbytes = max(s.packet_bytes for s in self.slabs)
        self._up = _packets(k, nbytes, "cuda")    # packet of slab r for the slab above
        self._down = _packets(k, nbytes, "cuda")  # packet of slab r for the slab below

    def close(self):
        for s in self.slabs:
            s.close()
        self.slabs = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def exchange(self, stream=None):
        """Every face's packet, packed then unpacked on `stream` (None: the slabs' stream)."""
        k, p = self.k, self.periodic
        sp = stream.cuda_stream if stream is not None else None
        for r, s in enumerate(self.slabs):
            down, up = neighbours(r, k, p)
            if up is not None:
                s.pack(1, self._up[r].data_ptr(), sp)
            if down is not None:
                s.pack(0, self._down[r].data_ptr(), sp)
        for r, s in enumerate(self.slabs):
            down, up = neighbours(r, k, p)
            if down is not None:
                s.unpack(0, self._up[down].data_ptr(), sp)
            if up is not None:
                s.unpack(1, self._down[up].data_ptr(), sp)

    def init(self):
        for s in self.slabs:
            s.init()
        self.exchange()

    def solve(self, nsteps=1):
        for _ in range(nsteps):
            if self.comm is None:
                for s in self.slabs:
                    s.solve(1)
                self.exchange()
                continue
            for s in self.slabs:
                s.step_part(1)
            self.comm.wait_stream(self.stream)
            self.exchange(self.comm)
            for s in self.slabs:
                s.step_part(2)
            self.stream.wait_stream(self.comm)

    def field(self, name):
        """The whole case's interior field, [x][y][z][component], from the owned planes."""
        self.stream.synchronize()
        return np.concatenate([s.own_field(name) for s in self.slabs], axis=2)

    def monitors(self):
        m = ke = 0.0
        for s in self.slabs:
            a, b = s.monitors()
            m += a
            ke += b
        return m, ke


class DistributedSlab:
    """The slab of this rank of a torch.distributed process group (one GPU per rank).
    overlap: each step updates the face planes first, then packs, sends, receives and
    unpacks on a second stream while the remaining planes update.
    staging: "device" moves the packets as device tensors (NCCL); "host" copies each packed
    packet into pinned host memory, sends it from there and copies received packets back
    before unpacking them, for process groups whose backend moves host tensors only (gloo).
    None picks "host" for gloo groups and "device" otherwise."""

    def __init__(self, config_path, precision="fp32", group=None, variant=None, seg=0, overlap=False,
                 staging=None):
        import torch
        import torch.distributed as dist
        self.dist, self.group = dist, group
        if staging is None:
            staging = "host" if dist.get_backend(group) == "gloo" else "device"
        if staging not in ("host", "device"):
            raise ValueError("staging must be 'host' or 'device'")
        self.staging = staging
        self.rank, self.k = dist.get_rank(group), dist.get_world_size(group)
        summary = config_summary(config_path)
        nz = summary["extent"][2] - 2
        self.periodic = summary["sides"][4] == PERIODIC
        zb, ze = slab_ranges(nz, self.k)[self.rank]
        self.slab = Slab(config_path, precision, zb, ze, exchange_faces(self.rank, self.k, self.periodic))
        # the solver works on a stream of its own; packing, the point-to-point messages (which
        # follow torch's current stream) and unpacking run on it, or on `comm` when the
        # exchange overlaps the interior update
        self.compute = torch.cuda.Stream()
        self.comm = torch.cuda.Stream() if overlap else None
        self.slab.set_stream(self.compute.cuda_stream)
        if variant is not None:
            self.slab.set_launch(variant, seg)
        n = self.slab.packet_bytes
        self._dsend = [torch.empty(n, dtype=torch.uint8, device="cuda") for _ in range(2)]
        self._drecv = [torch.empty(n, dtype=torch.uint8, device="cuda") for _ in range(2)]
        if staging == "host":
            self._send = [torch.empty(n, dtype=torch.uint8).pin_memory() for _ in range(2)]
            self._recv = [torch.empty(n, dtype=torch.uint8).pin_memory() for _ in range(2)]
        else:
            self._send, self._recv = self._dsend, self._drecv
        self._plan = exchange_plan(self.rank, self.k, self.periodic)

    def exchange(self, stream=None):
        """One boundary exchange on torch stream `stream` (None: the slab's stream): packing,
        the messages, host staging copies and unpacking, in that stream's order."""
        import torch
        st = stream if stream is not None else self.compute
        with torch.cuda.stream(st):
            self._exchange(st.cuda_stream)

    def _exchange(self, sp):
        if self.staging == "device":
            pack = lambda face, buf: self.slab.pack(face, buf.data_ptr(), sp)
            unpack = lambda face, buf: self.slab.unpack(face, buf.data_ptr(), sp)
        else:
            def pack(face, host):
                self.slab.pack(face, self._dsend[face].data_ptr(), sp)
                host.copy_(self._dsend[face])  # waits for the pack (same stream), then the copy

            def unpack(face, host):
                # a blocking copy: the host buffer is free for the next receive when it returns
                self._drecv[face].copy_(host)
                self.slab.unpack(face, self._drecv[face].data_ptr(), sp)
        run_exchange(self.dist, self.group, self._plan, self._send, self._recv, pack, unpack)

    def init(self):
        self.slab.init()
        self.exchange()

    def solve(self, nsteps=1):
        for _ in range(nsteps):
            if self.comm is None:
                self.slab.solve(1)
                self.exchange()
                continue
            self.slab.step_part(1)
            self.comm.wait_stream(self.compute)
            self.exchange(self.comm)
            self.slab.step_part(2)
            self.compute.wait_stream(self.comm)

    def close(self):
        self.slab.close()


def run_exchange(dist, group, plan, send, recv, pack, unpack):
    """One exchange: for each phase, pack the sends, post the phase's sends and receives
    as one batch (NCCL runs a send and a receive between the same two ranks only when they
    are grouped), wait, unpack the receives.  send / recv: one buffer per face (0: z-,
    1: z+)."""
    for phase in plan:
        ops, unpacks = [], []
        for op, peer, face in phase:
            if op == "send":
                pack(face, send[face])
                ops.append(dist.P2POp(dist.isend, send[face], peer, group))
            else:
                ops.append(dist.P2POp(dist.irecv, recv[face], peer, group))
                unpacks.append(face)
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()
        for face in unpacks:
            unpack(face, recv[face])
