"""The allocation-free monitor entry point, clipb_field_sums_noalloc, through the C ABI.

It is meant for callers that cannot allocate device memory when they need the mass and
kinetic-energy monitors (a pool or arena owning the device, allocation-free real-time
loops, hosts that only hand over their own buffers).  Its block partials live in a fixed
array of the library's device image, so this test checks that it returns the same sums as
the ordinary entry point, clipb_monitors, on two calls in a row (the array is reused), that
a request beyond the array's capacity is rejected, and that a NaN in the caller's field is
reported as divergence, as clipb_monitors reports it.  The file sorts last so that a
failure here does not hide the results of the other tests.
"""
import ctypes

import numpy as np
import pytest

from conftest import golden_config

import clip_b200 as cb

pytestmark = pytest.mark.gpu


def _noalloc(L):
    f = L.clipb_field_sums_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_double,
                  ctypes.c_double, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


@pytest.mark.parametrize("name", ["drop2d_small", "drop3d_small"])
def test_noalloc_sums_match_monitors_on_two_calls(name):
    import torch

    L = cb.load_library()
    fn = _noalloc(L)
    with cb.Solver(golden_config(name), "fp64") as s:
        s.init()
        n = int(np.prod(s.interior))
        prm = s.params()
        rho_l, drho = prm["RhoL"], prm["RhoH"] - prm["RhoL"]
        # caller-owned device buffers (the caller allocates; the entry point does not)
        c = torch.empty(n, dtype=torch.float64, device="cuda")
        u = torch.empty(n * s.dim, dtype=torch.float64, device="cuda")
        out = torch.zeros(2, dtype=torch.float64, device="cuda")
        for call, steps in enumerate((5, 3)):
            s.solve(steps)
            ref_mass, ref_ke = s.monitors()
            s.field_device("c", c.data_ptr(), n)
            s.field_device("vel", u.data_ptr(), n * s.dim)
            torch.cuda.synchronize()
            out.fill_(-1.0)
            torch.cuda.synchronize()
            rc = fn(c.data_ptr(), u.data_ptr(), s.dim, n, rho_l, drho, out.data_ptr(), 0, None)
            assert rc == 0, L.clipb_last_error().decode()
            torch.cuda.synchronize()
            mass, ke = out.tolist()
            assert abs(mass - ref_mass) <= 1e-12 * abs(ref_mass), (call, mass, ref_mass)
            assert abs(ke - ref_ke) <= 1e-12 * abs(ref_ke) + 1e-300, (call, ke, ref_ke)


def test_noalloc_rejects_more_blocks_than_its_scratch_holds():
    import torch

    L = cb.load_library()
    fn = _noalloc(L)
    c = torch.zeros(10, dtype=torch.float64, device="cuda")
    u = torch.zeros(20, dtype=torch.float64, device="cuda")
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    rc = fn(c.data_ptr(), u.data_ptr(), 2, 10, 1.0, 0.0, out.data_ptr(), 1025, None)
    assert rc == -3
    assert b"nblocks must be in [1, 1024]" in L.clipb_last_error()
    rc = fn(c.data_ptr(), u.data_ptr(), 2, 10, 1.0, 0.0, out.data_ptr(), 7, None)
    assert rc == 0
    torch.cuda.synchronize()
    assert out.tolist() == [0.0, 0.0]


def test_noalloc_reports_nan_as_diverged():
    import torch

    L = cb.load_library()
    fn = _noalloc(L)
    c = torch.ones(1000, dtype=torch.float64, device="cuda")
    u = torch.zeros(3000, dtype=torch.float64, device="cuda")
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    rc = fn(c.data_ptr(), u.data_ptr(), 3, 1000, 1.0, 0.0, out.data_ptr(), 0, None)
    assert rc == 0
    assert out.tolist() == [1000.0, 0.0]
    c[417] = float("nan")  # host-side fault: a NaN in the caller's field
    rc = fn(c.data_ptr(), u.data_ptr(), 3, 1000, 1.0, 0.0, out.data_ptr(), 0, None)
    assert rc == -6, rc
    assert b"diverged" in L.clipb_last_error()
