"""Initial field evaluated on the GPU (clipb_init_device) against the host evaluation of
clipb_init, which follows NSAllen::initialCondition (NsAllen.cu:768-824) bit for bit.

Both evaluate c = 1/2 +- 1/2 tanh(2 sdf / W) in FP64 with the same operation order; only
tanh differs (CUDA's against the C library's), and cos in the signed distance of the
Rayleigh-Taylor perturbation, so the fields agree to a few units in the last place (at
most 8 here), and the states built from them follow suit.
"""
import os

import numpy as np
import pytest

from conftest import golden_config

import clip_b200 as cb

pytestmark = pytest.mark.gpu

CASES = ["drop2d_small", "bubble2d_walls", "rti2d_small", "drop3d_small", "bubble3d_walls", "rti3d_small",
         "inlet3d_small"]
ULP = 2.3e-16  # c lies in [0, 1]: one unit in the last place of 1 is 2.2e-16


@pytest.mark.parametrize("name", CASES)
def test_device_initial_field_matches_host(name):
    with cb.Solver(golden_config(name), "fp64") as s:
        s.init()
        host = {f: s.field(f) for f in ("c", "f", "g", "p")}
    with cb.Solver(golden_config(name), "fp64") as s:
        s.init(on_device=True)
        dev = {f: s.field(f) for f in ("c", "f", "g", "p")}
    dc = np.abs(dev["c"] - host["c"])
    assert dc.max() <= 8 * ULP, (name, dc.max(), int((dc > 0).sum()))
    for f in ("f", "g", "p"):
        scale = max(1e-300, float(np.abs(host[f]).max()))
        assert float(np.abs(dev[f] - host[f]).max()) <= 1e-13 * scale, f


def test_device_initial_field_of_the_3d_bubble_workload():
    """The 128x256x128 rising bubble (whole extent on the device in one launch): same
    initial state as the host evaluation, to rounding, in FP32 storage."""
    case = os.path.join(os.path.dirname(cb.__file__), "workloads", "bubble3d_128x256x128.txt")
    with cb.Solver(case, "fp32") as s:
        s.init()
        s.solve(3)
        host_c = s.interior_field("c")
        host_m = s.monitors()[0]
    with cb.Solver(case, "fp32") as s:
        s.init(on_device=True)
        s.solve(3)
        dev_c = s.interior_field("c")
        dev_m = s.monitors()[0]
    assert float(np.abs(dev_c - host_c).max()) <= 1e-6
    assert abs(dev_m - host_m) <= 1e-9 * abs(host_m)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_large_upload_sends_the_non_uniform_rows_and_keeps_every_bit(prec):
    """The 128x256x128 bubble is above the pinned-staging size, where clipb_init sends per z
    plane only the rows between the first and the last one that is not uniform, and fills
    the uniform rows on the device.  Its stored c (ghosts included) equals the host initial
    field (FP64: bit for bit; FP32: rounded), and so does a field passed by the caller
    through clipb_device_initializer with non-uniform values scattered over the bulk."""
    path = os.path.join(os.path.dirname(cb.__file__), "workloads", "bubble3d_128x256x128.txt")
    with cb.Solver(path, prec) as s:
        ref = s.initial_condition()
        s.init()
        c = s.field("c")[..., 0]
        whole = ref.size * 8
        sent = s.upload_bytes()
        assert np.array_equal(c, ref if prec == "fp64" else ref.astype(np.float32).astype(np.float64))
        assert 0 < sent < whole // 2, (sent, whole)
        rng = np.random.default_rng(5)
        other = ref.copy()
        idx = tuple(rng.integers(0, n, 40) for n in other.shape)
        other[idx] = rng.uniform(0.0, 1.0, 40)
        s.device_initializer(other)
        c = s.field("c")[..., 0]
        assert np.array_equal(c, other if prec == "fp64" else other.astype(np.float32).astype(np.float64))
