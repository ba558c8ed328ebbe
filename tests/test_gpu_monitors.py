"""Monitors summed inside the last step (clipb_solve_monitored) against the separate
reduction (clipb_monitors), which follows Reporter::sum (Reporter.cu:95-114).

The fused sums add the same FP64 per-node values (stored c, 0.5 rho |u|^2 of the stored u)
in another fixed order: per row segment of 32 nodes in the step, then over the segments.
So they agree with clipb_monitors to rounding, do not depend on the launch shape, and
leave the state exactly as clipb_solve does."""
import os

import numpy as np
import pytest

from conftest import golden_config

import clip_b200 as cb

pytestmark = pytest.mark.gpu

DIVERGED = -6  # CLIPB_E_DIVERGED
BUBBLE = os.path.join(os.path.dirname(cb.__file__), "workloads", "bubble3d_128x256x128.txt")


def _run(path, prec, variant, seg, steps, fused):
    with cb.Solver(path, prec) as s:
        s.init()
        s.set_launch(variant, seg)
        if fused:
            m, k = s.solve_monitored(steps)
        else:
            s.solve(steps)
            m, k = s.monitors()
        return m, k, s.interior_field("c"), s.interior_field("vel")


@pytest.mark.parametrize("name,prec", [("bubble3d_walls", "fp64"), ("rti3d_small", "fp64"), ("drop3d_small", "fp32"),
                                       ("inlet3d_small", "fp32"), ("outflow3d_small", "fp32"), (BUBBLE, "fp32"),
                                       (BUBBLE, "fp16")])
def test_fused_monitors_agree_with_the_separate_reduction(name, prec):
    """Mass within 1e-13 and kinetic energy within 1e-12 relative; c and u bit for bit."""
    path = name if os.path.isabs(name) else golden_config(name)
    m0, k0, c0, u0 = _run(path, prec, 0, 0, 7, fused=False)
    m1, k1, c1, u1 = _run(path, prec, 0, 0, 7, fused=True)
    assert np.array_equal(c0, c1) and np.array_equal(u0, u1)
    assert abs(m1 - m0) <= 1e-13 * abs(m0), (m0, m1)
    assert abs(k1 - k0) <= 1e-12 * abs(k0) + 1e-300, (k0, k1)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_fused_monitors_do_not_depend_on_the_launch_shape(prec):
    """Every direct-load 3D variant and several plane counts give the same bits; a staged
    variant (FP32) falls back to the separate reduction."""
    variants = [(0, 0), (1, 5), (2, 0), (3, 16), (4, 3)] + ([(7, 8), (8, 8), (8, 5)] if prec == "fp32" else [])
    ref = None
    for v, seg in variants:
        m, k, _, _ = _run(BUBBLE, prec, v, seg, 5, fused=True)
        if ref is None:
            ref = (m, k)
        assert (m, k) == ref, (v, seg, m, k, ref)
    if prec == "fp32":
        m, k, _, _ = _run(BUBBLE, prec, 5, 32, 5, fused=True)
        ms, ks, _, _ = _run(BUBBLE, prec, 5, 32, 5, fused=False)
        assert (m, k) == (ms, ks)


def test_2d_case_falls_back_to_the_separate_reduction():
    m0, k0, _, _ = _run(golden_config("drop2d_small"), "fp32", 0, 0, 9, fused=False)
    m1, k1, _, _ = _run(golden_config("drop2d_small"), "fp32", 0, 0, 9, fused=True)
    assert (m0, k0) == (m1, k1)


def test_fused_monitors_report_divergence():
    """A NaN planted in the initial field reaches the fused sums: CLIPB_E_DIVERGED."""
    with cb.Solver(golden_config("drop3d_small"), "fp32") as s:
        c = s.initial_condition()
        c[tuple(e // 2 for e in s.extent)] = np.nan
        s.device_initializer(c)
        with pytest.raises(cb.ClipError) as e:
            s.solve_monitored(3)
        assert e.value.code == DIVERGED
