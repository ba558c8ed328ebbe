"""Failure detection of the step, made on the host (no GPU fault, trap or hang).

The reference's only failure check is the NaN test of its mass monitor
(Reporter.cu:124-144, Logger::Error throws).  Here clipb_monitors returns CLIPB_E_DIVERGED
instead; these tests plant the NaN in a host-prepared initial field, upload it through
clipb_device_initializer and step.  The staged step's bounded waits are covered in
test_gpu_staged.py.
"""
import numpy as np
import pytest

from conftest import golden_config

import clip_b200 as cb

pytestmark = pytest.mark.gpu

DIVERGED = -6


@pytest.mark.parametrize("name", ["drop2d_small", "drop3d_small"])
@pytest.mark.parametrize("prec", ["fp64", "fp32", "fp16"])
def test_nan_in_the_initial_field_is_reported_as_divergence(name, prec):
    with cb.Solver(golden_config(name), prec) as s:
        c = s.initial_condition()
        mid = tuple(e // 2 for e in s.extent)
        c[mid] = np.nan
        s.device_initializer(c)
        s.solve(3)
        with pytest.raises(cb.ClipError) as ei:
            s.monitors()
        assert ei.value.code == DIVERGED
        assert "diverged" in str(ei.value)


def test_clean_solver_after_a_diverged_one():
    """A diverged solver leaves the device and the library usable."""
    with cb.Solver(golden_config("drop2d_small"), "fp32") as s:
        c = s.initial_condition()
        c[3, 3, 0] = np.nan
        s.device_initializer(c)
        s.solve(5)
        with pytest.raises(cb.ClipError):
            s.monitors()
    with cb.Solver(golden_config("drop2d_small"), "fp32") as s:
        s.init()
        s.solve(5)
        mass, ke = s.monitors()
        assert np.isfinite(mass) and np.isfinite(ke)
