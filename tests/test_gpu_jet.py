"""Case 'jet' (velocity inlet at y+, free-convect outflow at y-, periodic x and z; the shape
of the reference's examples/3D/Jet/config.txt) on the CUDA path against the CPU oracle.

The reference reads an uninitialised body force for this case (NsAllen.cu:460-474), so its
own runs give no fixture; the oracle and this library define the jet's body force as zero
and are compared with each other.  The derived sigma and mu_H (InputData.cu:99-107) are
checked against the oracle in test_abi.py."""
import numpy as np
import pytest

from conftest import golden_config
import oracle as O

import clip_b200 as cb

pytestmark = pytest.mark.gpu

NAME = "jet3d_small"


def _interior(a):
    return a[1:-1, 1:-1, 1:-1]


def test_jet_fp64_bit_exact_vs_oracle():
    o = O.Oracle(golden_config(NAME))
    o.init()
    with cb.Solver(golden_config(NAME), "fp64") as s:
        s.init()
        cur = 0
        for step in (0, 1, 5, 20):
            s.solve(step - cur)
            o.solve(step - cur)
            cur = step
            for f in ("c", "p", "rho", "vel", "f", "g"):
                mine, ref = _interior(s.field(f)), _interior(o.get(f))
                bad = np.argwhere(mine != ref)
                assert bad.size == 0, f"{f} step {step}: {len(bad)} differ, first {tuple(bad[0])}"
        m, _ = s.monitors()
        assert abs(m - o.mass()) <= 1e-12 * abs(m)


def test_jet_reduced_precision():
    with cb.Solver(golden_config(NAME), "fp64") as s64:
        s64.init()
        s64.solve(40)
        c64 = s64.interior_field("c")
    for prec, tol in (("fp32", 1e-6), ("fp16", 2e-3)):
        with cb.Solver(golden_config(NAME), prec) as s:
            s.init()
            s.solve(40)
            assert np.abs(s.interior_field("c") - c64).max() <= tol, prec
