"""Free-convect, Neumann and slip-wall sides (reference: src/solver/Solver.cu:248-542) on the
CUDA path, against the reference's own dumps and the CPU oracle.

The cases (tests/golden/configs) put each side type next to walls, periodic axes and a
velocity inlet, in 2D and 3D; their fixtures come from the reference's build, with the
harness setting the side types that its parser cannot reach (make_golden.py, BC_OVERRIDE).
"""
import json

import numpy as np
import pytest

from conftest import golden_config, golden_npz
import oracle as O

import clip_b200 as cb

pytestmark = pytest.mark.gpu

CASES = ["neumann2d_small", "outflow2d_small", "mixed2d_small", "slip2d_walls", "outflow3d_small",
         "neumann3d_small", "mixed3d_small"]


def _interior(a, dim):
    return a[1:-1, 1:-1] if dim == 2 else a[1:-1, 1:-1, 1:-1]


def _assert_equal(mine, ref, what):
    bad = np.argwhere(mine != ref)
    assert bad.size == 0, (f"{what}: {len(bad)} differ; first {tuple(bad[0])}: "
                           f"{mine[tuple(bad[0])]!r} vs {ref[tuple(bad[0])]!r}")


@pytest.mark.parametrize("name", CASES)
def test_fp64_bit_exact_vs_reference_without_fma(name):
    """c, p, rho, u at every dumped step equal the reference's (-fmad=false build)."""
    a = np.load(golden_npz(name + "_nofma"))
    meta = json.loads(bytes(a["meta"]).decode())
    with cb.Solver(golden_config(name), "fp64") as s:
        s.init()
        cur = 0
        for step in meta["dumps"]:
            s.solve(step - cur)
            cur = step
            for f in ("c", "p", "rho", "vel"):
                _assert_equal(_interior(s.field(f), s.dim), _interior(a[f"{f}_{step}"], s.dim),
                              f"{name} {f} step {step}")


@pytest.mark.parametrize("name", CASES)
def test_fp64_every_field_bit_exact_vs_oracle(name):
    """All eight fields (interior) after 0, 1, 2 and 7 steps, plus the c ghost layer:
    f_post and g_post carry the free-convect and Neumann values directly."""
    o = O.Oracle(golden_config(name))
    o.init()
    with cb.Solver(golden_config(name), "fp64") as s:
        s.init()
        cur = 0
        for step in (0, 1, 2, 7):
            s.solve(step - cur)
            o.solve(step - cur)
            cur = step
            for f in ("c", "p", "rho", "vel", "f", "g", "f_post", "g_post"):
                if step == 0 and f in ("f_post", "g_post"):
                    continue
                _assert_equal(_interior(s.field(f), s.dim), _interior(o.get(f), s.dim), f"{name} {f} step {step}")
            if step > 0:
                _assert_equal(s.field("c"), o.get("c"), f"{name} c with ghosts step {step}")


@pytest.mark.parametrize("name", [n for n in CASES if n != "slip2d_walls"])
def test_reduced_precision_with_open_sides(name):
    """FP32 within 1e-6 and FP16 within 2e-3 of FP64 in c after 40 steps (u within 1e-6
    of max |u| for FP32).  slip2d_walls starts from a square, whose symmetric centre makes
    the interface normal a matter of rounding (see the bubble2d_walls test)."""
    with cb.Solver(golden_config(name), "fp64") as s64:
        s64.init()
        s64.solve(40)
        c64, u64 = s64.interior_field("c"), s64.interior_field("vel")
    for prec, tol in (("fp32", 1e-6), ("fp16", 2e-3)):
        with cb.Solver(golden_config(name), prec) as s:
            s.init()
            s.solve(40)
            assert np.abs(s.interior_field("c") - c64).max() <= tol, prec
            if prec == "fp32":
                assert np.abs(s.interior_field("vel") - u64).max() <= 1e-6 * max(np.abs(u64).max(), 1e-12) + 1e-12


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("name", ["outflow3d_small", "mixed3d_small"])
def test_3d_launch_variants_agree(name, prec):
    """Every launch shape gives the same bits; the staged (TMA) variants resolve only wall,
    periodic and inlet sides and are unavailable here."""
    ref = None
    with cb.Solver(golden_config(name), prec) as s:
        nvar = s.get_launch()[2]
        for v in range(nvar):
            if v in (5, 6, 9):
                with pytest.raises(cb.ClipError):
                    s.set_launch(v, 4)
                continue
            if prec == "fp64" and v >= 7:
                with pytest.raises(cb.ClipError):
                    s.set_launch(v, 4)
                continue
            s.set_launch(v, 4)
            s.init()
            s.set_graphs(False)
            s.solve(9)
            out = [s.field(f) for f in ("c", "vel", "f_post", "g_post")]
            if ref is None:
                ref = out
            else:
                for f, a, b in zip(("c", "vel", "f_post", "g_post"), out, ref):
                    _assert_equal(_interior(a, 3), _interior(b, 3), f"variant {v} {f}")


@pytest.mark.parametrize("name", ["outflow2d_small", "mixed2d_small"])
def test_2d_launch_variants_agree(name):
    ref = None
    with cb.Solver(golden_config(name), "fp32") as s:
        for v in range(s.get_launch()[2]):
            s.set_launch(v, 5)
            s.init()
            s.solve(9)
            c = s.field("c")
            if ref is None:
                ref = c
            else:
                _assert_equal(c, ref, f"variant {v}")


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("name", ["outflow2d_small", "mixed3d_small"])
def test_checkpoint_resume_carries_free_convect_state(name, prec, tmp_path):
    with cb.Solver(golden_config(name), prec) as a:
        a.init()
        a.solve(10)
        a.save(tmp_path / "ck")
        a.solve(10)
        want = a.field("c")
    with cb.Solver(golden_config(name), prec) as b:
        b.load(tmp_path / "ck")
        assert b.steps == 10
        b.solve(10)
        _assert_equal(b.field("c"), want, "resumed c")
    # the reference's files alone do not hold the populations of the step before
    (tmp_path / "ck" / "clipb_state.bin").unlink()
    with cb.Solver(golden_config(name), prec) as c:
        with pytest.raises(cb.ClipError, match="free-convect"):
            c.load(tmp_path / "ck")


def test_batches_and_derivatives_reject_open_sides():
    with pytest.raises(cb.ClipError):
        cb.Batch([golden_config("outflow2d_small")], "fp32")
    with pytest.raises(cb.ClipError):
        cb.Batch([golden_config("neumann2d_small")], "fp32")
    with cb.Solver(golden_config("neumann2d_small"), "fp64") as s:
        with pytest.raises(cb.ClipError):
            s.objective(5, (10.0, 10.0))
