"""CUDA path (libclipb.so through its C ABI) against the CPU oracle and the reference dumps.

FP64 is the parity path: compiled without FMA contraction it must equal the oracle -- and
therefore the reference built with -fmad=false -- bit for bit, on every field the
reference exposes (c, p, rho, u, f, g, f_post, g_post).  FP32 and FP16 storage are
checked against FP64 with the tolerances written in each test.
"""
import json

import numpy as np
import pytest

from conftest import golden_config, golden_npz
import oracle as O

import clip_b200 as cb

pytestmark = pytest.mark.gpu

DETERMINISTIC = ["drop2d_small", "bubble2d_walls", "rti2d_small", "inlet2d_small", "inlet2d_side",
                 "drop3d_small", "bubble3d_walls", "drop2d_64x128"]
ALL_SMALL = ["drop2d_small", "bubble2d_walls", "rti2d_small", "inlet2d_small", "inlet2d_side",
             "drop3d_small", "bubble3d_walls", "rti3d_small", "inlet3d_small"]


def _interior(a, dim):
    return a[1:-1, 1:-1] if dim == 2 else a[1:-1, 1:-1, 1:-1]


def _assert_equal(mine, ref, what):
    bad = np.argwhere(mine != ref)
    assert bad.size == 0, (f"{what}: {len(bad)} differ; first {tuple(bad[0])}: "
                           f"{mine[tuple(bad[0])]!r} vs {ref[tuple(bad[0])]!r}")


@pytest.mark.parametrize("name", DETERMINISTIC)
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
                ref = a[f"{f}_{step}"]
                mine = s.field(f)
                _assert_equal(_interior(mine, s.dim), _interior(ref, s.dim), f"{name} {f} step {step}")


@pytest.mark.parametrize("name", ALL_SMALL)
def test_fp64_every_field_bit_exact_vs_oracle(name):
    """All eight fields (interior) after 0, 1, 2 and 7 steps, plus the c ghost layer."""
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


def test_fp64_rti_256x1024_2000_steps_bit_exact():
    """The 256x1024 RTI grid, 2000 steps, against the -fmad=false reference (stride-2 sample)."""
    a = np.load(golden_npz("rti2d_256x1024_nofma"))
    with cb.Solver(golden_config("rti2d_256x1024"), "fp64") as s:
        s.init()
        s.solve(2000)
        for f in ("c", "p", "vel"):
            sub = s.interior_field(f)[::2, ::2]
            _assert_equal(sub, a[f + "_2000_sub"], f)
        m, _ = s.monitors()
        assert abs(m - a["c_2000_sum"][0]) <= 1e-12 * abs(m)


def test_fp64_shipped_reference_rounding_level_1000_steps():
    """The shipped (FMA) reference build after 1000 steps of the 64x128 drop: the FP64 path
    differs from it only by FMA rounding grown by the dynamics (1e-10 of max |c|)."""
    a = np.load(golden_npz("drop2d_64x128"))
    with cb.Solver(golden_config("drop2d_64x128"), "fp64") as s:
        s.init()
        s.solve(1000)
        c = s.field("c")
        assert np.abs(_interior(c - a["c_1000"], 2)).max() < 1e-10


@pytest.mark.parametrize("name", ["drop2d_small", "drop3d_small", "rti3d_small", "bubble3d_walls"])
def test_monitors_match_oracle(name):
    o = O.Oracle(golden_config(name))
    o.init()
    o.solve(5)
    with cb.Solver(golden_config(name), "fp64") as s:
        s.init()
        s.solve(5)
        m, ke = s.monitors()
        assert abs(m - o.mass()) <= 1e-12 * abs(o.mass())
        rho = _interior(o.get("rho"), s.dim)[..., 0]
        u = _interior(o.get("vel"), s.dim)
        ke_ref = float((0.5 * rho * (u * u).sum(axis=-1)).sum())
        assert abs(ke - ke_ref) <= 1e-10 * abs(ke_ref) + 1e-300


def test_monitors_conserve_mass_fp64():
    with cb.Solver(golden_config("drop2d_64x128"), "fp64") as s:
        s.init()
        m0, _ = s.monitors()
        s.solve(1000)
        m1, _ = s.monitors()
        assert abs(m1 - m0) <= 1e-13 * abs(m0)


@pytest.mark.parametrize("name,steps", [("drop2d_64x128", 1000), ("drop3d_small", 200), ("rti2d_small", 300)])
def test_fp32_within_1e5_of_fp64(name, steps):
    """FP32 populations: max |c32 - c64| <= 1e-5 and mass drift <= 1e-6 relative."""
    with cb.Solver(golden_config(name), "fp64") as s64, cb.Solver(golden_config(name), "fp32") as s32:
        s64.init()
        s32.init()
        m0, _ = s64.monitors()
        s64.solve(steps)
        s32.solve(steps)
        c64, c32 = s64.interior_field("c"), s32.interior_field("c")
        assert np.abs(c32 - c64).max() <= 1e-5
        m32, _ = s32.monitors()
        assert abs(m32 - m0) <= 1e-6 * abs(m0)


@pytest.mark.parametrize("name", ["rti3d_small", "inlet2d_small", "inlet2d_side", "inlet3d_small", "bubble3d_walls"])
def test_reduced_precision_across_boundaries(name):
    """Shifted g storage across periodic wraps, walls and inlet planes: FP32 within 1e-6 and
    FP16 within 2e-3 of FP64 after 40 steps (u within 1e-6 of max |u| for FP32)."""
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


def test_fp32_ill_conditioned_case_within_reference_build_spread():
    """bubble2d_walls: at the square bubble's symmetric centre |grad c| ~ 1e-17, so the
    interface normal grad c / |grad c| is set by rounding.  The reference's own builds (FMA
    and -fmad=false) already differ there; FP32 must stay within 5x that spread."""
    a = np.load(golden_npz("bubble2d_walls"))
    b = np.load(golden_npz("bubble2d_walls_nofma"))
    spread = np.abs(_interior(a["c_40"], 2) - _interior(b["c_40"], 2)).max()
    assert spread > 1e-6
    with cb.Solver(golden_config("bubble2d_walls"), "fp64") as s64, \
            cb.Solver(golden_config("bubble2d_walls"), "fp32") as s32:
        s64.init()
        s32.init()
        s64.solve(40)
        s32.solve(40)
        assert np.abs(s32.interior_field("c") - s64.interior_field("c")).max() <= 5 * spread


@pytest.mark.parametrize("name,steps", [("drop2d_64x128", 200), ("drop3d_small", 50)])
def test_fp16_storage_error_bounded(name, steps):
    """FP16 population storage (scaled f, w_q c-shifted g): max |c16 - c64| <= 2e-3."""
    with cb.Solver(golden_config(name), "fp64") as s64, cb.Solver(golden_config(name), "fp16") as s16:
        s64.init()
        s16.init()
        s64.solve(steps)
        s16.solve(steps)
        err = np.abs(s16.interior_field("c") - s64.interior_field("c")).max()
        assert err <= 2e-3, err


def test_reference_facade_matches_solver():
    """The reference-shaped call sequence (src/main.cu:53-89) drives the same kernels."""
    idata = cb.InputData(golden_config("drop2d_small"))
    dom = cb.Domain(idata)
    geo = cb.Geometry(idata)
    bc = cb.Boundary(idata, dom)
    DA = cb.DataArray(idata, dom, bc)
    DA.createVectors()
    ns = cb.NSAllen(idata, dom, DA, bc, geo)
    ns.initialCondition()
    DA.updateDevice()
    ns.deviceInitializer()
    for _ in range(10):
        ns.solve()
    host = DA.updateHost()
    o = O.Oracle(golden_config("drop2d_small"))
    o.init()
    o.solve(10)
    _assert_equal(_interior(host["c"], 2), _interior(o.get("c"), 2), "facade c")


def test_errors_are_reported_not_fatal():
    with cb.Solver(golden_config("drop2d_small"), "fp64") as s:
        with pytest.raises(cb.ClipError) as e:
            s.solve(1)  # before init
        assert e.value.code == -4
        s.init()
        rc = cb.load_library().clipb_get_field(s._h, 0, cb._dptr(np.empty(3)), 3)
        assert rc == -3 and b"count must be" in cb.load_library().clipb_last_error()
        s.solve(2)
        assert s.steps == 2
