"""The CPU oracle against the reference's own FP64 CUDA build (golden dumps).

Fixtures in tests/golden/ were produced by tests/golden/make_golden.py, which runs the
unmodified reference sources (compiled by oracle/Makefile) on a B200:
  <case>_nofma.npz  reference built with -fmad=false  -> the oracle must match bit for bit
  <case>.npz        reference as shipped (nvcc contracts mul+add into FMA) -> rounding-level
The reference is not deterministic on boxes periodic in two axes (its periodic ghost copy
writes edge cells from several threads, Solver.cu:96-136); those cases are checked for
the nondeterminism itself and for conservation only.
"""
import json

import numpy as np
import pytest

from conftest import golden_config, golden_npz
import oracle as O

DETERMINISTIC = ["drop2d_small", "bubble2d_walls", "rti2d_small", "inlet2d_small", "inlet2d_side",
                 "drop3d_small", "bubble3d_walls", "drop2d_64x128"]
# free-convect, Neumann and slip-wall sides (Solver.cu:248-542), alone and combined
OPEN_SIDES = ["neumann2d_small", "outflow2d_small", "mixed2d_small", "slip2d_walls", "outflow3d_small",
              "neumann3d_small", "mixed3d_small"]


def _meta(a):
    return json.loads(bytes(a["meta"]).decode())


def _run_and_compare(name, variant, check):
    a = np.load(golden_npz(name + variant))
    meta = _meta(a)
    o = O.Oracle(golden_config(name))
    o.init()
    cur = 0
    steps = sorted(set(meta["dumps"]) | set(meta.get("full", [])))
    compared = 0
    for s in steps:
        o.solve(s - cur)
        cur = s
        for k in a.files:
            if k == "meta" or k.endswith(("_sub", "_sum")):
                continue
            field, st = k.rsplit("_", 1)
            if int(st) != s:
                continue
            check(k, o.get(field), a[k])
            compared += 1
    assert compared > 0


@pytest.mark.parametrize("name", DETERMINISTIC + OPEN_SIDES)
def test_oracle_bit_exact_vs_reference_without_fma(name):
    def check(key, mine, ref):
        assert mine.shape == ref.shape, key
        bad = np.argwhere(mine != ref)
        assert bad.size == 0, f"{key}: {len(bad)} values differ, first at {bad[0]}: {mine[tuple(bad[0])]} vs {ref[tuple(bad[0])]}"

    _run_and_compare(name, "_nofma", check)


@pytest.mark.parametrize("name", ["drop2d_small", "rti2d_small", "inlet2d_small", "drop3d_small", "bubble3d_walls"])
def test_oracle_vs_shipped_reference_rounding_level(name):
    """The shipped (FMA) build differs from the oracle only by rounding: c, rho within
    1e-12 of max|field|, p and u within 1e-9 of max|field|, over these short runs."""

    def check(key, mine, ref):
        field = key.rsplit("_", 1)[0]
        if field not in ("c", "rho", "p", "vel"):
            return
        scale = max(np.abs(ref).max(), 1e-300)
        tol = 1e-12 if field in ("c", "rho") else 1e-9
        assert np.abs(mine - ref).max() <= tol * scale, key

    _run_and_compare(name, "", check)


@pytest.mark.parametrize("name", [n for n in OPEN_SIDES if n != "slip2d_walls"])
def test_oracle_open_sides_every_field_vs_shipped_reference(name):
    """Every dumped field, populations included (f_post/g_post carry the boundary
    conditions directly), within rounding of the shipped build: 1e-9 of max|field| over
    the interior nodes (the ghost layer's populations are scratch in both).  The slip-wall
    case starts from a square (as bubble2d_walls does), whose corners put |grad c| ~ 0 on
    the symmetry lines, where the normal amplifies FMA rounding; it is checked against the
    -fmad=false build only."""
    dim = 3 if "3d" in name else 2

    def check(key, mine, ref):
        inner = (slice(1, -1),) * dim
        mine, ref = mine[inner], ref[inner]
        scale = max(np.abs(ref).max(), 1e-300)
        assert np.abs(mine - ref).max() <= 1e-9 * scale, key

    _run_and_compare(name, "", check)


def test_oracle_drop_1000_steps_vs_shipped_reference():
    """The 64x128 drop, 1000 steps: the FMA build and the oracle agree to
    1e-15 for 100 steps; by 1000 steps rounding growth reaches ~1e-11 in c."""
    a = np.load(golden_npz("drop2d_64x128"))
    o = O.Oracle(golden_config("drop2d_64x128"))
    o.init()
    o.solve(100)
    assert np.abs(o.get("c") - a["c_100"]).max() < 1e-14
    o.solve(900)
    assert np.abs(o.get("c") - a["c_1000"]).max() < 1e-10
    ref_mass = a["c_1000"][1:-1, 1:-1].sum()
    assert abs(o.mass() - ref_mass) <= 1e-13 * abs(ref_mass)


def test_reference_is_nondeterministic_when_doubly_periodic():
    """Two identical runs of the reference on an x/z-periodic 3D box differ (ghost copy race)."""
    a = np.load(golden_npz("rti3d_small"))
    b = np.load(golden_npz("rti3d_small_repeat"))
    assert np.abs(a["c_20"] - b["c_20"]).max() > 1e-6


def test_oracle_doubly_periodic_conserves_mass_unlike_reference():
    """With true periodic images the oracle conserves sum(c) to rounding; the reference's
    racy edge copies lose conservation (both of its runs drift by more than 1e-8)."""
    o = O.Oracle(golden_config("rti3d_small"))
    o.init()
    m0 = o.mass()
    o.solve(20)
    assert abs(o.mass() - m0) <= 1e-13 * abs(m0)
    for name in ("rti3d_small", "rti3d_small_repeat"):
        a = np.load(golden_npz(name))
        ref = a["c_20"][1:-1, 1:-1, 1:-1].sum()
        assert abs(ref - m0) > 1e-8 * abs(m0)


def test_oracle_rti_256x1024_vs_reference_without_fma():
    """The 256x1024 RTI grid, 2000 steps: bit-exact against the -fmad=false build
    on the committed stride-2 subsample and the global sums."""
    a = np.load(golden_npz("rti2d_256x1024_nofma"))
    o = O.Oracle(golden_config("rti2d_256x1024"))
    o.init()
    o.solve(2000)
    for f in ("c", "p", "vel"):
        sub = o.interior(f)[::2, ::2, :, :]
        assert np.array_equal(sub, a[f + "_2000_sub"]), f
    ci = o.interior("c")
    assert ci.sum() == a["c_2000_sum"][0]
