"""Staged 3D step (bulk tensor copies into shared memory) and the variants that keep the
next plane's g in shared memory, against the direct-load step.

Both launch shapes compute every node with the same arithmetic in the same order, so the
staged variants must reproduce the direct variant bit for bit; the FP32/FP16 accuracy
against FP64 is covered by test_gpu_parity.py for the direct variant.  The case is the
128 x 256 x 128 rising bubble (periodic x and z, walls in y): its interior tiles take the
staged path, its boundary tiles and the planes next to z = 1 and z = n the direct one.
"""
import os

import numpy as np
import pytest

import clip_b200 as cb

pytestmark = pytest.mark.gpu

CASE = os.path.join(os.path.dirname(cb.__file__), "workloads", "bubble3d_128x256x128.txt")
STAGED = (5, 6, 9)


def _run(prec, variant, seg, steps):
    with cb.Solver(CASE, prec) as s:
        s.init()
        s.set_launch(variant, seg)
        s.solve(steps)
        mass, ke = s.monitors()  # raises if a bounded wait of the staged step gave up
        out = {f: s.interior_field(f) for f in ("c", "p", "vel")}
        out["mass"] = mass
        out["ke"] = ke
    return out


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_staged_variants_available(prec):
    with cb.Solver(CASE, prec) as s:
        assert s.get_launch()[2] == 10
        for v in STAGED:
            s.set_launch(v, 32)


def test_staged_unavailable_for_fp64():
    with cb.Solver(CASE, "fp64") as s:
        assert s.get_launch()[2] == 5
        with pytest.raises(cb.ClipError):
            s.set_launch(5, 32)


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
@pytest.mark.parametrize("variant,seg", [(5, 32), (6, 32), (5, 128), (6, 7), (7, 16), (8, 5), (9, 32), (9, 7)])
def test_staged_equals_direct(prec, variant, seg):
    """21 steps (one 16-step graph + single launches): c, p, u identical to variant 0."""
    ref = _run(prec, 0, seg, 21)
    got = _run(prec, variant, seg, 21)
    for f in ("c", "p", "vel"):
        bad = np.argwhere(got[f] != ref[f])
        assert bad.size == 0, (f"{prec} variant {variant} seg {seg} {f}: {len(bad)} nodes differ; first "
                               f"{tuple(bad[0])}: {got[f][tuple(bad[0])]!r} vs {ref[f][tuple(bad[0])]!r}")
    assert got["mass"] == ref["mass"] and got["ke"] == ref["ke"]


@pytest.mark.parametrize("variant", STAGED)
def test_wait_that_runs_out_is_reported_and_the_context_stays_usable(variant):
    """A bounded wait that cannot be met (the first bulk load of every block expects 16 bytes
    more than its copies bring) gives up after 20000 cycles: the blocks drain their copies
    and return, the solver reports the device flag, and the next solver on the same device
    runs normally."""
    with cb.Solver(CASE, "fp32") as s:
        s.init()
        s.set_launch(variant, 32)
        s.set_wait_limit(20000, 16)
        s.solve(2)
        with pytest.raises(cb.ClipError, match="bounded wait"):
            s.monitors()
    ref = _run("fp32", 0, 32, 5)
    with cb.Solver(CASE, "fp32") as s:
        s.init()
        s.set_launch(variant, 32)
        s.set_wait_limit(0, 0)
        s.solve(5)
        mass, _ = s.monitors()
        assert np.array_equal(s.interior_field("c"), ref["c"])
        assert mass == ref["mass"]
