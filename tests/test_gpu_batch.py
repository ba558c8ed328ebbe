"""Batched 2D cases (one persistent launch per step over many cases) against single
solvers of the same configs.  The batched kernel runs the same per-tile code on the same
inputs, so every field must match bit for bit, FP64 and FP32; one FP64 case is also checked
against the CPU oracle."""
import numpy as np
import pytest

import clip_b200 as cb
import oracle as O

pytestmark = pytest.mark.gpu

SEED = 12345


def _texts(n, seed=SEED):
    return [cb.seeded_case_config(seed, i) for i in range(n)]


def _single(text, prec, steps, tmp_path, i):
    p = tmp_path / f"single{i}.txt"
    p.write_text(text)
    with cb.Solver(str(p), prec) as s:
        s.init()
        s.solve(steps)
        return {f: s.interior_field(f) for f in ("c", "p", "vel", "g")}, s.monitors()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_batch_equals_single_solvers(prec, tmp_path):
    texts = _texts(6)
    steps = 21  # one 16-step graph replay plus single launches
    with cb.Batch(texts, prec, texts=True) as b:
        b.init()
        b.solve(steps)
        mass, ke = b.monitors()
        for i, t in enumerate(texts):
            ref, (m, k) = _single(t, prec, steps, tmp_path, i)
            s = b.case(i)
            assert s.steps == steps
            for f, r in ref.items():
                got = s.interior_field(f)
                assert np.array_equal(got, r), f"case {i} {f}: max diff {np.abs(got - r).max()}"
            assert mass[i] == m and ke[i] == k


def test_sequential_equals_batched_and_launch_shape_is_neutral():
    texts = _texts(5, seed=7)
    out = []
    for mode in ("batched", "sequential", "shape"):
        with cb.Batch(texts, "fp32", texts=True) as b:
            b.init()
            if mode == "shape":
                b.set_launch(1, 5, 1)
            if mode == "sequential":
                b.solve_sequential(18)
            else:
                b.solve(18)
            out.append([b.case(i).interior_field("c") for i in range(len(texts))])
    for i in range(len(texts)):
        assert np.array_equal(out[0][i], out[1][i])
        assert np.array_equal(out[0][i], out[2][i])


def test_batch_fp64_case_matches_oracle(tmp_path):
    # the smallest of the first seeded cases, against the CPU restatement of the step
    texts = _texts(8)
    sizes = []
    for i, t in enumerate(texts):
        p = tmp_path / f"c{i}.txt"
        p.write_text(t)
        e = cb.config_summary(str(p))["extent"]
        sizes.append((e[0] * e[1], i, str(p)))
    _, idx, path = min(sizes)
    o = O.Oracle(path)
    o.init()
    o.solve(12)
    with cb.Batch(texts, "fp64", texts=True) as b:
        b.init()
        b.solve(12)
        s = b.case(idx)
        for f in ("c", "p", "vel"):
            mine = s.interior_field(f)
            ref = o.interior(f)
            assert np.array_equal(mine.reshape(ref.shape), ref), f


def test_batch_autotune_keeps_results():
    texts = _texts(4, seed=3)
    with cb.Batch(texts, "fp32", texts=True) as b:
        b.init()
        v, r, bps, ms = b.autotune(2)
        assert ms > 0 and r in (4, 8, 16, 32, 64)
        b.solve(10)
        c_tuned = [b.case(i).interior_field("c") for i in range(4)]
    with cb.Batch(texts, "fp32", texts=True) as b:
        b.init()
        b.solve(10)
        for i in range(4):
            assert np.array_equal(b.case(i).interior_field("c"), c_tuned[i])


def test_batch_rejects_bad_input(tmp_path):
    with pytest.raises(cb.ClipError):
        cb.Batch(["case = drop\n"], "fp32", texts=True)
    with cb.Batch(_texts(2), "fp32", texts=True) as b:
        with pytest.raises(cb.ClipError):
            b.solve(1)  # before init
        with pytest.raises(cb.ClipError):
            b.set_launch(9, 8)
