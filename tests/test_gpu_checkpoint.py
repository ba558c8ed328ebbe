"""Checkpoint and resume: clipb_save writes the reference's CheckPointer files plus this
build's exact state; clipb_load resumes bit for bit from the latter, and from the
reference's files alone rebuilds the state by replaying the last step (c exact)."""
import os

import numpy as np
import pytest

from conftest import golden_config

import clip_b200 as cb

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["fp64", "fp32", "fp16"])
@pytest.mark.parametrize("name", ["drop2d_small", "bubble3d_walls", "inlet2d_small"])
def test_exact_resume(name, prec, tmp_path):
    cfg = golden_config(name)
    with cb.Solver(cfg, prec) as s:
        s.init()
        s.solve(13)
        s.save(tmp_path / "ck")
        s.solve(20)
        ref = {f: s.field(f) for f in ("c", "vel", "f", "g", "p")}
    with cb.Solver(cfg, prec) as s:
        s.load(tmp_path / "ck")
        assert s.steps == 13
        s.solve(20)
        assert s.steps == 33
        for f, r in ref.items():
            assert np.array_equal(s.field(f), r), f


def test_reference_files_layout(tmp_path):
    cfg = golden_config("drop2d_small")
    with cb.Solver(cfg, "fp64") as s:
        s.init()
        s.solve(5)
        s.save(tmp_path / "ck")
        n = int(np.prod(s.extent))
        for f, name in (("f", "dev_f"), ("g", "dev_g"), ("f_post", "dev_f_post"), ("g_post", "dev_g_post")):
            raw = np.fromfile(tmp_path / "ck" / f"{name}.bin", dtype=np.float64)
            assert raw.size == n * s.Q
            assert np.array_equal(raw.reshape(s.field(f).shape), s.field(f))
        ti = np.fromfile(tmp_path / "ck" / "timeInfo.bin", dtype=np.uint8)
        assert ti.size == 32 and int(np.frombuffer(ti[8:12].tobytes(), dtype=np.int32)[0]) == 5
        N = np.fromfile(tmp_path / "ck" / "domainSize.bin", dtype=np.float64)
        assert N.size == 3 and N[0] == s.extent[0] - 2


@pytest.mark.parametrize("name", ["drop2d_small", "rti2d_small"])
def test_resume_from_reference_files(name, tmp_path):
    cfg = golden_config(name)
    with cb.Solver(cfg, "fp64") as s:
        s.init()
        s.solve(30)
        s.save(tmp_path / "ck")
        c30, u30 = s.interior_field("c"), s.interior_field("vel")
        f30, g30 = s.field("f"), s.field("g")
        s.solve(10)
        c40 = s.interior_field("c")
    os.remove(tmp_path / "ck" / "clipb_state.bin")  # as the reference writes it
    with cb.Solver(cfg, "fp64") as s:
        s.load(tmp_path / "ck")
        assert s.steps == 30
        assert np.array_equal(s.interior_field("c"), c30)
        assert np.array_equal(s.field("f"), f30) and np.array_equal(s.field("g"), g30)
        u = s.interior_field("vel")
        assert np.abs(u - u30).max() <= 0.05 * np.abs(u30).max() + 1e-12
        s.solve(10)
        # the approximate previous velocity perturbs the continuation slightly (3.4e-6 in c
        # after 10 steps of the unstable RTI case, less for the drop)
        assert np.abs(s.interior_field("c") - c40).max() < 1e-5


def test_load_errors(tmp_path):
    with cb.Solver(golden_config("drop2d_small"), "fp64") as s:
        with pytest.raises(cb.ClipError):
            s.load(tmp_path / "missing")
        s.init()
        s.solve(2)
        s.save(tmp_path / "ck")
    with cb.Solver(golden_config("drop2d_64x128"), "fp64") as s:
        with pytest.raises(cb.ClipError, match="domain size"):
            s.load(tmp_path / "ck")
    with cb.Solver(golden_config("drop2d_small"), "fp32") as s:
        with pytest.raises(cb.ClipError, match="precision"):
            s.load(tmp_path / "ck")


@pytest.mark.parametrize("name,free_convect", [("outflow2d_small", True), ("drop2d_small", False)])
def test_free_convect_file_set(name, free_convect, tmp_path):
    """A free-convect case also writes the reference's dev_f_prev.bin / dev_g_prev.bin
    (CheckPointer.cu:69-73), which its load reads; they hold the post-streaming values, which
    the reference's next step copies into its prev arrays before reading them."""
    with cb.Solver(golden_config(name), "fp64") as s:
        s.init()
        s.solve(7)
        s.save(tmp_path / "ck")
        for prev, post in (("dev_f_prev", "f_post"), ("dev_g_prev", "g_post")):
            path = tmp_path / "ck" / f"{prev}.bin"
            assert path.exists() == free_convect
            if free_convect:
                raw = np.fromfile(path, dtype=np.float64)
                assert np.array_equal(raw.reshape(s.field(post).shape), s.field(post))
