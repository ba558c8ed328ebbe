"""z slabs (clipb_slab_*) on one GPU: k slabs exchanging their boundary planes through
device packets must reproduce the whole case bit for bit, in every precision, on walled
and periodic z axes.  (Several GPUs move the same packets with NCCL, clip_b200.slabs.)"""
import numpy as np
import pytest

from conftest import golden_config

import clip_b200 as cb
from clip_b200.slabs import Slab, SlabGroup

pytestmark = pytest.mark.gpu


def _whole(name, prec, steps, variant=None):
    with cb.Solver(golden_config(name), prec) as s:
        if variant is not None:
            s.set_launch(variant, 4)
        s.init()
        s.set_graphs(False)
        s.solve(steps)
        return {f: s.interior_field(f) for f in ("c", "vel", "p")}, s.monitors()


def _assert_equal(mine, ref, what):
    bad = np.argwhere(mine != ref)
    assert bad.size == 0, f"{what}: {len(bad)} differ, first {tuple(bad[0])}: {mine[tuple(bad[0])]!r} vs {ref[tuple(bad[0])]!r}"


@pytest.mark.parametrize("overlap", [False, True])
@pytest.mark.parametrize("prec", ["fp64", "fp32", "fp16"])
@pytest.mark.parametrize("name,k", [("drop3d_small", 2), ("drop3d_small", 3), ("rti3d_small", 2),
                                    ("rti3d_small", 4), ("bubble3d_walls", 2)])
def test_slabs_equal_the_whole_case(name, k, prec, overlap):
    """drop3d_small / bubble3d_walls: walls in z; rti3d_small: periodic z (the first and
    last slabs exchange too).  overlap: the step in two parts, with the packets moved on a
    second stream while the planes away from the faces update (slabs of more than 4 planes
    split; smaller ones take the whole step in part 1)."""
    steps = 12
    want, (m_want, _) = _whole(name, prec, steps)
    with SlabGroup(golden_config(name), prec, k, overlap=overlap) as grp:
        grp.init()
        grp.solve(steps)
        for f in ("c", "vel", "p"):
            _assert_equal(grp.field(f), want[f], f"{name} k={k} {prec} {f}")
        m, _ = grp.monitors()
        assert abs(m - m_want) <= 1e-12 * abs(m_want)


@pytest.mark.parametrize("overlap", [False, True])
@pytest.mark.parametrize("variant", [0, 1, 3, 7, 8])
def test_slabs_with_each_launch_shape(variant, overlap):
    want, _ = _whole("drop3d_small", "fp32", 9)
    with SlabGroup(golden_config("drop3d_small"), "fp32", 3, variant=variant, seg=3, overlap=overlap) as grp:
        grp.init()
        grp.solve(9)
        _assert_equal(grp.field("c"), want["c"], f"variant {variant}")


def test_slab_arguments_are_checked():
    cfg = golden_config("drop3d_small")  # 14 interior planes, walls in z
    with pytest.raises(cb.ClipError):
        Slab(cfg, "fp32", 3, 3, 3)  # one plane
    with pytest.raises(cb.ClipError):
        Slab(cfg, "fp32", 1, 7, 3)  # exchange on the case's wall
    with pytest.raises(cb.ClipError):
        Slab(cfg, "fp32", 5, 9, 2)  # an inner face not exchanged
    with pytest.raises(cb.ClipError):
        Slab(golden_config("inlet3d_small"), "fp32", 1, 7, 2)  # velocity sides
    s = Slab(cfg, "fp32", 1, 7, 2)
    assert (s.z_begin, s.z_end, s.zlo, s.zhi) == (1, 7, 1, 7)
    assert s.interior[2] == 8  # 7 own planes + the neighbour's boundary plane
    s.init()
    with pytest.raises(cb.ClipError):
        s.pack(0, 0)  # null packet
    s.close()


def test_slab_vts_files_cover_their_own_planes(tmp_path):
    """Each slab writes its own planes at their global z; together they hold the whole
    case's arrays."""
    from test_vts import parse_binary

    name = "drop3d_small"
    with cb.Solver(golden_config(name), "fp64") as s:
        s.init()
        s.solve(5)
        _, whole = parse_binary(s.write_vts(tmp_path / "whole", "r", "binary64"))
    with SlabGroup(golden_config(name), "fp64", 3) as grp:
        grp.init()
        grp.solve(5)
        parts = []
        for r, sl in enumerate(grp.slabs):
            head, arrays = parse_binary(sl.write_vts(tmp_path / f"slab{r}", "r", "binary64"))
            assert f'WholeExtent="1 16 1 20 {sl.z_begin} {sl.z_end}"' in head
            parts.append(arrays)
    for k in ("Points", "Velocity", "C", "P", "Rho"):
        np.testing.assert_array_equal(np.concatenate([p[k] for p in parts]), whole[k], err_msg=k)


def test_split_step_order_is_checked():
    cfg = golden_config("drop3d_small")
    with cb.Solver(cfg, "fp32") as whole:
        whole.init()
        with pytest.raises(cb.ClipError, match="not a slab"):
            load_step_part(whole, 1)
    with Slab(cfg, "fp32", 1, 7, 2) as s:
        s.init()
        with pytest.raises(cb.ClipError, match="before part 1"):
            s.step_part(2)
        s.step_part(1)
        with pytest.raises(cb.ClipError, match="part 2"):
            s.solve(1)
        with pytest.raises(cb.ClipError, match="part 2"):
            s.step_part(1)
        s.step_part(2)
        assert s.steps == 1
        with pytest.raises(cb.ClipError):
            s.step_part(3)


def load_step_part(solver, part):
    """clipb_slab_step_part on any solver handle (the Python Slab class only wraps slabs)."""
    from clip_b200 import _check, load_library
    _check(load_library().clipb_slab_step_part(solver._h, part))
