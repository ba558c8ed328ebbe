"""Boundary types accepted by the config reader (CPU only): free convect, Neumann and slip
wall next to the reference's wall, periodic and velocity sides, with the same acceptance
rules in the CUDA library's reader and in the oracle."""
import os

import pytest

from conftest import golden_config
import oracle as O

import clip_b200 as cb

WALL, SLIP, FREE, PERIODIC, NEUMANN, VELOCITY = 0, 1, 2, 3, 4, 5


def _config(tmp_path, sides):
    base = open(golden_config("drop2d_small")).read()
    head = base.split("boundary = [")[0]
    blocks = "".join(f'  {{\n    side = "{s}"\n    type = "{t}"\n  }},\n' for s, t in sides)
    p = tmp_path / "config.txt"
    p.write_text(head + "boundary = [\n" + blocks + "]\n")
    return str(p)


def _accepts(path):
    ok_lib = ok_orc = True
    try:
        cb.config_summary(path)
    except cb.ClipError:
        ok_lib = False
    try:
        O.Oracle(path)
    except ValueError:
        ok_orc = False
    assert ok_lib == ok_orc, "library and oracle disagree"
    return ok_lib


@pytest.mark.parametrize("spelling", ["free convect", "freeconvect", "Free Convect"])
def test_free_convect_reachable_in_both_spellings(tmp_path, spelling):
    p = _config(tmp_path, [("x-", "periodic"), ("x+", "periodic"), ("y-", spelling), ("y+", "wall")])
    assert _accepts(p)
    assert cb.config_summary(p)["sides"][:4] == [PERIODIC, PERIODIC, FREE, WALL]


def test_neumann_and_slip_wall(tmp_path):
    p = _config(tmp_path, [("x-", "neumann"), ("x+", "slip wall"), ("y-", "wall"), ("y+", "free convect")])
    assert _accepts(p)
    assert cb.config_summary(p)["sides"][:4] == [NEUMANN, SLIP, WALL, FREE]


@pytest.mark.parametrize("sides", [
    # two adjacent sides of one of these types: the reference's threads race on their edge
    [("x-", "neumann"), ("x+", "wall"), ("y-", "neumann"), ("y+", "wall")],
    [("x-", "free convect"), ("x+", "wall"), ("y-", "wall"), ("y+", "free convect")],
    # a slip wall without a wall side gets no bounce-back in the reference
    [("x-", "periodic"), ("x+", "periodic"), ("y-", "slip wall"), ("y+", "neumann")],
    # do nothing / unknown
    [("x-", "periodic"), ("x+", "periodic"), ("y-", "do nothing"), ("y+", "wall")],
    [("x-", "periodic"), ("x+", "periodic"), ("y-", "outflow"), ("y+", "wall")],
])
def test_rejected_side_combinations(tmp_path, sides):
    assert not _accepts(_config(tmp_path, sides))


def test_opposite_sides_of_one_type_accepted(tmp_path):
    p = _config(tmp_path, [("x-", "neumann"), ("x+", "neumann"), ("y-", "free convect"), ("y+", "wall")])
    assert _accepts(p)
