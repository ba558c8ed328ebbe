"""Host-side checks of libclipb.so that need no GPU: exported symbols and config parsing."""
import os
import re

import numpy as np
import pytest

from conftest import REPO, golden_config
import oracle as O

import clip_b200 as cb

CONFIGS = sorted(f[:-4] for f in os.listdir(os.path.join(REPO, "tests", "golden", "configs")))


def test_library_exports_every_declared_symbol():
    header = open(os.path.join(REPO, "include", "clipb.h")).read()
    declared = set(re.findall(r"\b(clipb_[a-z_0-9]+)\s*\(", header))
    L = cb.load_library()
    missing = [n for n in sorted(declared) if not hasattr(L, n)]
    assert not missing, missing
    assert declared == set(cb.EXPORTS)


@pytest.mark.parametrize("name", CONFIGS)
def test_config_parser_matches_oracle(name):
    path = golden_config(name)
    mine = cb.config_summary(path)
    o = O.Oracle(path)
    ref = o.params()
    for k, v in ref.items():
        assert mine["params"][k] == v, k  # bit-identical derivation
    assert mine["dim"] == o.dim
    assert tuple(mine["extent"]) == o.extent
    types, _vals = o.boundary()
    assert mine["sides"][: 2 * o.dim] == types[: 2 * o.dim]


def test_workload_configs_parse():
    for f in sorted(os.listdir(cb.WORKLOADS)):
        s = cb.config_summary(os.path.join(cb.WORKLOADS, f))
        assert s["dim"] in (2, 3)


def _write(tmp_path, text):
    p = tmp_path / "config.txt"
    p.write_text(text)
    return str(p)


BASE = """case = drop
N = [16, 16, 1]
referenceLength = 8
We = 2
Re = 20
gravity = [0, -1e-5, 0]
mobility = 0.02
interfaceWidth = 4
muRatio = 10
rhoRatio = 10
geometry = [
  {
    type = "circle"
    center = [8, 8, 0]
    radius = 3
    id = 0
  }
]
boundary = [
%s
]
"""


def _sides(**types):
    out = []
    for side in ("x-", "x+", "y-", "y+"):
        t = types.get(side.replace("-", "m").replace("+", "p"), "periodic")
        if t is None:
            continue
        out.append('  {\n    side = "%s"\n    type = "%s"\n  },' % (side, t))
    return "\n".join(out)


@pytest.mark.parametrize("sides,msg", [
    (dict(yp=None), "Missing boundary conditions for sides: y+"),
    (dict(xm="do nothing", xp="wall", ym="wall", yp="wall"), "supported boundaries are"),
    (dict(xm="neumann", xp="wall", ym="neumann", yp="wall"), "two adjacent"),
    (dict(xm="slip wall", xp="neumann"), "a slip wall needs a wall side"),
    (dict(xm="wall", xp="periodic"), "periodic on both sides"),
])
def test_config_errors(tmp_path, sides, msg):
    path = _write(tmp_path, BASE % _sides(**sides))
    with pytest.raises(cb.ClipError) as e:
        cb.config_summary(path)
    assert e.value.code == -1
    assert msg in str(e.value)


def test_config_unknown_case_and_jet(tmp_path):
    with pytest.raises(cb.ClipError, match="Unknown case type: pool"):
        cb.config_summary(_write(tmp_path, (BASE % _sides()).replace("case = drop", "case = pool")))
    # case 'jet' derives sigma and mu_H from the reference velocity (InputData.cu:99-107)
    text = (BASE % _sides()).replace("case = drop", "case = Jet\nreferenceVelocity = 0.02")
    p = cb.config_summary(_write(tmp_path, text))["params"]
    assert p["caseType"] == 3
    o = O.Oracle(_write(tmp_path, text)).params()
    assert p["sigma"] == o["sigma"] and p["muH"] == o["muH"]


def test_config_missing_file():
    with pytest.raises(cb.ClipError, match="cannot open config file"):
        cb.config_summary("/nonexistent/config.txt")


def test_parse_quirks_follow_reference(tmp_path):
    """Scalar keys take the first match anywhere (InputData.cu:294-317); RTI derives the
    mobility from Pe and overwrites the config value (InputData.cu:95-97)."""
    text = (BASE % _sides(ym="wall", yp="wall")).replace("case = drop", "case = RTI\nPe = 50\nCa = 0.2")
    text = text.replace("mobility = 0.02", "mobility = 0.02\nmobility = 0.7")
    s = cb.config_summary(_write(tmp_path, text))
    L, g = 8.0, 1e-5
    assert s["params"]["mobility"] == (np.sqrt(g * L) * L) / 50.0
    assert s["sides"][:4] == [3, 3, 0, 0]


def test_three_d_extent_includes_ghosts(tmp_path):
    text = (BASE % _sides()).replace("N = [16, 16, 1]", "N = [10, 12, 8]")
    text = text.replace('  },\n]\n', '  },\n  {\n    side = "z-"\n    type = "wall"\n  },\n  {\n    side = "z+"\n    type = "wall"\n  },\n]\n')
    s = cb.config_summary(_write(tmp_path, text))
    assert s["dim"] == 3 and s["extent"] == (10, 12, 8)
