"""The C++ host driver clipb_run (the reference's main loop, src/main.cu:39-92, over the C
ABI) run as a subprocess: its printed sum(c) against the CPU oracle, checkpoint folders
rotated as CheckPointer::rotateFolders does, and -resume continuing bit for bit."""
import os
import re
import subprocess

import pytest

from conftest import REPO, golden_config
import oracle as O

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(REPO, "clip_b200", "clipb_run")
LINE = re.compile(r"^step (\d+)  sum\(c\) (\S+)  kinetic (\S+)$", re.M)


def _config(tmp_path, name, **keys):
    text = open(golden_config(name)).read()
    for k, v in keys.items():
        text, n = re.subn(rf"^{k} = .*$", f"{k} = {v}", text, flags=re.M)
        assert n == 1, k
    path = tmp_path / "config.txt"
    path.write_text(text)
    return str(path)


def _run(args, cwd):
    res = subprocess.run([DRIVER] + args, cwd=cwd, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout + res.stderr
    return {int(m.group(1)): (m.group(2), m.group(3)) for m in LINE.finditer(res.stdout)}, res.stdout


def test_driver_monitors_match_the_oracle(tmp_path):
    cfg = _config(tmp_path, "drop2d_small", finalStep=30, reportInterval=10)
    got, _ = _run([cfg], tmp_path)
    assert sorted(got) == [10, 20, 30]
    o = O.Oracle(golden_config("drop2d_small"))
    o.init()
    for step in (10, 20, 30):
        o.solve(10)
        mass = float(got[step][0])
        assert abs(mass - o.mass()) <= 1e-12 * abs(mass), step


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_driver_checkpoints_and_resume(tmp_path, precision):
    cfg = _config(tmp_path, "drop3d_small", finalStep=30, reportInterval=5, checkpointInterval=10,
                  checkpointCopy=2)
    full, out = _run([cfg, "--precision", precision], tmp_path)
    assert "checkpoint of step 30 saved" in out
    # CheckPointer::rotateFolders: the newest in Checkpoint, older ones in Checkpoint_1, _2
    for d, step in (("Checkpoint", 30), ("Checkpoint_1", 20), ("Checkpoint_2", 10)):
        info = (tmp_path / d / "info.txt").read_text()
        assert f"CurrentStep: {step}" in info, (d, info)
        assert (tmp_path / d / "dev_f.bin").exists() and (tmp_path / d / "clipb_state.bin").exists()
    resumed, out = _run([cfg, "--precision", precision, "-resume", "--checkpoint-dir", "Checkpoint_1"], tmp_path)
    assert "resumed from Checkpoint_1 at step 20" in out
    assert sorted(resumed) == [25, 30]
    for step in (25, 30):
        assert resumed[step] == full[step], step  # printed to 17 digits: bit for bit
