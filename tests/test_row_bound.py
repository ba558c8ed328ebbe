"""The row bound that lets clipb_init skip saturated rows of the initial field
(row_distance_sign in clip_b200/csrc/config.hpp), checked on the host: compiled with the
library's own config reader, run over every workload and golden config.  Every row it
reports must hold, node by node, the value the per-node evaluation gives."""
import glob
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(REPO, "clip_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_reported_rows_hold_the_saturated_value(tmp_path):
    exe = str(tmp_path / "row_bound_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, "-I", os.path.join(REPO, "include"),
                    os.path.join(HERE, "native", "row_bound_check.cpp"), os.path.join(CSRC, "config.cpp"), "-o", exe],
                   check=True)
    configs = sorted(glob.glob(os.path.join(REPO, "clip_b200", "workloads", "*.txt")) +
                     glob.glob(os.path.join(HERE, "golden", "configs", "*.txt")))
    res = subprocess.run([exe] + configs, capture_output=True, text=True)
    assert res.returncode == 0, res.stdout + res.stderr
    lines = res.stdout.strip().splitlines()
    assert len(lines) == len(configs)
    reported = {os.path.basename(l.split()[0]): int(l.split()[4]) for l in lines}
    # the benchmark bubble: most rows lie where the profile is saturated
    assert reported["bubble3d_256x512x256.txt"] > 100000
