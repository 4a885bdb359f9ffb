"""The package's fix styles inside the reference's own loop, on the host: with
the reference's CPU pair style, fix langevin/b200 and fix deform/b200 must
behave exactly as the reference's fix langevin and fix deform (they only add
what run_b200 reads).  Runs the harness executable oracle/_ref/cac_b200
(``make -C oracle app``) and the reference executable; no GPU is used."""
import os
import subprocess

import numpy as np
import pytest

from cac_b200 import gen
from helpers import CASES

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
APP = os.path.join(ROOT, "oracle", "_ref", "cac_b200")

HEADER = """units metal
dimension 3
boundary p p p
atom_style atomic
element_style cac 8 1 wscale 1 1 1 1
read_data data.cac
pair_style lj/cut 5.5
pair_coeff 1 1 0.4093 2.338
neighbor 1.0 bin
neigh_modify every 10 delay 0 check no
timestep 0.001
fix 1 all nve
"""


def run(exe, tmp_path, body):
    (tmp_path / "in.cac").write_text(HEADER + body + "run 12\nrun 7\noracle_dump end.txt state\n")
    r = subprocess.run([exe, "-in", "in.cac"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    return (tmp_path / "end.txt").read_text()


@pytest.mark.parametrize("fix", [
    "fix 2 all langevin{s} 40.0 90.0 0.05 1234 zero yes\n",
    "fix 3 all deform{s} 1 x erate 0.5 y volume z wiggle 0.2 0.01 units box remap x\n",
])
def test_fix_styles_equal_reference_fixes_in_reference_loop(fix, oracle_mod, tmp_path):
    if not os.path.exists(APP):
        pytest.skip("harness executable not built (make -C oracle app)")
    if not os.path.exists(oracle_mod.REF_EXE):
        pytest.skip("reference executable not built (make -C oracle reference)")
    gen.write_data(CASES["tiny_lj"][0](), str(tmp_path / "data.cac"))
    ours = run(APP, tmp_path, fix.format(s="/b200"))
    ref = run(oracle_mod.REF_EXE, tmp_path, fix.format(s=""))
    assert ours == ref


def test_min_style_fire_b200_registered_and_needs_a_b200_pair(tmp_path):
    """min_style fire/b200 is a min style of the harness executable (the
    reference has no FIRE style); with a CPU pair style its setup stops with
    the style's own message, before any device is touched."""
    if not os.path.exists(APP):
        pytest.skip("harness executable not built (make -C oracle app)")
    gen.write_data(CASES["tiny_lj"][0](), str(tmp_path / "data.cac"))
    (tmp_path / "in.cac").write_text(HEADER.replace("fix 1 all nve\n", "") +
                                     "min_style fire/b200\nminimize 0.0 1e-6 10 100\n")
    r = subprocess.run([APP, "-in", "in.cac"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    out = r.stdout + r.stderr
    assert r.returncode != 0
    assert "min_style fire/b200 needs pair style lj/cut/b200 or eam/alloy/b200" in out
    (tmp_path / "in2.cac").write_text(HEADER + "min_style fire\n")
    r = subprocess.run([APP, "-in", "in2.cac"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode != 0 and "Illegal min_style command" in r.stdout + r.stderr
