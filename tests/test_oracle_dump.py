"""The reference executable's two read-out forms agree: `oracle_dump FILE
compute` (text, every double printed with 17 digits) and `oracle_dump FILE
compute binary` (raw float64, for systems of millions of sites) give the same
values through oracle.read_dump and oracle.read_dump_binary, on the small EAM
fixture system (runs on the CPU)."""
import os
import sys

import numpy as np

from cac_b200 import gen
from helpers import CASES

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

DECK = """units metal
dimension 3
boundary p p p
atom_style atomic
element_style cac 8 1 wscale 1 1 1 1
read_data data.cac
pair_style eam/alloy
pair_coeff * * cu.setfl Cu
neighbor 1.0 bin
neigh_modify every 10 delay 0 check no
timestep 0.001
fix 1 all nve
run 0
oracle_dump setup.txt compute
oracle_dump setup.bin compute binary
run 5
oracle_dump end.txt state
oracle_dump end.bin state binary
"""


def test_binary_dump_equals_text_dump(tmp_path):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    assert os.path.exists(O.REF_EXE_EAMFIX), "build the reference: make -C oracle reference"
    build, pair, _ = CASES["tiny_eam"]
    gen.write_data(build(), str(tmp_path / "data.cac"))
    gen.write_setfl(gen.EamParams(), str(tmp_path / "cu.setfl"))
    (tmp_path / "in.cac").write_text(DECK)
    O.run_reference(str(tmp_path), "in.cac", exe=O.REF_EXE_EAMFIX, timeout=600)
    for name in ("setup", "end"):
        a = O.read_dump(str(tmp_path / f"{name}.txt"))
        b = O.read_dump_binary(str(tmp_path / f"{name}.bin"))
        assert a["natoms"] > 0 and a["nelements"] > 0
        for k, v in a.items():
            if isinstance(v, np.ndarray):
                assert np.array_equal(v, b[k]), (name, k)
            else:
                assert v == b[k], (name, k)
