"""The CUDA path against the reference executable at the workloads' own scale.

The small fixtures of tests/golden pin the path on 1.5 k - 6 k sites; here the
reference executable (``oracle/_ref/cac_eamfix``: the reference compiled from
its sources, EAM energies read on the F(rho) row) runs on the same host as the
GPU, on the same seeded inputs, for

* the EAM workload at scale (1,049,760 atoms + 20,000 elements, 1,209,760
  sites, 300 K) and the 3 %-strained mixed-precision workload's system
  (4,179,600 atoms + 100,000 elements, 4,979,600 sites) in FP64: setup
  forces (atoms, nodes, Gauss points), energy, virial and per-site energy
  and virial after one evaluation (``Verlet::setup``, verlet.cpp:64-152);
* a 3 %-strained slab of 313,120 sites (272,160 atoms + 5,120 elements, the
  strained shape of the mixed-precision workload at a quarter of its height):
  half and full neighbour lists as sorted index sets, bit for bit
  (``npair_half_bin_newton.cpp:25-392``, ``npair_full_bin.cpp:23-358``),
  setup forces, energy and virial, and the state after 20 velocity-Verlet
  steps with a rebuild at step 10 (``verlet.cpp:218-360``, ``fix_nve.cpp:62-219``).

Tolerances are those of the small cases: lists equal; FP64 forces, energies,
virials and states within 1e-10 relative (max per-site norm of the difference
over the largest per-site norm).
"""
import os

import numpy as np
import pytest

from cac_b200 import gen
from helpers import N2G, SKIN, counts, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-10
NSTEPS = 20

HEADER = """units metal
dimension 3
boundary p p p
atom_style atomic
element_style cac 8 1 wscale 1 1 1 1
read_data data.cac
"""
TAIL = "neighbor 1.0 bin\nneigh_modify every 10 delay 0 check no\ntimestep 0.001\nfix 1 all nve\n"
EAM = "pair_style eam/alloy\npair_coeff * * cu.setfl Cu\n"
# the reference's full list (NPairFullBin) exposed through a pair style that requests it
FULL = "pair_style lj/cut/fulllist 5.0\npair_coeff 1 1 0.4093 2.338\n"


def strained_slab():
    return gen.build_slab(8, 5, 32, 42, temperature=300.0, strain=0.03, seed=9)


def reference(work, system, body, pair=EAM):
    import oracle as O
    if not os.path.exists(os.path.join(work, "data.cac")):
        gen.write_data(system, os.path.join(work, "data.cac"))
        gen.write_setfl(gen.EamParams(), os.path.join(work, "cu.setfl"))
    with open(os.path.join(work, "in.cac"), "w") as f:
        f.write(HEADER + pair + TAIL + body)
    if not os.path.exists(O.REF_EXE_EAMFIX):
        pytest.fail("oracle/_ref/cac_eamfix is missing: build it with make -C oracle reference")
    O.run_reference(work, "in.cac", exe=O.REF_EXE_EAMFIX, timeout=1800.0)
    return O


def engine(system, work):
    from cac_b200.api import Engine
    e = Engine(0)
    e.upload(system)
    e.pair_eam(os.path.join(work, "cu.setfl"))
    e.neighbor(SKIN, 10)
    return e


def check_setup(e, d):
    e.compute()
    f, nf, gf = e.forces()
    ev = e.energy()
    assert rel_err(f, d["f"]) < TOL
    assert rel_err(nf, d["nodef"]) < TOL
    assert rel_err(gf[:, N2G, :], d["gaussf_at_node"]) < TOL
    assert abs(ev["energy"] - d["energy"]) / abs(d["energy"]) < TOL
    assert np.abs(ev["virial"] - d["virial"]).max() / np.abs(d["virial"]).max() < TOL
    escale = np.abs(d["eatom"]).max()
    assert np.abs(ev["eatom"] - d["eatom"]).max() / escale < TOL
    assert np.abs(ev["enode"] - d["enode"]).max() / escale < TOL
    vscale = np.abs(d["vatom"]).max()
    assert np.abs(ev["vatom"] - d["vatom"]).max() / vscale < TOL
    assert np.abs(ev["vnode"] - d["vnode"]).max() / vscale < TOL


def test_eam_1m_setup_vs_reference(tmp_path):
    """1,209,760 sites: one evaluation, every read-out of the reference."""
    s = gen.eam_1m()
    work = str(tmp_path)
    O = reference(work, s, "run 0\noracle_dump setup.txt compute\n")
    d = O.read_dump(os.path.join(work, "setup.txt"))
    assert d["natoms"] == s.natoms and d["nelements"] == s.nelements
    e = engine(s, work)
    check_setup(e, d)
    e.close()


def test_eam_4m_strained_setup_vs_reference(tmp_path):
    """4,979,600 sites (4,179,600 atoms + 100,000 elements, 3 % strain: the
    mixed-precision workload's own system): one evaluation, every read-out of
    the reference (its dump in binary form) in FP64, and the mixed form's
    forces, energy and virial against the same reference read-out."""
    s = gen.eam_4m_strained()
    work = str(tmp_path)
    O = reference(work, s, "run 0\noracle_dump setup.bin compute binary\n")
    d = O.read_dump_binary(os.path.join(work, "setup.bin"))
    os.remove(os.path.join(work, "data.cac"))
    assert d["natoms"] == s.natoms and d["nelements"] == s.nelements
    assert s.natoms + 8 * s.nelements == 4979600
    e = engine(s, work)
    check_setup(e, d)
    e.close()
    # the mixed form against the same reference read-out: largest per-site
    # force error under 1e-5 of the largest force, energy and virial to 1e-6
    from cac_b200.api import MIXED
    e = engine(s, work)
    e.set_precision(MIXED)
    e.compute()
    f, nf, _ = e.forces()
    ev = e.energy(peratom=False)
    e.close()
    assert rel_err(f, d["f"]) < 1e-5
    assert rel_err(nf, d["nodef"]) < 1e-5
    assert abs(ev["energy"] - d["energy"]) / abs(d["energy"]) < 1e-6
    assert np.abs(ev["virial"] - d["virial"]).max() / np.abs(d["virial"]).max() < 1e-6


@pytest.fixture(scope="module")
def strained(tmp_path_factory):
    """The reference's read-outs of the strained slab, run once for the tests below."""
    s = strained_slab()
    work = str(tmp_path_factory.mktemp("strained"))
    O = reference(work, s, "run 0\noracle_dump setup.txt compute\noracle_dump_neigh half.bin binary\n")
    out = {"setup": O.read_dump(os.path.join(work, "setup.txt")),
           "half": O.read_neigh_binary(os.path.join(work, "half.bin"))}
    os.remove(os.path.join(work, "half.bin"))
    reference(work, s, "run 0\noracle_dump_neigh full.bin binary\n", pair=FULL)
    out["full"] = O.read_neigh_binary(os.path.join(work, "full.bin"))
    os.remove(os.path.join(work, "full.bin"))
    reference(work, s, f"run {NSTEPS}\noracle_dump end.txt state\n")
    out["end"] = O.read_dump(os.path.join(work, "end.txt"))
    return s, work, out


def test_strained_lists_bit_exact_vs_reference(strained):
    s, work, ref = strained
    assert s.natoms + 8 * s.nelements == 313120
    e = engine(s, work)
    nsites = s.natoms + 8 * s.nelements
    # the full list of the step loop's build (no half list), then both
    e.build_lists(half=False)
    rows = e.neighbor_list(False)
    assert np.array_equal(rows, ref["full"])
    del rows
    e.build_lists(half=True)
    for half, key in ((True, "half"), (False, "full")):
        rows = e.neighbor_list(half)
        assert np.array_equal(counts(rows, nsites), counts(ref[key], nsites)), key
        assert np.array_equal(rows, ref[key]), key
    e.close()


def test_strained_setup_vs_reference(strained):
    s, work, ref = strained
    e = engine(s, work)
    check_setup(e, ref["setup"])
    e.close()


def test_strained_trajectory_vs_reference(strained):
    """20 velocity-Verlet steps, lists rebuilt at step 10."""
    s, work, ref = strained
    g = ref["end"]
    e = engine(s, work)
    e.setup()
    e.run_nve(NSTEPS, 0.001)
    x, v, nx, nv = e.state()
    f, nf, _ = e.forces()
    assert np.abs(x - g["x"]).max() < 1e-10
    assert np.abs(nx - g["nodex"]).max() < 1e-10
    assert rel_err(v, g["v"]) < TOL
    assert rel_err(nv, g["nodev"]) < TOL
    assert rel_err(f, g["f"]) < TOL
    assert rel_err(nf, g["nodef"]) < TOL
    e.close()
