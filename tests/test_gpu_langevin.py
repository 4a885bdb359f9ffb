"""fix langevin on the device (cacb200_set_langevin) against the reference.

The device draws the reference's own RanMars stream, so its forces and
trajectories follow the reference's: the setup forces (pair forces plus the
first draws) within 1e-12 relative; the state after consecutive runs within
1e-10 (the FP64 trajectory bar of the force path).  Graph replay equals eager
stepping bit for bit, and each replica of a batch equals the same system run
alone with seed + r bit for bit."""
import numpy as np
import pytest

from cac_b200 import gen
from helpers import CASES, LJ, SKIN, rel_err, setfl_path

pytestmark = pytest.mark.gpu

TOL_SETUP = 1e-12
TOL_TRAJ = 1e-10


def make_engine(system, pair, tmp_path, graphs=True):
    from cac_b200.api import Engine
    e = Engine(0)
    e.upload(system)
    if pair == "lj":
        e.pair_lj(*LJ)
    else:
        e.pair_eam(setfl_path(tmp_path))
    e.neighbor(SKIN, 10)
    e.graphs(graphs)
    return e


def lgv_args(g):
    t0, t1, damp, seed, zero = g["lgv_params"]
    return float(t0), float(t1), float(damp), int(seed), bool(zero)


@pytest.mark.parametrize("case", ["tiny_lj", "tiny_eam", "lj_small"])
def test_langevin_setup_forces_vs_reference(case, golden, tmp_path):
    g = golden(case)
    build, pair, _ = CASES[case]
    e = make_engine(build(), pair, tmp_path)
    e.langevin(*lgv_args(g))
    e.run_nve(0)
    f, nf, _ = e.forces()
    assert rel_err(f, g["lgv_setup_f"]) < TOL_SETUP
    assert rel_err(nf, g["lgv_setup_nodef"]) < TOL_SETUP
    e.close()


@pytest.mark.parametrize("case", ["tiny_lj", "tiny_eam", "lj_small"])
def test_langevin_trajectory_vs_reference(case, golden, tmp_path):
    g = golden(case)
    build, pair, _ = CASES[case]
    e = make_engine(build(), pair, tmp_path)
    e.langevin(*lgv_args(g))
    for n in g["lgv_runs"]:
        e.run_nve(int(n))
    x, v, nx, nv = e.state()
    f, nf, _ = e.forces()
    e.close()
    assert np.abs(x - g["lgv_end_x"]).max() < TOL_TRAJ
    assert np.abs(nx - g["lgv_end_nodex"]).max() < TOL_TRAJ
    assert rel_err(v, g["lgv_end_v"]) < TOL_TRAJ
    assert rel_err(nv, g["lgv_end_nodev"]) < TOL_TRAJ
    assert rel_err(f, g["lgv_end_f"]) < TOL_TRAJ
    assert rel_err(nf, g["lgv_end_nodef"]) < TOL_TRAJ


def test_langevin_graphs_equal_eager(tmp_path):
    s = gen.replica(3000, 60, temperature=200.0, strain=0.01, seed=51)
    out = []
    for graphs in (True, False):
        e = make_engine(s, "eam", tmp_path, graphs=graphs)
        e.langevin(300.0, 100.0, 0.1, 777, zero=True)
        e.run_nve(25)
        e.run_nve(12)
        out.append(e.state() + e.forces()[:2])
        if graphs:
            assert e.graph_launches() > 0
        e.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("zero", [False, True])
def test_langevin_batch_equals_alone(zero, tmp_path):
    from cac_b200.api import Engine
    systems = [
        gen.replica(2000, 50, temperature=120.0, strain=0.0, seed=61),
        gen.replica(4000, 90, temperature=400.0, strain=0.03, seed=62),
        gen.replica(1500, 20, temperature=60.0, strain=0.01, seed=63),
    ]
    seed = 4242
    b = Engine(0)
    b.upload_batch(systems)
    b.pair_lj(*LJ)
    b.neighbor(SKIN, 10)
    b.langevin(100.0, 250.0, 0.08, seed, zero=zero)
    b.run_nve(14)
    xb, vb, nxb, nvb = b.state()
    b.close()
    a0 = e0 = 0
    for r, s in enumerate(systems):
        e = make_engine(s, "lj", tmp_path)
        e.langevin(100.0, 250.0, 0.08, seed + r, zero=zero)
        e.run_nve(14)
        x, v, nx, nv = e.state()
        e.close()
        na, ne = x.shape[0], nx.shape[0]
        assert np.array_equal(x, xb[a0:a0 + na]), r
        assert np.array_equal(v, vb[a0:a0 + na]), r
        assert np.array_equal(nx, nxb[e0:e0 + ne]), r
        assert np.array_equal(nv, nvb[e0:e0 + ne]), r
        a0 += na
        e0 += ne


def test_langevin_arguments_and_unset(tmp_path):
    """The reference's argument checks; unset returns to plain NVE."""
    from cac_b200.api import CacB200Error
    s = CASES["tiny_lj"][0]()
    e = make_engine(s, "lj", tmp_path)
    for bad in ((10.0, 10.0, 0.0, 5), (10.0, 10.0, 0.1, 0), (10.0, 10.0, 0.1, 900000001)):
        with pytest.raises(CacB200Error):
            e.langevin(*bad)
    e.run_nve(5)
    ref = e.state()
    e.close()
    e = make_engine(s, "lj", tmp_path)
    e.langevin(50.0, 50.0, 0.1, 99)
    e.unset_langevin()
    e.run_nve(5)
    for a, b in zip(ref, e.state()):
        assert np.array_equal(a, b)
    e.close()
