"""fix deform on the device (cacb200_set_deform) against the reference.

The box after consecutive runs equals the reference's bit for bit (the same
host arithmetic); atoms, nodes, velocities and forces within 1e-10 (the FP64
trajectory bar).  Each replica of a batch deforms like the same system alone,
bit for bit.  The mixed form follows the FP64 trajectory within its force
accuracy, and the thermo volume follows the box."""
import numpy as np
import pytest

from cac_b200 import gen
from helpers import CASES, LJ, SKIN, rel_err, setfl_path

pytestmark = pytest.mark.gpu

TOL_TRAJ = 1e-10
STYLES = ("none", "final", "delta", "scale", "vel", "erate", "trate", "wiggle", "volume")


def make_engine(system, pair, tmp_path, form=0):
    from cac_b200.api import Engine
    e = Engine(0)
    e.upload(system)
    if pair == "lj":
        e.pair_lj(*LJ)
    else:
        e.pair_eam(setfl_path(tmp_path))
    e.neighbor(SKIN, 10)
    e.set_precision(form)
    return e


def apply_deform(e, g):
    dims = {}
    for d, name in enumerate("xyz"):
        dims[name] = (STYLES[int(g["dfm_style"][d])], float(g["dfm_a"][d]), float(g["dfm_b"][d]))
    e.deform(int(g["dfm_nevery"]), **dims)


@pytest.mark.parametrize("case", ["tiny_lj", "tiny_eam", "lj_small"])
def test_deform_trajectory_vs_reference(case, golden, tmp_path):
    g = golden(case)
    build, pair, _ = CASES[case]
    e = make_engine(build(), pair, tmp_path)
    apply_deform(e, g)
    for n in g["dfm_runs"]:
        e.run_nve(int(n))
    lo, hi = e.box()
    x, v, nx, nv = e.state()
    f, nf, _ = e.forces()
    t = e.thermo()
    e.close()
    box = g["dfm_end_box"]
    assert list(lo) == [box[0], box[2], box[4]]
    assert list(hi) == [box[1], box[3], box[5]]
    assert t["vol"] == (box[1] - box[0]) * (box[3] - box[2]) * (box[5] - box[4])
    assert np.abs(x - g["dfm_end_x"]).max() < TOL_TRAJ
    assert np.abs(nx - g["dfm_end_nodex"]).max() < TOL_TRAJ
    assert rel_err(v, g["dfm_end_v"]) < TOL_TRAJ
    assert rel_err(nv, g["dfm_end_nodev"]) < TOL_TRAJ
    assert rel_err(f, g["dfm_end_f"]) < TOL_TRAJ
    assert rel_err(nf, g["dfm_end_nodef"]) < TOL_TRAJ


def test_deform_batch_equals_alone(tmp_path):
    from cac_b200.api import Engine
    systems = [
        gen.replica(2000, 50, temperature=120.0, strain=0.0, seed=71),
        gen.replica(4000, 90, temperature=300.0, strain=0.02, seed=72),
    ]
    spec = dict(x=("erate", 0.8), y=("volume",), z=("wiggle", 0.2, 0.015))
    b = Engine(0)
    b.upload_batch(systems)
    b.pair_eam(setfl_path(tmp_path))
    b.neighbor(SKIN, 10)
    b.deform(1, **spec)
    b.run_nve(23)
    xb, vb, nxb, nvb = b.state()
    b.close()
    a0 = e0 = 0
    for r, s in enumerate(systems):
        e = make_engine(s, "eam", tmp_path)
        e.deform(1, **spec)
        e.run_nve(23)
        x, v, nx, nv = e.state()
        e.close()
        na, ne = x.shape[0], nx.shape[0]
        assert np.array_equal(x, xb[a0:a0 + na]), r
        assert np.array_equal(v, vb[a0:a0 + na]), r
        assert np.array_equal(nx, nxb[e0:e0 + ne]), r
        assert np.array_equal(nv, nvb[e0:e0 + ne]), r
        a0 += na
        e0 += ne


def test_deform_mixed_form_follows_fp64(tmp_path):
    s = gen.replica(3000, 60, temperature=150.0, strain=0.0, seed=73)
    out = []
    for form in (0, 1):
        e = make_engine(s, "eam", tmp_path, form=form)
        e.deform(1, x=("erate", 1.0), z=("scale", 1.01))
        e.run_nve(15)
        out.append((e.state(), e.box()))
        e.close()
    (x0, _, nx0, _), box0 = out[0]
    (x1, _, nx1, _), box1 = out[1]
    assert np.array_equal(box0[0], box1[0]) and np.array_equal(box0[1], box1[1])
    assert np.abs(x1 - x0).max() < 1e-5
    assert np.abs(nx1 - nx0).max() < 1e-5


def test_deform_arguments_and_unset(tmp_path):
    from cac_b200.api import CacB200Error
    s = CASES["tiny_lj"][0]()
    e = make_engine(s, "lj", tmp_path)
    with pytest.raises(CacB200Error):
        e.deform(0, x=("erate", 0.1))
    with pytest.raises(CacB200Error):
        e.deform(1, x=("volume",))
    with pytest.raises(CacB200Error):
        e.deform(1, x=("wiggle", 0.1, 0.0))
    lo0, hi0 = e.box()
    e.deform(1, x=("erate", 0.5))
    e.unset_deform()
    e.run_nve(5)
    lo, hi = e.box()
    assert np.array_equal(lo, lo0) and np.array_equal(hi, hi0)
    e.close()


def test_run_starts_from_forces_of_current_positions(tmp_path):
    """Like Verlet::setup, a run starts from the forces of the positions it
    is given: new positions through set_state are evaluated first, positions
    written back unchanged keep their forces (the same values either way)."""
    s = CASES["tiny_lj"][0]()
    e = make_engine(s, "lj", tmp_path)
    e.setup()
    x, v, nx, nv = e.state()
    e.set_state(x, v, nx, nv)          # unchanged
    f0, nf0, _ = e.forces()
    x2 = x.copy()
    x2[0, 0] += 0.01
    e.set_state(x2, v, nx, nv)
    e.run_nve(0)
    f1, _, _ = e.forces()
    e.close()
    r = make_engine(s, "lj", tmp_path)
    r.set_state(x2, v, nx, nv)
    r.setup()
    fr, _, _ = r.forces()
    r.close()
    assert not np.array_equal(f0, f1)
    assert rel_err(f1, fr) < 1e-13   # lists built from other positions: summation order may differ


def test_set_box_matches_fresh_upload(tmp_path):
    """A new box through cacb200_set_box (lists kept) gives the forces of the
    same positions uploaded in that box (lists built for it)."""
    from cac_b200.api import ENERGY_GLOBAL, VIRIAL_GLOBAL
    s = CASES["tiny_lj"][0]()
    lo = np.asarray(s.boxlo, dtype=np.float64)
    hi = np.asarray(s.boxhi, dtype=np.float64) + np.array([0.03, -0.02, 0.01])
    e = make_engine(s, "lj", tmp_path)
    e.setup()
    e.set_box(lo, hi)
    e.compute(ENERGY_GLOBAL, VIRIAL_GLOBAL)
    f1, nf1, _ = e.forces()
    ev1 = e.energy(peratom=False)
    e.close()
    s2 = CASES["tiny_lj"][0]()
    s2.boxhi = hi
    r = make_engine(s2, "lj", tmp_path)
    r.compute(ENERGY_GLOBAL, VIRIAL_GLOBAL)
    f2, nf2, _ = r.forces()
    ev2 = r.energy(peratom=False)
    r.close()
    assert rel_err(f1, f2) < 1e-13
    assert rel_err(nf1, nf2) < 1e-13
    assert abs(ev1["energy"] - ev2["energy"]) < 1e-12 * abs(ev2["energy"])


@pytest.mark.parametrize("case", ["tiny_lj", "tiny_eam", "lj_small"])
def test_langevin_and_deform_together_vs_reference(case, golden, tmp_path):
    """fix langevin (after the forces) and fix deform (at the end of the step)
    together, over the langevin case's runs: the reference's box bit for bit,
    its state within 1e-10."""
    g = golden(case)
    build, pair, _ = CASES[case]
    e = make_engine(build(), pair, tmp_path)
    t0, t1, damp, seed, zero = (float(v) for v in g["lgv_params"])
    e.langevin(t0, t1, damp, int(seed), bool(zero))
    apply_deform(e, g)
    for n in g["lgv_runs"]:
        e.run_nve(int(n))
    lo, hi = e.box()
    x, v, nx, nv = e.state()
    f, nf, _ = e.forces()
    e.close()
    box = g["both_end_box"]
    assert list(lo) == [box[0], box[2], box[4]] and list(hi) == [box[1], box[3], box[5]]
    assert np.abs(x - g["both_end_x"]).max() < TOL_TRAJ
    assert np.abs(nx - g["both_end_nodex"]).max() < TOL_TRAJ
    assert rel_err(v, g["both_end_v"]) < TOL_TRAJ
    assert rel_err(nv, g["both_end_nodev"]) < TOL_TRAJ
    assert rel_err(f, g["both_end_f"]) < TOL_TRAJ
    assert rel_err(nf, g["both_end_nodef"]) < TOL_TRAJ
