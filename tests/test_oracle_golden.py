"""The CPU restatement in oracle/ against the reference's own read-outs
(golden fixtures made by tests/golden/make_golden.py)."""
import numpy as np
import pytest

from helpers import CASES, G2N, LJ, N2G, SKIN, counts, digest, rel_err, setfl_path


@pytest.mark.parametrize("case", ["tiny_lj", "tiny_eam", "lj_small"])
def test_lists_match_reference(case, oracle_mod, golden):
    g = golden(case)
    build, pair, cutneigh = CASES[case]
    s = build()
    st = oracle_mod.OracleState(s)
    nsites = s.natoms + 8 * s.nelements
    for half, key in ((True, "half"), (False, "full")):
        L = oracle_mod.build_list(st, cutneigh, half)
        rows = L.canonical(s.natoms)
        oracle_mod.free_list(L)
        assert np.array_equal(counts(rows, nsites), g[key + "_counts"])
        assert digest(rows) == str(g[key + "_digest"])


@pytest.mark.parametrize("case", ["tiny_lj", "tiny_eam", "lj_small"])
def test_forces_energy_match_reference(case, oracle_mod, golden, tmp_path):
    g = golden(case)
    build, pair, cutneigh = CASES[case]
    s = build()
    st = oracle_mod.OracleState(s)
    L = oracle_mod.build_list(st, cutneigh, True)
    if pair == "lj":
        ev = oracle_mod.lj_forces(st, L, *LJ)
    else:
        ev = oracle_mod.eam_forces(st, L, oracle_mod.Eam(setfl_path(tmp_path)))
    oracle_mod.free_list(L)
    fscale = max(np.abs(g["f"]).max(), np.abs(g["nodef"]).max())
    assert np.abs(st.f - g["f"]).max() / fscale < 1e-12
    assert np.abs(st.nodef - g["nodef"]).max() / fscale < 1e-12
    assert np.abs(st.gaussf[:, N2G, :] - g["gaussf_at_node"]).max() / fscale < 1e-12
    assert abs(ev.energy - float(g["energy"])) / abs(float(g["energy"])) < 1e-12
    assert np.abs(ev.virial - g["virial"]).max() / np.abs(g["virial"]).max() < 1e-12
    assert np.abs(ev.eatom - g["eatom"]).max() < 1e-11
    assert np.abs(ev.enode - g["enode"]).max() < 1e-11
    if "vatom" in g:
        assert np.abs(ev.vatom - g["vatom"]).max() < 1e-11
        assert np.abs(ev.vnode - g["vnode"]).max() < 1e-11


def test_eam_reference_energy_quirk_is_real(golden):
    """The unpatched reference reads the embedding energy from a stale spline
    row (pair_eam.cpp:819-833 with compute_fp's coefficient pointer passed by
    value); the fixture records both values and they differ grossly."""
    g = golden("tiny_eam")
    assert abs(float(g["energy_unpatched"]) - float(g["energy"])) > 1.0


@pytest.mark.parametrize("case", ["tiny_lj", "tiny_eam", "lj_small"])
def test_trajectory_matches_reference(case, oracle_mod, golden, tmp_path):
    g = golden(case)
    build, pair, cutneigh = CASES[case]
    s = build()
    st = oracle_mod.OracleState(s)
    n = int(g["nsteps"])
    if pair == "lj":
        oracle_mod.run_nve(st, "lj", lj=LJ, skin=SKIN, nsteps=n, every=10)
    else:
        oracle_mod.run_nve(st, "eam", eam=oracle_mod.Eam(setfl_path(tmp_path)), skin=SKIN, nsteps=n, every=10)
    assert np.abs(st.x - g["end_x"]).max() < 1e-10
    assert np.abs(st.nodex - g["end_nodex"]).max() < 1e-10
    assert rel_err(st.f, g["end_f"]) < 1e-10
    assert rel_err(st.nodef, g["end_nodef"]) < 1e-10
    assert rel_err(st.v, g["end_v"]) < 1e-10
    assert rel_err(st.nodev, g["end_nodev"]) < 1e-10


def thermo_err(got: dict, ref_row, fields) -> float:
    """Largest error over thermo fields: energies and temperature relative to
    their own size, pressures relative to the largest pressure component."""
    ref = dict(zip(fields, ref_row))
    pk = ("press", "pxx", "pyy", "pzz", "pxy", "pxz", "pyz")
    pscale = max(abs(ref[k]) for k in pk if k in ref) if any(k in ref for k in pk) else 1.0
    err = 0.0
    for k, r in ref.items():
        scale = pscale if k in pk else abs(r)
        err = max(err, abs(got[k] - r) / scale)
    return err


@pytest.mark.parametrize("case", ["tiny_lj", "tiny_eam", "lj_small"])
def test_thermo_matches_reference(case, oracle_mod, golden):
    """The thermo restatement against the reference's own thermo lines: at
    step 0 from the setup tallies (every field), at the last step from the
    reference's end velocities (temperature, kinetic energy, volume)."""
    g = golden(case)
    build, _, _ = CASES[case]
    s = build()
    rows = g["thermo_rows"]
    fields = oracle_mod.THERMO_FIELDS
    assert tuple(g["thermo_columns"][1:]) == oracle_mod.THERMO_COLUMNS
    t0 = oracle_mod.thermo(s.v, s.nodev, s.mass, s.boxlo, s.boxhi, g["energy"], g["virial"])
    assert rows[0, 0] == 0
    assert thermo_err(t0, rows[0, 1:], fields) < 1e-14
    tn = oracle_mod.thermo(g["end_v"], g["end_nodev"], s.mass, s.boxlo, s.boxhi, 0.0, np.zeros(6))
    assert rows[1, 0] == int(g["nsteps"])
    keep = [fields.index(k) for k in ("temp", "ke", "vol")]
    assert thermo_err(tn, rows[1, 1:][keep], [fields[i] for i in keep]) < 1e-12


def test_thermo_units_and_empty(oracle_mod):
    """metalgpa pressures are metal's divided by 1e4; a system with no sites
    has zero temperature (ComputeTemp::dof_compute sets tfactor 0)."""
    s = CASES["tiny_lj"][0]()
    w = np.arange(1.0, 7.0)
    a = oracle_mod.thermo(s.v, s.nodev, s.mass, s.boxlo, s.boxhi, -1.0, w, units="metal")
    b = oracle_mod.thermo(s.v, s.nodev, s.mass, s.boxlo, s.boxhi, -1.0, w, units="metalgpa")
    assert abs(a["press"] / 1e4 - b["press"]) < 1e-12 * abs(a["press"])
    e = oracle_mod.thermo(np.zeros((0, 3)), np.zeros((0, 8, 3)), 1.0, [0, 0, 0], [1, 1, 1], 0.0, np.zeros(6))
    assert e["temp"] == 0.0 and e["ke"] == 0.0 and e["press"] == 0.0


@pytest.mark.parametrize("case", ["tiny_lj", "tiny_eam", "lj_small"])
def test_langevin_setup_matches_reference(case, oracle_mod, golden):
    """The RanMars and FixLangevin restatement against the reference's setup
    forces with fix langevin: its pair forces plus the first draws, bit for
    bit with zero no (the same operations in the same order), and with zero
    yes (the mean is summed in the same sequential order)."""
    g = golden(case)
    s = CASES[case][0]()
    t0, _, damp, seed, zero = g["lgv_params"]
    f, nf = g["f"].copy(), g["nodef"].copy()
    rng = oracle_mod.RanMars(int(seed))
    oracle_mod.langevin_post_force(f, nf, np.asarray(s.v), np.asarray(s.nodev), rng, s.mass,
                                   oracle_mod.langevin_target(t0, 0.0, 0, 0, 1), damp, 0.001, bool(zero))
    assert np.array_equal(f, g["lgv_setup_f"])
    assert np.array_equal(nf, g["lgv_setup_nodef"])


def test_ranmars_restatement_properties(oracle_mod):
    """RanMars values are multiples of 2^-24 in [0, 1); different seeds give
    different streams; the reference's seed bounds are enforced."""
    a, b = oracle_mod.RanMars(1), oracle_mod.RanMars(2)
    xa = [a.uniform() for _ in range(1000)]
    xb = [b.uniform() for _ in range(1000)]
    assert all(0.0 <= x < 1.0 and x * 16777216.0 == int(x * 16777216.0) for x in xa)
    assert xa != xb
    assert abs(np.mean(xa) - 0.5) < 0.05
    for bad in (0, 900000001):
        with pytest.raises(ValueError):
            oracle_mod.RanMars(bad)


@pytest.mark.parametrize("case", ["tiny_lj", "tiny_eam", "lj_small"])
def test_deform_box_matches_reference(case, oracle_mod, golden):
    """The fix deform box arithmetic restated against the reference's box
    after consecutive runs (every style of the cases: erate, volume, vel,
    trate, wiggle, final, scale, delta), bit for bit."""
    g = golden(case)
    s = CASES[case][0]()
    lo, hi = oracle_mod.deform_boxes(s.boxlo, s.boxhi, int(g["dfm_nevery"]), g["dfm_style"], g["dfm_a"],
                                     g["dfm_b"], [int(n) for n in g["dfm_runs"]])
    box = g["dfm_end_box"]
    assert lo == [box[0], box[2], box[4]]
    assert hi == [box[1], box[3], box[5]]
