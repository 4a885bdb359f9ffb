"""CUDA path (through the C ABI) against the reference's golden read-outs and
the CPU restatement.  Tolerances: lists bit-exact; FP64 forces, energies and
virials within 1e-10 relative (max per-site norm over the largest per-site
norm), the FP64 parity bar of the reference path."""
import numpy as np
import pytest

from cac_b200 import gen
from helpers import CASES, LJ, N2G, SKIN, counts, digest, rel_err, setfl_path

pytestmark = pytest.mark.gpu

TOL = 1e-10


def make_engine(system, pair, tmp_path):
    from cac_b200.api import Engine
    e = Engine(0)
    e.upload(system)
    if pair == "lj":
        e.pair_lj(*LJ)
    else:
        e.pair_eam(setfl_path(tmp_path))
    e.neighbor(SKIN, 10)
    return e


@pytest.mark.parametrize("case", ["tiny_lj", "tiny_eam", "lj_small"])
def test_lists_bit_exact_vs_reference(case, golden, tmp_path):
    g = golden(case)
    build, pair, _ = CASES[case]
    s = build()
    e = make_engine(s, pair, tmp_path)
    e.build_lists(half=True)
    nsites = s.natoms + 8 * s.nelements
    for half, key in ((True, "half"), (False, "full")):
        rows = e.neighbor_list(half)
        assert np.array_equal(counts(rows, nsites), g[key + "_counts"]), key
        assert digest(rows) == str(g[key + "_digest"]), key
    e.close()


@pytest.mark.parametrize("case", ["tiny_lj", "tiny_eam", "lj_small"])
def test_full_list_built_alone_bit_exact_vs_reference(case, golden, tmp_path):
    """The full list of a build that makes no half list (the build the step
    loop runs) equals the reference's."""
    g = golden(case)
    build, pair, _ = CASES[case]
    s = build()
    e = make_engine(s, pair, tmp_path)
    e.build_lists(half=False)
    rows = e.neighbor_list(False)
    nsites = s.natoms + 8 * s.nelements
    assert np.array_equal(counts(rows, nsites), g["full_counts"])
    assert digest(rows) == str(g["full_digest"])
    e.close()


@pytest.mark.parametrize("case", ["tiny_lj", "tiny_eam", "lj_small"])
def test_forces_energy_vs_reference(case, golden, tmp_path):
    g = golden(case)
    build, pair, _ = CASES[case]
    s = build()
    e = make_engine(s, pair, tmp_path)
    e.compute()
    f, nf, gf = e.forces()
    ev = e.energy()
    assert rel_err(f, g["f"]) < TOL
    assert rel_err(nf, g["nodef"]) < TOL
    assert rel_err(gf[:, N2G, :], g["gaussf_at_node"]) < TOL
    assert abs(ev["energy"] - float(g["energy"])) / abs(float(g["energy"])) < TOL
    assert np.abs(ev["virial"] - g["virial"]).max() / np.abs(g["virial"]).max() < TOL
    escale = np.abs(g["eatom"]).max()
    assert np.abs(ev["eatom"] - g["eatom"]).max() / escale < TOL
    assert np.abs(ev["enode"] - g["enode"]).max() / escale < TOL
    if "vatom" in g:
        vscale = np.abs(g["vatom"]).max()
        assert np.abs(ev["vatom"] - g["vatom"]).max() / vscale < TOL
        assert np.abs(ev["vnode"] - g["vnode"]).max() / vscale < TOL
    e.close()


@pytest.mark.parametrize("case", ["tiny_lj", "tiny_eam", "lj_small"])
def test_trajectory_vs_reference(case, golden, tmp_path):
    g = golden(case)
    build, pair, _ = CASES[case]
    s = build()
    e = make_engine(s, pair, tmp_path)
    e.setup()
    e.run_nve(int(g["nsteps"]), 0.001)
    x, v, nx, nv = e.state()
    f, nf, _ = e.forces()
    assert np.abs(x - g["end_x"]).max() < 1e-10
    assert np.abs(nx - g["end_nodex"]).max() < 1e-10
    assert rel_err(v, g["end_v"]) < TOL
    assert rel_err(nv, g["end_nodev"]) < TOL
    assert rel_err(f, g["end_f"]) < TOL
    assert rel_err(nf, g["end_nodef"]) < TOL
    e.close()


@pytest.mark.parametrize("seed,pair,T", [(101, "lj", 10.0), (202, "eam", 300.0), (303, "eam", 600.0)])
def test_seeded_vs_oracle(seed, pair, T, oracle_mod, tmp_path):
    """Fresh seeded systems (not in the fixtures) against the restatement."""
    s = gen.build_slab(4, 1, 2, 6, temperature=T, seed=seed, strain=0.01 * (seed % 3))
    cut = 6.5 if pair == "lj" else 6.0
    st = oracle_mod.OracleState(s)
    e = make_engine(s, pair, tmp_path)
    e.build_lists(half=True)
    for half in (True, False):
        L = oracle_mod.build_list(st, cut, half)
        ref = L.canonical(s.natoms)
        assert np.array_equal(e.neighbor_list(half), ref)
        if half:
            if pair == "lj":
                ev = oracle_mod.lj_forces(st, L, *LJ)
            else:
                ev = oracle_mod.eam_forces(st, L, oracle_mod.Eam(setfl_path(tmp_path)))
        oracle_mod.free_list(L)
    e.compute()
    f, nf, _ = e.forces()
    out = e.energy()
    assert rel_err(f, st.f) < TOL
    assert rel_err(nf, st.nodef) < TOL
    assert abs(out["energy"] - ev.energy) / abs(ev.energy) < TOL
    assert np.abs(out["eatom"] - ev.eatom).max() / np.abs(ev.eatom).max() < TOL
    e.close()


@pytest.mark.parametrize("shift", [0.0, 4000.0])
def test_tall_and_offset_boxes_vs_oracle(shift, oracle_mod, tmp_path):
    """A 1,434 A tall box, and the same box moved 4,000 A from the origin:
    the FP32 screens of the list build must stay exact where coordinates are
    large (lists bit-exact, forces within the FP64 tolerance)."""
    s = gen.replica(1500, 600, temperature=100.0, strain=0.02, seed=5)
    if shift:
        for a in (s.x, s.nodex):
            a[..., 2] += shift
        s.boxlo[2] += shift
        s.boxhi[2] += shift
    st = oracle_mod.OracleState(s)
    e = make_engine(s, "eam", tmp_path)
    e.build_lists(half=True)
    for half in (True, False):
        L = oracle_mod.build_list(st, 6.0, half)
        assert np.array_equal(e.neighbor_list(half), L.canonical(s.natoms))
        if half:
            oracle_mod.eam_forces(st, L, oracle_mod.Eam(setfl_path(tmp_path)))
        oracle_mod.free_list(L)
    e.compute()
    f, nf, _ = e.forces()
    assert rel_err(f, st.f) < TOL
    assert rel_err(nf, st.nodef) < TOL
    e.close()


def test_empty_and_atoms_only_and_elements_only(tmp_path, oracle_mod):
    """Edge cases: no elements; no atoms."""
    s = gen.build_slab(3, 1, 0, 6, temperature=20.0, seed=5)
    assert s.nelements == 0
    e = make_engine(s, "lj", tmp_path)
    e.compute()
    f, _, _ = e.forces()
    st = oracle_mod.OracleState(s)
    L = oracle_mod.build_list(st, 6.5, True)
    oracle_mod.lj_forces(st, L, *LJ)
    oracle_mod.free_list(L)
    assert rel_err(f, st.f) < TOL
    e.close()
    s = gen.build_slab(3, 1, 1, 0, temperature=20.0, seed=6)
    assert s.natoms == 0
    e = make_engine(s, "eam", tmp_path)
    e.compute()
    _, nf, _ = e.forces()
    st = oracle_mod.OracleState(s)
    L = oracle_mod.build_list(st, 6.0, True)
    oracle_mod.eam_forces(st, L, oracle_mod.Eam(setfl_path(tmp_path)))
    oracle_mod.free_list(L)
    assert rel_err(nf, st.nodef) < TOL
    e.close()


def test_errors_are_reported_not_fatal(tmp_path):
    from cac_b200.api import CacB200Error, Engine
    e = Engine(0)
    with pytest.raises(CacB200Error):
        e.compute()               # no system yet
    s = gen.tiny()
    e.upload(s)
    with pytest.raises(CacB200Error):
        e.compute()               # no pair style
    with pytest.raises(CacB200Error):
        e.pair_lj(0.4, -1.0, 5.5)  # invalid sigma
    e.pair_lj(*LJ)
    e.neighbor(SKIN, 10)
    e.compute()                   # context still usable
    e.close()


def test_size_limits_refused_before_any_work():
    """List entries address sites with 26 bits: a system whose atoms and Gauss
    points reach 2^26, or whose lattice-site ids reach 2^30, is refused with
    EINVAL (checked before any array is read, so none is passed here); the
    context stays usable."""
    import ctypes as C
    import numpy as np
    from cac_b200.api import Engine
    e = Engine(0)
    lo = np.zeros(3)
    hi = np.full(3, 100.0)
    dp = C.POINTER(C.c_double)
    for na, ne in [(1 << 26, 0), (0, (1 << 23)), ((1 << 26) - 8, 1), (0, (1 << 30) // 729 + 1)]:
        rc = e.lib.cacb200_upload_system(e.h, lo.ctypes.data_as(dp), hi.ctypes.data_as(dp), na, None, None,
                                         ne, None, None, 1.0)
        assert rc == -1, (na, ne, rc)
        assert b"too large" in e.lib.cacb200_last_error(e.h)
    e.upload(gen.tiny())
    e.pair_lj(*LJ)
    e.neighbor(SKIN, 10)
    e.compute()
    e.close()
