"""Mixed-precision form against the FP64 form, and FIRE against its C
restatement.  Mixed tolerance: max per-site force error under 1e-5 of the
largest per-site force (the mixed form's stated bound); energies within 1e-6
relative."""
import numpy as np
import pytest

from cac_b200 import gen
from helpers import LJ, SKIN, rel_err, setfl_path

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-5


def engine(system, pair, tmp_path, form):
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


@pytest.mark.parametrize("pair,builder", [
    ("lj", lambda: gen.lj_small(seed=1)),
    ("eam", lambda: gen.build_slab(4, 2, 3, 9, temperature=300.0, seed=21)),
    ("eam", lambda: gen.build_slab(4, 2, 3, 9, temperature=300.0, strain=0.03, seed=22)),
])
def test_mixed_forces_within_bound(pair, builder, tmp_path):
    from cac_b200.api import FP64, MIXED
    s = builder()
    ref = engine(s, pair, tmp_path, FP64)
    ref.compute()
    f64, nf64, gf64 = ref.forces()
    e64 = ref.energy()
    mix = engine(s, pair, tmp_path, MIXED)
    mix.compute()
    f32, nf32, gf32 = mix.forces()
    e32 = mix.energy()
    scale = max(np.linalg.norm(f64, axis=1).max(), np.linalg.norm(gf64.reshape(-1, 3), axis=1).max())
    err = max(np.linalg.norm(f32 - f64, axis=1).max(),
              np.linalg.norm((gf32 - gf64).reshape(-1, 3), axis=1).max()) / scale
    assert err < MIXED_TOL, err
    assert rel_err(nf32, nf64) < 10 * MIXED_TOL
    assert abs(e32["energy"] - e64["energy"]) / abs(e64["energy"]) < 1e-6
    assert np.abs(e32["virial"] - e64["virial"]).max() / np.abs(e64["virial"]).max() < 1e-5
    ref.close()
    mix.close()


def test_mixed_trajectory_tracks_fp64(tmp_path):
    from cac_b200.api import FP64, MIXED
    s = gen.build_slab(4, 2, 3, 9, temperature=300.0, seed=23)
    out = []
    for form in (FP64, MIXED):
        e = engine(s, "eam", tmp_path, form)
        e.setup()
        e.run_nve(50, 0.001)
        out.append(e.state())
        e.close()
    (x64, v64, nx64, nv64), (x32, v32, nx32, nv32) = out
    assert np.abs(x32 - x64).max() < 1e-4
    assert np.abs(nx32 - nx64).max() < 1e-4


@pytest.mark.parametrize("pair", ["lj"])
def test_fire_matches_restatement(pair, oracle_mod, tmp_path):
    """Same algorithm, same operation order: both converge (FTOL on the max
    per-site force, 1e-6 eV/A) in (nearly) the same number of iterations at the
    same energy and configuration."""
    s = gen.tiny(seed=9, temperature=0.0)
    maxiter = 2500
    e = engine(s, pair, tmp_path, 0)
    code, it, en, fn = e.minimize_fire(ftol=1e-6, maxiter=maxiter, norm="max")
    x, _, nx, _ = e.state()
    st = oracle_mod.OracleState(s)
    eam = oracle_mod.Eam(setfl_path(tmp_path)) if pair == "eam" else None
    ocode, oit, oen, ofn = oracle_mod.minimize_fire(st, pair, lj=LJ, eam=eam, ftol=1e-6, maxiter=maxiter,
                                                    norm="max")
    assert code == ocode == 3
    assert abs(it - oit) <= max(2, oit // 50)
    assert abs(en - oen) / abs(oen) < 1e-8
    assert np.abs(x - st.x).max() < 1e-5
    assert np.abs(nx - st.nodex).max() < 1e-5
    e.close()


@pytest.mark.parametrize("pair", ["lj", "eam"])
def test_fire_short_run_bitwise_close(pair, oracle_mod, tmp_path):
    """20 iterations: positions agree to 1e-10 (only summation order differs)."""
    s = gen.tiny(seed=12, temperature=0.0)
    e = engine(s, pair, tmp_path, 0)
    e.minimize_fire(ftol=0.0, maxiter=20, norm="two")
    x, _, nx, _ = e.state()
    st = oracle_mod.OracleState(s)
    eam = oracle_mod.Eam(setfl_path(tmp_path)) if pair == "eam" else None
    oracle_mod.minimize_fire(st, pair, lj=LJ, eam=eam, ftol=0.0, maxiter=20, norm="two")
    assert np.abs(x - st.x).max() < 1e-10
    assert np.abs(nx - st.nodex).max() < 1e-10
    e.close()


@pytest.mark.parametrize("pair", ["lj", "eam"])
def test_fire_check_yes_matches_restatement(pair, oracle_mod, tmp_path):
    """The reference Min's neighbour rule (every 1 delay 0 check yes) on the
    device and in the C restatement: 20 iterations agree to 1e-10, and a
    converged run stops like the restatement."""
    s = gen.tiny(seed=12, temperature=0.0)
    eam = oracle_mod.Eam(setfl_path(tmp_path)) if pair == "eam" else None
    e = engine(s, pair, tmp_path, 0)
    e.neighbor(SKIN, 1)
    e.neighbor_modify(0, True)
    e.minimize_fire(ftol=0.0, maxiter=20, norm="two")
    x, _, nx, _ = e.state()
    e.close()
    st = oracle_mod.OracleState(s)
    oracle_mod.minimize_fire(st, pair, lj=LJ, eam=eam, ftol=0.0, maxiter=20, norm="two", every=1, check=True)
    assert np.abs(x - st.x).max() < 1e-10
    assert np.abs(nx - st.nodex).max() < 1e-10
    if pair == "lj":
        e = engine(s, pair, tmp_path, 0)
        e.neighbor(SKIN, 1)
        e.neighbor_modify(0, True)
        code, it, en, fn = e.minimize_fire(ftol=1e-6, maxiter=2500, norm="max")
        x, _, nx, _ = e.state()
        e.close()
        st = oracle_mod.OracleState(s)
        ocode, oit, oen, ofn = oracle_mod.minimize_fire(st, pair, lj=LJ, ftol=1e-6, maxiter=2500, norm="max",
                                                        every=1, check=True)
        assert code == ocode == 3
        assert abs(it - oit) <= max(2, oit // 50)
        assert abs(en - oen) / abs(oen) < 1e-8
        assert np.abs(x - st.x).max() < 1e-5
        assert np.abs(nx - st.nodex).max() < 1e-5
