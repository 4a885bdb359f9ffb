"""Serving: jobs served concurrently must equal the same jobs run alone.

Each worker owns a context and runs a job through the same calls as a single
run, so the final state, energy, iteration count and stop code of every job
must match a run of that job alone bit for bit, whatever ran beside it, in
either precision form.  Admission follows the memory budget: a job larger than
the budget is refused at submission, and a budget that fits two small jobs at
a time still completes every job."""
import numpy as np
import pytest

from cac_b200 import gen
from helpers import SKIN, setfl_path

pytestmark = pytest.mark.gpu

NVE_STEPS = 30
FIRE_ITERS = 60
FTOL = 1e-6


def jobs():
    out = []
    for k, (ta, te, kind) in enumerate([(2000, 40, 0), (4000, 80, 1), (1500, 30, 1),
                                         (6000, 120, 0), (2500, 50, 1), (3000, 60, 0)]):
        s = gen.replica(ta, te, temperature=200.0 if kind == 0 else 0.0, strain=0.01 * k, seed=70 + k)
        out.append((s, kind))
    return out


def alone(s, kind, form, setfl):
    from cac_b200.api import ENERGY_GLOBAL, Engine
    e = Engine(0)
    e.upload(s)
    e.pair_eam(setfl)
    e.neighbor(SKIN, 10)
    e.set_precision(form)
    if kind == 0:
        e.setup()
        e.run_nve(NVE_STEPS, 0.001, eflag=ENERGY_GLOBAL)
        energy, it, code = e.energy(peratom=False)["energy"], NVE_STEPS, -1
    else:
        code, it, energy, _ = e.minimize_fire(0.0, FTOL, FIRE_ITERS, 0.001, norm="max")
    x, v, nx, nv = e.state()
    e.close()
    return x, v, nx, nv, energy, it, code


@pytest.mark.parametrize("form", [0, 1])
def test_served_jobs_equal_alone(form, tmp_path):
    from cac_b200.api import Server
    setfl = setfl_path(tmp_path)
    js = jobs()
    srv = Server(0, workers=3, budget_gb=8.0, precision=form)
    srv.pair_eam(setfl)
    srv.neighbor(SKIN, 10)
    srv.start()
    ids = [srv.submit(s, kind, NVE_STEPS if kind == 0 else FIRE_ITERS, 0.001, 0.0, FTOL) for s, kind in js]
    for j in ids:
        assert srv.wait(j) == 0, srv.last_error()
    for (s, kind), j in zip(js, ids):
        got = srv.result(j)
        want = alone(s, kind, form, setfl)
        for a, b in zip(got[:4], want[:4]):
            assert np.array_equal(a, b)
        assert got[4] == want[4]
        assert got[5] == want[5] and got[6] == want[6]
        t = got[7]
        assert t[0] >= 0.0 and t[1] > 0.0 and abs(t[2] - t[0] - t[1]) < 1e-6
        srv.release(j)
    srv.close()


def test_budget_admission(tmp_path):
    from cac_b200.api import CacB200Error, Server
    setfl = setfl_path(tmp_path)
    big = gen.replica(60000, 2000, temperature=10.0, strain=0.0, seed=90)
    srv = Server(0, workers=2, budget_gb=0.2, precision=0)
    srv.pair_eam(setfl)
    srv.neighbor(SKIN, 10)
    srv.start()
    with pytest.raises(CacB200Error):
        srv.submit(big, 0, 5)
    small = [gen.replica(2000, 40, temperature=50.0, strain=0.0, seed=91 + k) for k in range(3)]
    ids = [srv.submit(s, 0, 5) for s in small]
    for j in ids:
        assert srv.wait(j) == 0, srv.last_error()
    srv.close()


def test_served_nvt_and_thermo_equal_alone(tmp_path):
    """NVT jobs (fix langevin) served beside NVE and FIRE jobs equal the same
    run on one context bit for bit, and each job's device thermo line equals
    the context's read-out after that run."""
    from cac_b200.api import ENERGY_GLOBAL, VIRIAL_GLOBAL, Engine, Server
    setfl = setfl_path(tmp_path)
    js = jobs()[:4]
    lgv = (150.0, 250.0, 0.05, 8811, True)
    srv = Server(0, workers=3, budget_gb=8.0, precision=0)
    srv.pair_eam(setfl)
    srv.neighbor(SKIN, 10)
    srv.start()
    ids = []
    for k, (s, kind) in enumerate(js):
        if k % 2 == 0:
            ids.append((srv.submit_nvt(s, NVE_STEPS, 0.001, *lgv), "nvt"))
        else:
            ids.append((srv.submit(s, kind, NVE_STEPS if kind == 0 else FIRE_ITERS, 0.001, 0.0, FTOL),
                        "nve" if kind == 0 else "fire"))
    for j, _ in ids:
        assert srv.wait(j) == 0, srv.last_error()
    for (s, kind), (j, what) in zip(js, ids):
        x, v, nx, nv, energy, _, _, _ = srv.result(j)
        th = srv.thermo(j)
        e = Engine(0)
        e.upload(s)
        e.pair_eam(setfl)
        e.neighbor(SKIN, 10)
        if what == "fire":
            e.minimize_fire(0.0, FTOL, FIRE_ITERS, 0.001, norm="max")
            e.compute(ENERGY_GLOBAL, VIRIAL_GLOBAL)
        else:
            if what == "nvt":
                e.langevin(*lgv)
            e.setup()
            e.run_nve(NVE_STEPS, 0.001, ENERGY_GLOBAL, VIRIAL_GLOBAL)
        ref = e.thermo()
        xr, vr, nxr, nvr = e.state()
        e.close()
        assert np.array_equal(x, xr) and np.array_equal(v, vr), what
        assert np.array_equal(nx, nxr) and np.array_equal(nv, nvr), what
        for key, val in ref.items():
            assert th[key] == val, (what, key)
        srv.release(j)
    srv.close()
