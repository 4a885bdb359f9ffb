"""Thermo read-outs reduced on the device (cacb200_thermo) against the
reference's own thermo lines and the CPU restatement.

Tolerances: at step 0 every field within 1e-12 (energies and temperature
relative to their size, pressures relative to the largest pressure
component): the same terms summed in another order.  After N velocity-Verlet
steps within 1e-9, the trajectory's own FP64 agreement.  Batches: each
replica's read-out within 1e-12 of the same system run alone (per-site sums
instead of the global tally)."""
import math

import numpy as np
import pytest

from cac_b200 import gen
from helpers import CASES, LJ, SKIN, setfl_path
from test_oracle_golden import thermo_err

pytestmark = pytest.mark.gpu

FIELDS = ("temp", "ke", "pe", "etotal", "press", "pxx", "pyy", "pzz", "pxy", "pxz", "pyz", "vol")


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


@pytest.mark.parametrize("case", ["tiny_lj", "tiny_eam", "lj_small"])
def test_thermo_vs_reference(case, golden, tmp_path):
    from cac_b200.api import ENERGY_GLOBAL, VIRIAL_GLOBAL
    g = golden(case)
    build, pair, _ = CASES[case]
    e = make_engine(build(), pair, tmp_path)
    e.compute(ENERGY_GLOBAL, VIRIAL_GLOBAL)
    rows = g["thermo_rows"]
    assert thermo_err(e.thermo(), rows[0, 1:], FIELDS) < 1e-12
    gpa = e.thermo("metalgpa")
    assert abs(gpa["press"] * 1e4 - rows[0, 5]) < 1e-12 * abs(rows[0, 5])
    e.run_nve(int(g["nsteps"]), 0.001, ENERGY_GLOBAL, VIRIAL_GLOBAL)
    assert thermo_err(e.thermo(), rows[1, 1:], FIELDS) < 1e-9
    e.close()


def test_thermo_untallied_reads_nan(oracle_mod, tmp_path):
    """After force-only steps the energy and pressure fields read NaN; the
    kinetic fields still come from the current velocities."""
    s = CASES["tiny_eam"][0]()
    e = make_engine(s, "eam", tmp_path)
    e.setup()
    e.run_nve(7)
    t = e.thermo()
    for k in ("pe", "etotal", "press", "pxx", "pyz"):
        assert math.isnan(t[k]), k
    _, v, _, nv = e.state()
    ref = oracle_mod.thermo(v, nv, s.mass, s.boxlo, s.boxhi, 0.0, np.zeros(6))
    for k in ("temp", "ke", "vol"):
        assert abs(t[k] - ref[k]) <= 1e-13 * abs(ref[k]), k
    e.close()


def test_thermo_mixed_form(golden, tmp_path):
    """The mixed form's read-out: kinetic fields from the same FP64
    velocities, potential energy and pressure within the form's accuracy."""
    from cac_b200.api import ENERGY_GLOBAL, VIRIAL_GLOBAL
    g = golden("tiny_eam")
    e = make_engine(CASES["tiny_eam"][0](), "eam", tmp_path, form=1)
    e.compute(ENERGY_GLOBAL, VIRIAL_GLOBAL)
    t = e.thermo()
    ref = dict(zip(FIELDS, g["thermo_rows"][0, 1:]))
    assert abs(t["temp"] - ref["temp"]) <= 1e-13 * ref["temp"]
    assert abs(t["pe"] - ref["pe"]) <= 1e-6 * abs(ref["pe"])
    assert thermo_err(t, g["thermo_rows"][0, 1:], FIELDS) < 1e-5
    e.close()


@pytest.mark.parametrize("pair", ["lj", "eam"])
def test_thermo_batch_equals_alone(pair, tmp_path):
    from cac_b200.api import ENERGY_ATOM, ENERGY_GLOBAL, VIRIAL_ATOM, VIRIAL_GLOBAL, Engine
    systems = [
        gen.replica(2000, 50, temperature=120.0, strain=0.0, seed=41),
        gen.replica(4000, 90, temperature=400.0, strain=0.03, seed=42),
        gen.replica(1500, 0, temperature=60.0, strain=0.01, seed=43),
    ]
    b = Engine(0)
    b.upload_batch(systems)
    b.pair_lj(*LJ) if pair == "lj" else b.pair_eam(setfl_path(tmp_path))
    b.neighbor(SKIN, 10)
    b.setup()
    b.run_nve(12, 0.001, ENERGY_GLOBAL | ENERGY_ATOM, VIRIAL_GLOBAL | VIRIAL_ATOM)
    tb = b.thermo()
    b.run_nve(1)
    assert np.isnan(b.thermo()["pe"]).all()
    b.close()
    for r, s in enumerate(systems):
        e = make_engine(s, pair, tmp_path)
        e.setup()
        e.run_nve(12, 0.001, ENERGY_GLOBAL, VIRIAL_GLOBAL)
        ta = e.thermo()
        e.close()
        assert thermo_err({k: tb[k][r] for k in FIELDS}, [ta[k] for k in FIELDS], FIELDS) < 1e-12, r
