"""Accuracy of the mixed-precision form against the FP64 form on one system.

    python -m cac_b200.accuracy --workload eam_small --steps 50

Prints one JSON line: for the starting state, the largest and the RMS
per-site force error (atoms and Gauss points; nodes separately) relative to
the largest FP64 per-site force, and the relative potential-energy and
virial errors; along a velocity-Verlet trajectory of --steps steps run from
the same state in both forms, the largest relative deviation of the mixed
potential energy from the FP64 one, and the final position deviation.
Systems are the seeded generator's workloads (``bench.py`` names).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _system(name: str):
    from cac_b200 import gen
    table = {
        "lj_small": (lambda: gen.lj_small(seed=1), "lj"),
        "eam_small": (lambda: gen.eam_small(seed=5), "eam"),
        "eam_1m": (lambda: gen.eam_1m(seed=2), "eam"),
        "eam_4m_strained": (lambda: gen.eam_4m_strained(seed=3), "eam"),
    }
    if name not in table:
        raise SystemExit(f"unknown workload {name}")
    make, pair = table[name]
    return make(), pair


def _engine(s, pair, form, setfl):
    from cac_b200 import api
    e = api.Engine(0)
    e.upload(s)
    if pair == "eam":
        e.pair_eam(setfl)
    else:
        e.pair_lj(0.4093, 2.338, 5.5)
    e.neighbor(1.0, 10)
    e.set_precision(form)
    return e


def measure(name: str, steps: int) -> dict:
    from cac_b200 import api, gen
    s, pair = _system(name)
    setfl = os.path.join(tempfile.mkdtemp(), "cu.setfl")
    gen.write_setfl(gen.EamParams(), setfl)
    out = {"workload": name, "sites": s.nsites, "pair": pair, "steps": steps}
    ref = _engine(s, pair, api.FP64, setfl)
    mix = _engine(s, pair, api.MIXED, setfl)
    for e in (ref, mix):
        e.compute(api.ENERGY_GLOBAL, api.VIRIAL_GLOBAL)
    f64, nf64, gf64 = ref.forces()
    f32, nf32, gf32 = mix.forces()
    site64 = np.concatenate([f64, gf64.reshape(-1, 3)])
    site32 = np.concatenate([f32, gf32.reshape(-1, 3)])
    scale = np.linalg.norm(site64, axis=1).max()
    err = np.linalg.norm(site32 - site64, axis=1) / scale
    nscale = np.linalg.norm(nf64.reshape(-1, 3), axis=1).max()
    nerr = np.linalg.norm((nf32 - nf64).reshape(-1, 3), axis=1) / nscale if s.nelements else np.zeros(1)
    e64, e32 = ref.energy(peratom=False), mix.energy(peratom=False)
    out.update({
        "force_err_max": float(err.max()), "force_err_rms": float(np.sqrt(np.mean(err ** 2))),
        "node_force_err_max": float(nerr.max()),
        "energy_rel_err": abs(e32["energy"] - e64["energy"]) / abs(e64["energy"]),
        "virial_rel_err": float(np.abs(e32["virial"] - e64["virial"]).max() / np.abs(e64["virial"]).max()),
    })
    # trajectories from the same state
    dev = 0.0
    for e in (ref, mix):
        e.setup()
    for k in range(steps):
        pe = []
        for e in (ref, mix):
            e.run_nve(1, 0.001, eflag=api.ENERGY_GLOBAL)
            pe.append(e.energy(peratom=False)["energy"])
        dev = max(dev, abs(pe[1] - pe[0]) / abs(pe[0]))
    x64 = ref.state()[0]
    x32 = mix.state()[0]
    L = np.asarray(s.boxhi) - np.asarray(s.boxlo)
    d = x32 - x64
    d -= np.round(d / L) * L
    out.update({"energy_traj_max_rel_dev": dev, "final_pos_dev_max_A": float(np.abs(d).max()) if len(d) else 0.0})
    ref.close()
    mix.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="eam_small")
    ap.add_argument("--steps", type=int, default=50)
    a = ap.parse_args()
    print(json.dumps(measure(a.workload, a.steps)))


if __name__ == "__main__":
    main()
