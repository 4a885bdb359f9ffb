"""Generate the golden fixtures of this directory by running the CAC reference
(compiled by ``oracle/Makefile`` into ``oracle/_ref/``) on seeded systems from
``cac_b200.gen``.

Run from the repository root where the reference tree is available:

    make -C oracle reference && python tests/golden/make_golden.py

Each fixture ``<case>.npz`` holds the reference's own read-outs:
  setup forces (atom f, nodal f, Gauss-point f), energy, virial and per-site
  energy/virial (``oracle_dump compute``); the sha256 digest and per-site
  counts of its half and full neighbour lists (``oracle_dump_neigh``); for
  trajectory cases the state after N velocity-Verlet steps; and its thermo
  lines (``thermo_style custom step temp ke pe etotal press pxx pyy pzz pxy
  pxz pyz vol``, printed with ``%.17g``) at step 0 and step N; and with
  ``fix langevin`` (the ``LANGEVIN`` cases) its setup forces and the state
  after consecutive runs; with ``fix deform`` (the ``DEFORM`` cases) the
  state and box after consecutive runs; and with both fixes together.
EAM energies come from the executable with the patched ``compute_fp``
(``cac_eamfix``); the unpatched reference energy is kept as ``energy_unpatched``.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from cac_b200 import gen  # noqa: E402
import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

HEADER = """units metal
dimension 3
boundary p p p
atom_style atomic
element_style cac 8 1 wscale 1 1 1 1
read_data data.cac
"""


def pair_lines(pair: str) -> str:
    if pair == "lj":
        return "pair_style lj/cut 5.5\npair_coeff 1 1 0.4093 2.338\n"
    if pair == "lj_full":
        return "pair_style lj/cut/fulllist 5.5\npair_coeff 1 1 0.4093 2.338\n"
    if pair == "eam":
        return "pair_style eam/alloy\npair_coeff * * cu.setfl Cu\n"
    raise ValueError(pair)


def digest(rows: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(rows, dtype="<i8").tobytes()).hexdigest()


def counts(rows: np.ndarray, nsites: int) -> np.ndarray:
    return np.bincount(rows[:, 0], minlength=nsites).astype(np.int32)


def run(work: str, script: str, exe: str) -> None:
    with open(os.path.join(work, "in.cac"), "w") as f:
        f.write(script)
    O.run_reference(work, "in.cac", exe=exe)


THERMO = ("thermo_style custom step temp ke pe etotal press pxx pyy pzz pxy pxz pyz vol\n"
          "thermo_modify format float %.17g\n")


def thermo_rows(work: str, pair: str, nsteps: int, exe: str) -> dict:
    """The reference's thermo lines (full precision) at step 0 and step
    ``nsteps``: columns Step, then ``O.THERMO_COLUMNS``."""
    tail = "neighbor 1.0 bin\nneigh_modify every 10 delay 0 check no\ntimestep 0.001\nfix 1 all nve\n"
    with open(os.path.join(work, "in.cac"), "w") as f:
        f.write(HEADER + pair_lines(pair) + tail + THERMO + f"thermo {max(nsteps, 1)}\nrun {nsteps}\n")
    rows = O.read_thermo(O.run_reference(work, "in.cac", exe=exe))
    if rows.shape[0] != (2 if nsteps else 1):
        raise RuntimeError(f"unexpected thermo output: {rows.shape[0]} rows")
    return {"thermo_rows": rows, "thermo_columns": np.array(("Step",) + O.THERMO_COLUMNS)}


# fix langevin cases: t_start, t_stop, t_period, seed, zero; the run lengths
LANGEVIN = {
    "tiny_lj": ((50.0, 150.0, 0.05, 48279, 1), (20, 20)),
    "tiny_eam": ((300.0, 300.0, 0.1, 9173, 0), (30,)),
    "lj_small": ((80.0, 20.0, 0.2, 5501, 1), (15, 10)),
}


def langevin_rows(work: str, pair: str, exe: str, params, runs) -> dict:
    """The reference with ``fix langevin`` after ``fix nve``: the forces of
    its setup (``run 0``: pair forces plus the fix's first draws), and the
    state after the given consecutive runs (each run draws again at its
    setup and ramps the target over its own steps)."""
    t0, t1, damp, seed, zero = params
    tail = "neighbor 1.0 bin\nneigh_modify every 10 delay 0 check no\ntimestep 0.001\nfix 1 all nve\n"
    fix = f"fix 2 all langevin {t0!r} {t1!r} {damp!r} {seed} zero {'yes' if zero else 'no'}\n"
    out = {"lgv_params": np.array(params, dtype=np.float64), "lgv_runs": np.array(runs, dtype=np.int64)}
    run(work, HEADER + pair_lines(pair) + tail + fix + "run 0\noracle_dump lgv0.txt state\n", exe)
    d = O.read_dump(os.path.join(work, "lgv0.txt"))
    out["lgv_setup_f"], out["lgv_setup_nodef"] = d["f"], d["nodef"]
    script = HEADER + pair_lines(pair) + tail + fix + "".join(f"run {n}\n" for n in runs)
    run(work, script + "oracle_dump lgv1.txt state\n", exe)
    e = O.read_dump(os.path.join(work, "lgv1.txt"))
    for k in ("x", "v", "f", "nodex", "nodev", "nodef"):
        out["lgv_end_" + k] = e[k]
    return out


def add_langevin(name: str, system, pair: str) -> None:
    """Add the fix langevin read-outs to an existing fixture."""
    path = os.path.join(OUT, name + ".npz")
    with np.load(path) as z:
        out = {k: z[k] for k in z.files}
    work = tempfile.mkdtemp(prefix="cacgold_")
    try:
        gen.write_data(system, os.path.join(work, "data.cac"))
        gen.write_setfl(gen.EamParams(), os.path.join(work, "cu.setfl"))
        out.update(langevin_rows(work, pair, O.REF_EXE, *LANGEVIN[name]))
    finally:
        shutil.rmtree(work, ignore_errors=True)
    np.savez_compressed(path, **out)
    print(name, "langevin", float(np.abs(out["lgv_end_v"]).max()))


# fix deform cases: N, per-dimension (style, a, b) in box units, the run lengths;
# "final" edges are offsets from the case's own box
DEFORM_STYLES = ("none", "final", "delta", "scale", "vel", "erate", "trate", "wiggle", "volume")
DEFORM = {
    "tiny_lj": (1, (("erate", 0.5, 0.0), ("volume", 0.0, 0.0), ("vel", 0.4, 0.0)), (20, 20)),
    "tiny_eam": (2, (("trate", 0.2, 0.0), ("none", 0.0, 0.0), ("wiggle", 0.3, 0.01)), (30,)),
    "lj_small": (1, (("final", -0.05, 0.05), ("scale", 0.995, 0.0), ("delta", -0.02, 0.03)), (25,)),
}


def deform_spec(name: str, system):
    """(N, styles, a, b, runs) with final edges made absolute for this system."""
    nevery, dims, runs = DEFORM[name]
    style, a, b = [], [], []
    for d, (st, x, y) in enumerate(dims):
        if st == "final":
            x, y = float(system.boxlo[d]) + x, float(system.boxhi[d]) + y
        style.append(DEFORM_STYLES.index(st))
        a.append(float(x))
        b.append(float(y))
    return nevery, style, a, b, runs


def deform_rows(work: str, pair: str, exe: str, system, name: str) -> dict:
    """The reference with ``fix deform ... units box remap x`` after ``fix
    nve``: the state and box after the given consecutive runs."""
    nevery, style, a, b, runs = deform_spec(name, system)
    args = []
    for d in range(3):
        st = DEFORM_STYLES[style[d]]
        if st == "none":
            continue
        n = {"final": 2, "delta": 2, "wiggle": 2, "scale": 1, "vel": 1, "erate": 1, "trate": 1, "volume": 0}[st]
        args.append(" ".join(["xyz"[d], st] + [repr(v) for v in (a[d], b[d])[:n]]))
    tail = "neighbor 1.0 bin\nneigh_modify every 10 delay 0 check no\ntimestep 0.001\nfix 1 all nve\n"
    fix = f"fix 3 all deform {nevery} {' '.join(args)} units box remap x\n"
    script = HEADER + pair_lines(pair) + tail + fix + "".join(f"run {n}\n" for n in runs)
    run(work, script + "oracle_dump dfm1.txt state\n", exe)
    e = O.read_dump(os.path.join(work, "dfm1.txt"))
    out = {"dfm_nevery": np.int64(nevery), "dfm_style": np.array(style, dtype=np.int64),
           "dfm_a": np.array(a), "dfm_b": np.array(b), "dfm_runs": np.array(runs, dtype=np.int64),
           "dfm_end_box": e["box"]}
    for k in ("x", "v", "f", "nodex", "nodev", "nodef"):
        out["dfm_end_" + k] = e[k]
    return out


def both_rows(work: str, pair: str, exe: str, system, name: str) -> dict:
    """The reference with fix langevin (post_force) and fix deform
    (end_of_step) together after fix nve, over the langevin case's runs."""
    nevery, style, a, b, _ = deform_spec(name, system)
    t0, t1, damp, seed, zero = LANGEVIN[name][0]
    runs = LANGEVIN[name][1]
    args = []
    for d in range(3):
        st = DEFORM_STYLES[style[d]]
        if st == "none":
            continue
        n = {"final": 2, "delta": 2, "wiggle": 2, "scale": 1, "vel": 1, "erate": 1, "trate": 1, "volume": 0}[st]
        args.append(" ".join(["xyz"[d], st] + [repr(v) for v in (a[d], b[d])[:n]]))
    tail = "neighbor 1.0 bin\nneigh_modify every 10 delay 0 check no\ntimestep 0.001\nfix 1 all nve\n"
    fixes = (f"fix 2 all langevin {t0!r} {t1!r} {damp!r} {seed} zero {'yes' if zero else 'no'}\n"
             f"fix 3 all deform {nevery} {' '.join(args)} units box remap x\n")
    run(work, HEADER + pair_lines(pair) + tail + fixes + "".join(f"run {n}\n" for n in runs) +
        "oracle_dump both.txt state\n", exe)
    e = O.read_dump(os.path.join(work, "both.txt"))
    out = {"both_end_box": e["box"]}
    for k in ("x", "v", "f", "nodex", "nodev", "nodef"):
        out["both_end_" + k] = e[k]
    return out


def add_both(name: str, system, pair: str) -> None:
    """Add the langevin + deform read-outs to an existing fixture."""
    path = os.path.join(OUT, name + ".npz")
    with np.load(path) as z:
        out = {k: z[k] for k in z.files}
    work = tempfile.mkdtemp(prefix="cacgold_")
    try:
        gen.write_data(system, os.path.join(work, "data.cac"))
        gen.write_setfl(gen.EamParams(), os.path.join(work, "cu.setfl"))
        out.update(both_rows(work, pair, O.REF_EXE, system, name))
    finally:
        shutil.rmtree(work, ignore_errors=True)
    np.savez_compressed(path, **out)
    print(name, "langevin + deform box", out["both_end_box"].tolist())


def add_deform(name: str, system, pair: str) -> None:
    """Add the fix deform read-outs to an existing fixture."""
    path = os.path.join(OUT, name + ".npz")
    with np.load(path) as z:
        out = {k: z[k] for k in z.files}
    work = tempfile.mkdtemp(prefix="cacgold_")
    try:
        gen.write_data(system, os.path.join(work, "data.cac"))
        gen.write_setfl(gen.EamParams(), os.path.join(work, "cu.setfl"))
        out.update(deform_rows(work, pair, O.REF_EXE, system, name))
    finally:
        shutil.rmtree(work, ignore_errors=True)
    np.savez_compressed(path, **out)
    print(name, "deform box", out["dfm_end_box"].tolist())


def add_thermo(name: str, system, pair: str) -> None:
    """Add the thermo rows to an existing fixture, leaving its other arrays as they are."""
    path = os.path.join(OUT, name + ".npz")
    with np.load(path) as z:
        out = {k: z[k] for k in z.files}
    nsteps = int(out.get("nsteps", 0))
    work = tempfile.mkdtemp(prefix="cacgold_")
    try:
        gen.write_data(system, os.path.join(work, "data.cac"))
        gen.write_setfl(gen.EamParams(), os.path.join(work, "cu.setfl"))
        out.update(thermo_rows(work, pair, nsteps, O.REF_EXE_EAMFIX if pair == "eam" else O.REF_EXE))
    finally:
        shutil.rmtree(work, ignore_errors=True)
    np.savez_compressed(path, **out)
    print(name, "thermo", out["thermo_rows"][:, :3].tolist())


def make_case(name: str, system, pair: str, nsteps: int = 0, peratom_virial: bool = True) -> None:
    work = tempfile.mkdtemp(prefix="cacgold_")
    try:
        gen.write_data(system, os.path.join(work, "data.cac"))
        gen.write_setfl(gen.EamParams(), os.path.join(work, "cu.setfl"))
        tail = "neighbor 1.0 bin\nneigh_modify every 10 delay 0 check no\ntimestep 0.001\nfix 1 all nve\n"
        out = {}
        exe_e = O.REF_EXE_EAMFIX if pair == "eam" else O.REF_EXE
        run(work, HEADER + pair_lines(pair) + tail +
            "run 0\noracle_dump setup.txt compute\noracle_dump_neigh half.txt\n", exe_e)
        d = O.read_dump(os.path.join(work, "setup.txt"))
        for k in ("f", "nodef", "gaussf_at_node", "eatom", "enode", "virial"):
            out[k] = d[k]
        if peratom_virial:
            out["vatom"], out["vnode"] = d["vatom"], d["vnode"]
        out["energy"] = np.float64(d["energy"])
        if pair == "eam":
            run(work, HEADER + pair_lines(pair) + tail + "run 0\noracle_dump unpatched.txt compute\n", O.REF_EXE)
            out["energy_unpatched"] = np.float64(O.read_dump(os.path.join(work, "unpatched.txt"))["energy"])
        nsites = system.natoms + 8 * system.nelements
        half = O.read_neigh(os.path.join(work, "half.txt"), system.natoms)
        full_pair = "lj_full" if pair.startswith("lj") else "lj_full"
        fscript = HEADER + pair_lines(full_pair)
        if pair == "eam":
            fscript = fscript.replace("5.5", "5.0")
        run(work, fscript + tail + "run 0\noracle_dump_neigh full.txt\n", O.REF_EXE)
        full = O.read_neigh(os.path.join(work, "full.txt"), system.natoms)
        out["half_digest"] = np.array(digest(half))
        out["full_digest"] = np.array(digest(full))
        out["half_counts"] = counts(half, nsites)
        out["full_counts"] = counts(full, nsites)
        if nsteps:
            run(work, HEADER + pair_lines(pair) + tail + f"run {nsteps}\noracle_dump end.txt state\n", exe_e)
            e = O.read_dump(os.path.join(work, "end.txt"))
            out["nsteps"] = np.int64(nsteps)
            for k in ("x", "v", "f", "nodex", "nodev", "nodef"):
                out["end_" + k] = e[k]
        out.update(thermo_rows(work, pair, nsteps, exe_e))
        out.update(langevin_rows(work, pair, O.REF_EXE, *LANGEVIN[name]))
        out.update(deform_rows(work, pair, O.REF_EXE, system, name))
        out.update(both_rows(work, pair, O.REF_EXE, system, name))
        meta = dict(system.meta)
        out["meta"] = np.array(repr(sorted(meta.items())))
        np.savez_compressed(os.path.join(OUT, name + ".npz"), **out)
        print(name, "sites", nsites, "half", len(half), "full", len(full), "energy", out["energy"])
    finally:
        shutil.rmtree(work, ignore_errors=True)


CASES = (
    ("tiny_lj", lambda: gen.tiny(seed=7, temperature=50.0), "lj", dict(nsteps=100)),
    ("tiny_eam", lambda: gen.tiny(seed=11, temperature=300.0), "eam", dict(nsteps=50)),
    ("lj_small", lambda: gen.lj_small(seed=1), "lj", dict(nsteps=100, peratom_virial=False)),
)


def main():
    """``make_golden.py`` writes every fixture; ``make_golden.py thermo``,
    ``langevin``, ``deform`` or ``both`` only adds those read-outs to the fixtures
    already here."""
    if not os.path.exists(O.REF_EXE):
        raise SystemExit("build the reference first: make -C oracle reference")
    only = sys.argv[1] if sys.argv[1:] else None
    if only not in (None, "thermo", "langevin", "deform", "both"):
        raise SystemExit(f"unknown mode {only!r}")
    for name, system, pair, kw in CASES:
        if only == "thermo":
            add_thermo(name, system(), pair)
        elif only == "langevin":
            add_langevin(name, system(), pair)
        elif only == "deform":
            add_deform(name, system(), pair)
        elif only == "both":
            add_both(name, system(), pair)
        else:
            make_case(name, system(), pair, **kw)


if __name__ == "__main__":
    main()
