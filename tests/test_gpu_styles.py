"""The package's reference-side styles (cac_b200/styles) inside the reference's
own executable: pair_style lj/cut/b200 and eam/alloy/b200 as drop-ins for
lj/cut and eam/alloy, run_b200 and write_b200_neighbor.  The harness
executable oracle/_ref/cac_b200 is built by ``make -C oracle app``."""
import os
import subprocess

import numpy as np
import pytest

from cac_b200 import gen
from helpers import CASES, N2G, counts, digest, rel_err

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
APP = os.path.join(ROOT, "oracle", "_ref", "cac_b200")
TOL = 1e-10

HEADER = """units metal
dimension 3
boundary p p p
atom_style atomic
element_style cac 8 1 wscale 1 1 1 1
read_data data.cac
"""
TAIL = "neighbor 1.0 bin\nneigh_modify every 10 delay 0 check no\ntimestep 0.001\nfix 1 all nve\n"


def pair_lines(pair):
    if pair == "lj":
        return "pair_style lj/cut/b200 5.5\npair_coeff 1 1 0.4093 2.338\n"
    return "pair_style eam/alloy/b200\npair_coeff * * cu.setfl Cu\n"


def run_app(tmp_path, case, body):
    import oracle
    build, pair, _ = CASES[case]
    s = build()
    gen.write_data(s, str(tmp_path / "data.cac"))
    gen.write_setfl(gen.EamParams(), str(tmp_path / "cu.setfl"))
    (tmp_path / "in.cac").write_text(HEADER + pair_lines(pair) + TAIL + body)
    r = subprocess.run([APP, "-in", "in.cac"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    return s, oracle


@pytest.fixture(scope="module", autouse=True)
def app_present():
    if not os.path.exists(APP):
        pytest.fail("oracle/_ref/cac_b200 is missing: build it with make -C oracle app")


@pytest.mark.parametrize("case", ["tiny_lj", "tiny_eam"])
def test_pair_style_drop_in_setup_forces(case, golden, tmp_path):
    g = golden(case)
    s, O = run_app(tmp_path, case, "run 0\noracle_dump setup.txt compute\n")
    d = O.read_dump(str(tmp_path / "setup.txt"))
    assert rel_err(d["f"], g["f"]) < TOL
    assert rel_err(d["nodef"], g["nodef"]) < TOL
    assert rel_err(d["gaussf_at_node"], g["gaussf_at_node"]) < TOL
    assert abs(d["energy"] - float(g["energy"])) / abs(float(g["energy"])) < TOL
    assert np.abs(d["virial"] - g["virial"]).max() / np.abs(g["virial"]).max() < TOL
    assert np.abs(d["eatom"] - g["eatom"]).max() / np.abs(g["eatom"]).max() < TOL
    assert np.abs(d["enode"] - g["enode"]).max() / np.abs(g["eatom"]).max() < TOL


@pytest.mark.parametrize("case", ["tiny_lj", "tiny_eam"])
@pytest.mark.parametrize("mode", ["run", "run_b200", "run_style verlet/b200\nrun"])
def test_trajectory_in_reference_loop(case, mode, golden, tmp_path):
    """`run N` (reference Verlet + fix nve, device forces), `run_b200 N`
    and `run_style verlet/b200` + `run N` (the reference's run command with
    the whole step loop on the device) all reproduce the reference
    trajectory."""
    g = golden(case)
    n = int(g["nsteps"])
    s, O = run_app(tmp_path, case, f"{mode} {n}\noracle_dump end.txt state\n")
    e = O.read_dump(str(tmp_path / "end.txt"))
    assert np.abs(e["x"] - g["end_x"]).max() < 1e-10
    assert np.abs(e["nodex"] - g["end_nodex"]).max() < 1e-10
    assert rel_err(e["v"], g["end_v"]) < TOL
    assert rel_err(e["nodev"], g["end_nodev"]) < TOL
    assert rel_err(e["f"], g["end_f"]) < TOL
    assert rel_err(e["nodef"], g["end_nodef"]) < TOL


@pytest.mark.parametrize("case", ["tiny_lj", "tiny_eam"])
def test_device_lists_written_by_the_style(case, golden, tmp_path):
    g = golden(case)
    s, O = run_app(tmp_path, case, "write_b200_neighbor half.txt half\nwrite_b200_neighbor full.txt full\n")
    nsites = s.natoms + 8 * s.nelements
    for key in ("half", "full"):
        rows = O.read_neigh(str(tmp_path / f"{key}.txt"), s.natoms)
        assert np.array_equal(counts(rows, nsites), g[key + "_counts"])
        assert digest(rows) == str(g[key + "_digest"])


def lgv_fix(g):
    t0, t1, damp, seed, zero = (float(v) for v in g["lgv_params"])
    return f"fix 2 all langevin/b200 {t0!r} {t1!r} {damp!r} {int(seed)} zero {'yes' if zero else 'no'}\n"


def dfm_fix(g):
    names = ("none", "final", "delta", "scale", "vel", "erate", "trate", "wiggle", "volume")
    nargs = {"final": 2, "delta": 2, "wiggle": 2, "scale": 1, "vel": 1, "erate": 1, "trate": 1, "volume": 0}
    parts = []
    for d in range(3):
        st = names[int(g["dfm_style"][d])]
        if st == "none":
            continue
        vals = (float(g["dfm_a"][d]), float(g["dfm_b"][d]))[:nargs[st]]
        parts.append(" ".join(["xyz"[d], st] + [repr(v) for v in vals]))
    return f"fix 3 all deform/b200 {int(g['dfm_nevery'])} {' '.join(parts)} units box remap x\n"


def assert_state(e, g, prefix):
    assert np.abs(e["x"] - g[prefix + "x"]).max() < 1e-10
    assert np.abs(e["nodex"] - g[prefix + "nodex"]).max() < 1e-10
    assert rel_err(e["v"], g[prefix + "v"]) < TOL
    assert rel_err(e["nodev"], g[prefix + "nodev"]) < TOL
    assert rel_err(e["f"], g[prefix + "f"]) < TOL
    assert rel_err(e["nodef"], g[prefix + "nodef"]) < TOL


@pytest.mark.parametrize("order", [("run", "run_b200"), ("run_b200", "run")])
def test_langevin_style_mixes_reference_loop_and_device(order, golden, tmp_path):
    """fix langevin/b200 draws the reference's RanMars stream in both loops:
    20 steps in one and 20 in the other reproduce the reference's own
    fix langevin over two runs (the device continues the host generator, and
    the host generator is advanced past the device's draws)."""
    g = golden("tiny_lj")
    runs = [int(n) for n in g["lgv_runs"]]
    body = lgv_fix(g) + f"{order[0]} {runs[0]}\n{order[1]} {runs[1]}\noracle_dump end.txt state\n"
    s, O = run_app(tmp_path, "tiny_lj", body)
    assert_state(O.read_dump(str(tmp_path / "end.txt")), g, "lgv_end_")


def test_langevin_style_run_b200_eam(golden, tmp_path):
    g = golden("tiny_eam")
    body = lgv_fix(g) + f"run_b200 {int(g['lgv_runs'][0])}\noracle_dump end.txt state\n"
    s, O = run_app(tmp_path, "tiny_eam", body)
    assert_state(O.read_dump(str(tmp_path / "end.txt")), g, "lgv_end_")


@pytest.mark.parametrize("case,order", [("tiny_lj", ("run", "run_b200")), ("tiny_lj", ("run_b200", "run")),
                                        ("tiny_eam", ("run_b200",))])
def test_deform_style_mixes_reference_loop_and_device(case, order, golden, tmp_path):
    """fix deform/b200 in the reference loop and on the device: the box and
    the state equal the reference's own fix deform over the same runs."""
    g = golden(case)
    runs = [int(n) for n in g["dfm_runs"]]
    body = dfm_fix(g) + "".join(f"{m} {n}\n" for m, n in zip(order, runs)) + "oracle_dump end.txt state\n"
    s, O = run_app(tmp_path, case, body)
    e = O.read_dump(str(tmp_path / "end.txt"))
    assert np.array_equal(e["box"], g["dfm_end_box"])
    assert_state(e, g, "dfm_end_")


@pytest.mark.parametrize("case", ["tiny_lj", "tiny_eam"])
def test_deform_remap_v_on_device_vs_reference(case, golden, tmp_path):
    """remap v: in the reference it moves neither positions nor velocities
    (the velocity terms of Domain::remap are commented out), so run_b200 with
    fix deform/b200 ... remap v ends where the reference's own run with fix
    deform ... remap v does: the same box, positions and velocities."""
    import oracle as O
    g = golden(case)
    n = int(g["dfm_runs"][0])
    fix = dfm_fix(g).replace("remap x", "remap v")
    run_app(tmp_path, case, fix + f"run_b200 {n}\noracle_dump end.txt state\n")
    exe = O.REF_EXE_EAMFIX if CASES[case][1] == "eam" else O.REF_EXE
    reference_log(tmp_path, case, fix.replace("deform/b200", "deform") + f"run {n}\noracle_dump end.txt state\n", exe)
    a = O.read_dump(str(tmp_path / "end.txt"))
    b = O.read_dump(str(tmp_path / "ref" / "end.txt"))
    assert np.array_equal(a["box"], b["box"])
    assert np.abs(a["x"] - b["x"]).max() < 1e-10
    assert np.abs(a["nodex"] - b["nodex"]).max() < 1e-10
    assert rel_err(a["v"], b["v"]) < TOL
    assert rel_err(a["nodev"], b["nodev"]) < TOL


def test_run_b200_refuses_plain_langevin(tmp_path):
    import oracle  # noqa: F401
    build, pair, _ = CASES["tiny_lj"]
    s = build()
    gen.write_data(s, str(tmp_path / "data.cac"))
    (tmp_path / "in.cac").write_text(HEADER + pair_lines("lj") + TAIL +
                                     "fix 2 all langevin 10.0 10.0 0.1 5\nrun_b200 5\n")
    r = subprocess.run([APP, "-in", "in.cac"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode != 0
    assert "langevin/b200" in r.stdout + r.stderr


THERMO = ("thermo_style custom step temp ke pe etotal press pxx pyy pzz pxy pxz pyz vol\n"
          "thermo_modify format float %.17g\nthermo 10\n")


def app_log(tmp_path, case, body):
    """The harness executable's screen output for the /b200 deck."""
    build, pair, _ = CASES[case]
    gen.write_data(build(), str(tmp_path / "data.cac"))
    gen.write_setfl(gen.EamParams(), str(tmp_path / "cu.setfl"))
    (tmp_path / "in.cac").write_text(HEADER + pair_lines(pair) + TAIL + body)
    r = subprocess.run([APP, "-in", "in.cac"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    return r.stdout


def reference_log(tmp_path, case, body, exe):
    import oracle
    build, pair, _ = CASES[case]
    work = tmp_path / "ref"
    work.mkdir()
    gen.write_data(build(), str(work / "data.cac"))
    gen.write_setfl(gen.EamParams(), str(work / "cu.setfl"))
    plain = ("pair_style lj/cut 5.5\npair_coeff 1 1 0.4093 2.338\n" if pair == "lj"
             else "pair_style eam/alloy\npair_coeff * * cu.setfl Cu\n")
    (work / "in.cac").write_text(HEADER + plain + TAIL + body)
    return oracle.run_reference(str(work), "in.cac", exe=exe, timeout=600)


def assert_thermo_rows(ours, ref, O):
    assert ours.shape == ref.shape and ours.shape[0] >= 3
    assert np.array_equal(ours[:, 0], ref[:, 0])               # the same steps
    cols = ("step",) + O.THERMO_FIELDS
    p = [cols.index(k) for k in ("press", "pxx", "pyy", "pzz", "pxy", "pxz", "pyz")]
    pscale = np.abs(ref[:, p]).max()
    for c in range(1, ours.shape[1]):
        scale = pscale if c in p else np.abs(ref[:, c]).max()
        assert np.abs(ours[:, c] - ref[:, c]).max() <= 1e-9 * scale, cols[c]


@pytest.mark.parametrize("case", ["tiny_lj", "tiny_eam"])
def test_run_b200_prints_the_reference_thermo(case, tmp_path):
    """run_b200 under `thermo 10` prints the reference's thermo lines (its own
    Thermo, fed with the device state and tallies at each output step): step
    0, every 10 steps and the last step, equal to the reference's run."""
    import oracle as O
    pair = CASES[case][1]
    ours = O.read_thermo(app_log(tmp_path, case, THERMO + "run_b200 25\n"))
    exe = O.REF_EXE_EAMFIX if pair == "eam" else O.REF_EXE
    ref = O.read_thermo(reference_log(tmp_path, case, THERMO + "run 25\n", exe))
    assert list(ours[:, 0]) == [0, 10, 20, 25]
    assert_thermo_rows(ours, ref, O)


def test_run_b200_thermo_with_both_fixes(golden, tmp_path):
    import oracle as O
    g = golden("tiny_lj")
    fixes_b200 = lgv_fix(g) + dfm_fix(g)
    fixes_ref = fixes_b200.replace("langevin/b200", "langevin").replace("deform/b200", "deform")
    ours = O.read_thermo(app_log(tmp_path, "tiny_lj", fixes_b200 + THERMO + "run_b200 20\n"))
    ref = O.read_thermo(reference_log(tmp_path, "tiny_lj", fixes_ref + THERMO + "run 20\n", O.REF_EXE))
    assert list(ours[:, 0]) == [0, 10, 20]
    assert_thermo_rows(ours, ref, O)


# EAM FIRE on these systems does not converge (it ends with elements grown
# past the box, in the C restatement as on the device): EAM takes the
# fixed-iteration case only
@pytest.mark.parametrize("case,stop", [("tiny_lj", "ftol"), ("tiny_lj", "maxiter"), ("tiny_eam", "maxiter")])
def test_min_style_fire_b200_under_reference_minimize(case, stop, tmp_path):
    """min_style fire/b200 under the reference's own minimize command: the
    configuration it ends in is the device minimiser's run through the C ABI
    with the neighbour rule Min::init sets (every 1 delay 0 check yes), and
    the reference's Finish reports its stop reason and iteration count."""
    import oracle
    from cac_b200.api import Engine
    build, pair, _ = CASES[case]
    s = build()
    gen.write_data(s, str(tmp_path / "data.cac"))
    gen.write_setfl(gen.EamParams(), str(tmp_path / "cu.setfl"))
    ftol, maxiter = (1e-6, 3000) if stop == "ftol" else (0.0, 60)
    body = (f"min_style fire/b200\nmin_modify norm max\nminimize 0.0 {ftol} {maxiter} 100000\n"
            "oracle_dump end.txt state\n")
    (tmp_path / "in.cac").write_text(HEADER + pair_lines(pair) + TAIL + body)
    r = subprocess.run([APP, "-in", "in.cac"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    d = oracle.read_dump(str(tmp_path / "end.txt"))
    e = Engine(0)
    e.upload(s)
    if pair == "lj":
        e.pair_lj(0.4093, 2.338, 5.5)
    else:
        e.pair_eam(str(tmp_path / "cu.setfl"))
    e.neighbor(1.0, 1)
    e.neighbor_modify(0, True)
    code, it, en, fn = e.minimize_fire(ftol=ftol, maxiter=maxiter, norm="max")
    x, _, nx, _ = e.state()
    e.close()
    assert code == (3 if stop == "ftol" else 0)
    reason = {3: "force tolerance", 0: "max iterations"}[code]
    assert f"Stopping criterion = {reason}" in r.stdout
    if stop == "maxiter":
        assert f"Iterations, force evaluations = {it} {it}" in r.stdout
        assert np.abs(d["x"] - x).max() < 1e-10
        assert np.abs(d["nodex"] - nx).max() < 1e-10
    else:
        # converged: the same minimum, the iteration count within 2 %
        got = int(r.stdout.split("Iterations, force evaluations = ")[1].split()[0])
        assert abs(got - it) <= max(2, it // 50)
        assert np.abs(d["x"] - x).max() < 1e-5
        assert np.abs(d["nodex"] - nx).max() < 1e-5


def test_run_b200_check_yes_follows_the_reference(oracle_mod, tmp_path):
    """neigh_modify every 1 delay 3 check yes on a hot system (rebuilds only
    after a move past half the skin; the same system rebuilds at least twice
    in test_gpu_neigh_rule): run_b200 with lj/cut/b200 ends in the state the
    reference executable's own `run` reaches with lj/cut on the same deck."""
    if not os.path.exists(oracle_mod.REF_EXE):
        pytest.fail("reference executable oracle/_ref/cac is missing: build it with make -C oracle reference")
    s = gen.tiny(seed=32, temperature=1500.0)
    gen.write_data(s, str(tmp_path / "data.cac"))
    tail = ("neighbor 1.0 bin\nneigh_modify every 1 delay 3 check yes\ntimestep 0.001\nfix 1 all nve\n"
            "thermo 50\n")
    ends = []
    for exe, style, run in ((APP, "lj/cut/b200", "run_b200"), (oracle_mod.REF_EXE, "lj/cut", "run")):
        (tmp_path / "in.cac").write_text(HEADER + f"pair_style {style} 5.5\npair_coeff 1 1 0.4093 2.338\n" + tail +
                                         f"{run} 150\noracle_dump end.txt state\n")
        r = subprocess.run([exe, "-in", "in.cac"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
        ends.append((oracle_mod.read_dump(str(tmp_path / "end.txt")), r.stdout))
    (d, out), (ref, ref_out) = ends
    assert np.abs(d["x"] - ref["x"]).max() < 1e-10
    assert np.abs(d["nodex"] - ref["nodex"]).max() < 1e-10
    assert rel_err(d["v"], ref["v"]) < TOL
    assert rel_err(d["nodev"], ref["nodev"]) < TOL


def test_verlet_b200_thermo_every_step_copies_no_state(tmp_path):
    """run_style verlet/b200 with `thermo 1`: every step's thermo line comes
    from the device read-out (compute temp/b200 in place of thermo_temp, the
    pair's global tallies), equal to the reference's own run, and the device
    run copies no per-site state to the host for them."""
    import oracle as O
    deck = THERMO.replace("thermo 10", "thermo 1")
    out = app_log(tmp_path, "tiny_eam", deck + "run_style verlet/b200\nrun 25\n")
    ours = O.read_thermo(out)
    ref = O.read_thermo(reference_log(tmp_path, "tiny_eam", deck + "run 25\n", O.REF_EXE_EAMFIX))
    assert list(ours[:, 0]) == list(range(26))
    assert_thermo_rows(ours, ref, O)
    assert "b200 device run: 25 steps, 0 output steps with a host copy of the state" in out


def read_dump_frames(path):
    """Numeric rows of a dump custom file (ITEM: ATOMS section), sorted by
    their columns."""
    rows, on = [], False
    with open(path) as f:
        for ln in f:
            if ln.startswith("ITEM:"):
                on = ln.startswith("ITEM: ATOMS")
                continue
            if on and ln.strip():
                rows.append([float(t) for t in ln.split()])
    a = np.array(rows)
    return a[np.lexsort(a.T[::-1])]


@pytest.mark.parametrize("case", ["tiny_lj", "tiny_eam"])
def test_verlet_b200_dumps_with_device_peratom_computes(case, tmp_path):
    """A deck with per-site computes and a dump every 10 steps, run by the
    reference's `run` under run_style verlet/b200 with compute pe/atom/b200
    and stress/atom/b200: the dump files equal the reference's own run with
    compute pe/atom and stress/atom at the dump's print precision, and the
    device run copies the state only at the two dump steps inside it.  The
    reference side runs cac_eamfix for both pair styles: the stock
    ComputePEAtom never returns on a system with elements (its clear loop of
    node_energy reuses the inner loop's variable in the outer loop,
    compute_pe_atom.cpp:130) and folds only node 0 of ghost elements into
    their owners (:235, :254); that executable carries the fixes."""
    import oracle as O
    dump = ("dump 1 all custom 10 d.* id type x y z fx fy fz c_pa c_sa[1] c_sa[2] c_sa[3] c_sa[4] "
            "c_sa[5] c_sa[6]\n")
    ours_deck = ("compute pa all pe/atom/b200\ncompute sa all stress/atom/b200 NULL\n" + dump + THERMO +
                 "run_style verlet/b200\nrun 20\n")
    ref_deck = "compute pa all pe/atom\ncompute sa all stress/atom NULL\n" + dump + THERMO + "run 20\n"
    out = app_log(tmp_path, case, ours_deck)
    reference_log(tmp_path, case, ref_deck, O.REF_EXE_EAMFIX)
    assert "b200 device run: 20 steps, 2 output steps with a host copy of the state" in out
    for step in (0, 10, 20):
        a = read_dump_frames(str(tmp_path / f"d.{step}"))
        b = read_dump_frames(str(tmp_path / "ref" / f"d.{step}"))
        assert a.shape == b.shape and a.shape[0] > 0
        assert np.array_equal(a[:, :2], b[:, :2])
        for c in range(2, a.shape[1]):
            scale = max(np.abs(b[:, c]).max(), 1e-30)
            assert np.abs(a[:, c] - b[:, c]).max() <= 1e-5 * scale, (step, c)


@pytest.mark.parametrize("case", ["tiny_lj", "tiny_eam"])
def test_reference_neighbor_debug_dump_reads_the_device_list(case, tmp_path):
    """The reference's own write_dump_neighbor_debug with a /b200 pair style:
    its list is served by NPair half/bin/newton/b200, which outside a run
    fills the host list from the device's half list.  The whole-list dump
    (per site: coordinates, tag, neighbour count) equals the reference's own
    file, and one atom's and one Gauss point's neighbours (coordinates, tag,
    lattice site) equal the reference's as sets.  Both sides run the
    command with its three defects fixed (cac_eamfix, and the same objects in
    the harness): the stock code reads an unset element index in its header
    and gauss form, and leaves a deleted atom map in use after the atom form
    (write_dump_neighbor_debug.cpp:48, 220, 302), so its third call crashes."""
    import oracle as O
    body = ("write_dump_neighbor_debug nb\nwrite_dump_neighbor_debug na atom 5\n"
            "write_dump_neighbor_debug ng gauss 3 0 2\n")
    app_log(tmp_path, case, body)
    reference_log(tmp_path, case, body, O.REF_EXE_EAMFIX)
    with open(tmp_path / "nb_proc_0.dat") as f1, open(tmp_path / "ref" / "nb_proc_0.dat") as f2:
        assert f1.read() == f2.read()
    for name in ("na_proc_0", "ng_proc_0"):
        with open(tmp_path / name) as f1, open(tmp_path / "ref" / name) as f2:
            a, b = f1.read().splitlines(), f2.read().splitlines()
        head = next(k for k, ln in enumerate(b) if ln.startswith("ITEM: ATOMS")) + 2
        assert a[:head] == b[:head]
        assert len(a) == len(b) and len(a) > head + 10
        assert sorted(" ".join(ln.split()[1:]) for ln in a[head:]) == \
            sorted(" ".join(ln.split()[1:]) for ln in b[head:])
