"""The spatial decomposition of one system over ranks (cac_b200.halo) on the
CPU: two and three gloo ranks, each evaluating its slab plus ghosts with the C
restatement standing in for the rank's GPU context, against the
restatement's own run of the whole periodic system.  The decomposition is
what is under test here (ownership, ghost shells, the forward halo of
positions, migration at every rebuild); the same run on the device is in
test_gpu_halo.py.  Tolerance: the FP64 bar, 1e-10 relative."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LJ = (0.4093, 2.338, 5.5)
TOL = 1e-10
NSTEPS = 20


class OracleBackend:
    """A rank's evaluation by the C restatement (test stand-in for
    halo.EngineBackend): the list is built at each upload (a rebuild) and kept
    until the next, as the device keeps its lists."""

    def __init__(self, pair, setfl=None, skin=1.0):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        self.O = oracle
        self.pair, self.skin = pair, skin
        self.eam = oracle.Eam(setfl) if pair == "eam" else None
        self.cutneigh = (LJ[2] if pair == "lj" else self.eam.cut) + skin
        self.st = None
        self.L = None

    def upload(self, boxlo, boxhi, x, v, nodex, nodev, mass):
        from cac_b200.gen import System
        if self.L is not None:
            self.O.free_list(self.L)
        self.st = self.O.OracleState(System(x=x, v=v, nodex=nodex, nodev=nodev, boxlo=np.asarray(boxlo),
                                            boxhi=np.asarray(boxhi), mass=mass))
        self.L = self.O.build_list(self.st, self.cutneigh, True)

    def forces(self):
        if self.pair == "lj":
            self.O.lj_forces(self.st, self.L, *LJ)
        else:
            self.O.eam_forces(self.st, self.L, self.eam)

    def nve_initial(self, dt):
        self.O.lib().oracle_nve_initial(self.st.ref, dt)

    def nve_final(self, dt):
        self.O.lib().oracle_nve_final(self.st.ref, dt)

    def positions(self):
        return self.st.x.copy(), self.st.nodex.copy()

    def set_positions(self, x, nodex):
        self.st.x[...] = x
        self.st.nodex[...] = nodex

    def state(self):
        s = self.st
        return s.x.copy(), s.v.copy(), s.nodex.copy(), s.nodev.copy(), s.f.copy(), s.nodef.copy()


def system():
    sys.path.insert(0, ROOT)
    from cac_b200 import gen
    return gen.build_slab(3, 1, 2, 12, temperature=300.0, seed=21, strain=0.01)


def _worker(rank, ws, port, pair, setfl, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from cac_b200 import halo
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=120))
    try:
        b = OracleBackend(pair, setfl)
        run = halo.HaloRun(halo.TorchComm(dist), b, system(), b.cutneigh, every=10,
                           hops=1 if pair == "lj" else 2)
        nown = (len(run.parts[rank].own_atoms), len(run.parts[rank].own_elems),
                len(run.parts[rank].ghost_atoms), len(run.parts[rank].ghost_elems))
        run.run(NSTEPS, 0.001)
        x, v, nx, nv, f, nf = run.gather()
        out.put((rank, nown, x, v, nx, nv, f, nf))
    finally:
        dist.destroy_process_group()


def reference(pair, setfl):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    st = oracle.OracleState(system())
    if pair == "lj":
        oracle.run_nve(st, "lj", lj=LJ, skin=1.0, nsteps=NSTEPS, every=10)
    else:
        oracle.run_nve(st, "eam", eam=oracle.Eam(setfl), skin=1.0, nsteps=NSTEPS, every=10)
    return st


def rel(a, b):
    a = np.asarray(a).reshape(-1, 3)
    b = np.asarray(b).reshape(-1, 3)
    return float(np.linalg.norm(a - b, axis=1).max() / np.linalg.norm(b, axis=1).max())


def wrapped_diff(a, b, L):
    d = (np.asarray(a) - np.asarray(b)).reshape(-1, 3)
    d -= np.round(d / L) * L
    return float(np.abs(d).max())


@pytest.mark.parametrize("pair,ws", [("lj", 2), ("eam", 2), ("lj", 3)])
def test_gloo_ranks_equal_one_system(pair, ws, tmp_path):
    import socket
    import torch.multiprocessing as mp
    sys.path.insert(0, ROOT)
    from cac_b200 import gen
    setfl = str(tmp_path / "cu.setfl")
    gen.write_setfl(gen.EamParams(), setfl)
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, pair, setfl, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=600) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    s = system()
    ref = reference(pair, setfl)
    L = np.asarray(s.boxhi) - np.asarray(s.boxlo)
    # every rank owns sites (three slabs: the outer ones hold only elements)
    # and ghosts, and gathers the same global state
    for (_, nown, *_a) in res:
        assert nown[0] + nown[1] > 0 and nown[2] + nown[3] > 0
    assert sum(r[1][0] for r in res) == s.natoms and sum(r[1][1] for r in res) == s.nelements
    for other in res[1:]:
        for k in range(2, 8):
            assert np.array_equal(res[0][k], other[k])
    _, _, x, v, nx, nv, f, nf = res[0]
    assert wrapped_diff(x, ref.x, L) < 1e-10
    assert wrapped_diff(nx, ref.nodex, L) < 1e-10
    assert rel(v, ref.v) < TOL
    assert rel(nv, ref.nodev) < TOL
    assert rel(f, ref.f) < TOL
    assert rel(nf, ref.nodef) < TOL


def test_slab_plan_owns_every_site_once():
    sys.path.insert(0, ROOT)
    from cac_b200 import halo
    s = system()
    x, nx = np.array(s.x), np.array(s.nodex)
    halo.wrap_atoms(x, s.boxlo, s.boxhi)
    halo.wrap_elements(nx, s.boxlo, s.boxhi)
    for n in (1, 2, 3):
        plan = halo.SlabPlan(s.boxlo, s.boxhi, n, 6.5, hops=2, margin=1.0)
        parts = plan.split(x, nx)
        own_a = np.sort(np.concatenate([p.own_atoms for p in parts]))
        own_e = np.sort(np.concatenate([p.own_elems for p in parts]))
        assert np.array_equal(own_a, np.arange(s.natoms))
        assert np.array_equal(own_e, np.arange(s.nelements))
        for p in parts:
            # no site is both owned and an unshifted ghost; ghosts lie in the rank's box
            assert not np.intersect1d(p.own_atoms, p.ghost_atoms[p.ghost_atom_shift == 0]).size
            a = plan.axis
            zg = x[p.ghost_atoms, a] + p.ghost_atom_shift * plan.L
            assert (zg > p.boxlo[a]).all() and (zg < p.boxhi[a]).all()
