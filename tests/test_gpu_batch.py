"""Batched replicas and graph-replayed NVE cycles.

A batch runs independent replicas (own boxes, sizes, temperatures, strains)
through the same kernels as a single system, so every replica's trajectory,
forces and energy must equal the same replica run alone: bit for bit for
positions, velocities and forces (the same per-site arithmetic in the same
order), and within 1e-12 relative for the per-replica energy (a different
summation order of the same terms).  Graph replay of the rebuild cycle must
equal eager stepping bit for bit."""
import numpy as np
import pytest

from cac_b200 import gen
from helpers import LJ, SKIN, setfl_path

pytestmark = pytest.mark.gpu

STEPS = 25   # two rebuild cycles and a partial one


def replicas():
    return [
        gen.replica(2000, 50, temperature=120.0, strain=0.0, seed=31),
        gen.replica(5000, 120, temperature=450.0, strain=0.04, seed=32),
        gen.replica(3000, 60, temperature=20.0, strain=0.02, seed=33),
    ]


def configure(e, pair, tmp_path, form):
    if pair == "lj":
        e.pair_lj(*LJ)
    else:
        e.pair_eam(setfl_path(tmp_path))
    e.neighbor(SKIN, 10)
    e.set_precision(form)


def run(e, steps):
    from cac_b200.api import ENERGY_ATOM, ENERGY_GLOBAL
    e.setup()
    e.run_nve(steps, 0.001)
    x, v, nx, nv = e.state()
    f, nf, gf = e.forces()
    e.compute(ENERGY_GLOBAL | ENERGY_ATOM, 0)
    return x, v, nx, nv, f, nf, gf


@pytest.mark.parametrize("pair,form", [("lj", 0), ("eam", 0), ("eam", 1)])
def test_batch_equals_alone(pair, form, tmp_path):
    from cac_b200.api import Engine
    reps = replicas()
    b = Engine(0)
    b.upload_batch(reps)
    configure(b, pair, tmp_path, form)
    got = run(b, STEPS)
    e_batch = b.replica_energy()
    assert b.graph_launches() > 0
    a_off = np.concatenate([[0], np.cumsum([r.natoms for r in reps])])
    e_off = np.concatenate([[0], np.cumsum([r.nelements for r in reps])])
    for k, s in enumerate(reps):
        a = Engine(0)
        a.upload(s)
        configure(a, pair, tmp_path, form)
        want = run(a, STEPS)
        e_alone = a.energy(peratom=False)["energy"]
        sl_a = slice(a_off[k], a_off[k + 1])
        sl_e = slice(e_off[k], e_off[k + 1])
        for g, w, per_atom in zip(got, want, (1, 1, 0, 0, 1, 0, 0)):
            part = g[sl_a] if per_atom else g[sl_e]
            assert np.array_equal(part, w), f"replica {k} differs from its run alone"
        assert abs(e_batch[k] - e_alone) <= 1e-12 * abs(e_alone), (k, e_batch[k], e_alone)
        a.close()
    b.close()


@pytest.mark.parametrize("pair", ["lj", "eam"])
def test_graph_cycles_equal_eager(pair, tmp_path):
    from cac_b200.api import Engine
    s = gen.lj_small(seed=1) if pair == "lj" else gen.build_slab(4, 2, 3, 9, temperature=300.0, seed=21)
    out = []
    for graphs in (True, False):
        e = Engine(0)
        e.upload(s)
        configure(e, pair, tmp_path, 0)
        e.graphs(graphs)
        e.setup()
        e.run_nve(STEPS, 0.001)
        out.append((e.state(), e.forces(), e.graph_launches()))
        e.close()
    (s1, f1, n1), (s2, f2, n2) = out
    assert n1 > 0 and n2 == 0
    for a, b in zip(s1 + f1, s2 + f2):
        assert np.array_equal(a, b)


def test_batch_rejects_half_lists(tmp_path):
    from cac_b200.api import CacB200Error, Engine
    b = Engine(0)
    b.upload_batch(replicas()[:2])
    configure(b, "lj", tmp_path, 0)
    with pytest.raises(CacB200Error):
        b.build_lists(half=True)
    b.close()


def test_work_queue_launches_equal_grid_launches(tmp_path):
    """Mixed-form batches run the EAM passes as persistent work-queue
    launches with per-size-class tiles; the forces equal those of the grid
    launches bit for bit (every slot's arithmetic is the same), over steps
    with a rebuild and after the tiles were tuned."""
    from cac_b200.api import MIXED, Engine
    reps = gen.replica_set(12, seed=31, atoms=(600, 40000), elements=(20, 900))
    out = []
    for on in (True, False):
        e = Engine(0)
        e.upload_batch(reps)
        e.pair_eam(setfl_path(tmp_path))
        e.set_precision(MIXED)
        e.neighbor(1.0, 10)
        tiles = e.work_queue(on)
        e.setup()
        e.run_nve(12, 0.001)
        f, nf, gf = e.forces()
        x = e.state()[0]
        tiles = e.work_queue()
        out.append((f, gf, x, tiles))
        e.close()
    (f1, g1, x1, t1), (f0, g0, x0, t0) = out
    assert all(t in (128, 512, 2048) for t in t1 if t)
    assert any(t1)
    assert np.array_equal(f1, f0) and np.array_equal(g1, g0) and np.array_equal(x1, x0)


@pytest.mark.parametrize("form,strain", [(0, 0.0), (1, 0.0), (1, 0.03)])
def test_sm_local_runs_equal_grid_launches(form, strain, tmp_path):
    """A single system runs the atom-list build, and in the FP64 form the
    force-only EAM passes, over SM-local runs of cells and list slots (work
    queue on, the default); the lists, forces and trajectory equal those of
    the grid launches (work queue off) bit for bit, over steps with rebuilds
    (FP64 and mixed)."""
    from cac_b200.api import Engine
    s = gen.build_slab(6, 3, 8, 24, temperature=300.0, strain=strain, seed=14)
    out = []
    for on in (True, False):
        e = Engine(0)
        e.upload(s)
        e.pair_eam(setfl_path(tmp_path))
        e.set_precision(form)
        e.neighbor(1.0, 10)
        e.work_queue(on)
        e.setup()
        e.run_nve(25, 0.001)
        f, nf, gf = e.forces()
        x, v, nx, nv = e.state()
        e.build_lists()
        lst = e.neighbor_list()
        out.append((f, nf, gf, x, v, nx, nv, lst))
        e.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)
