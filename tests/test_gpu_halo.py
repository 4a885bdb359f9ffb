"""The spatial decomposition of one system (cac_b200.halo) with a device
context per rank: two and three ranks driven from one process (LocalComm;
their kernels run one rank after another, none waits on another), each
holding its slab plus ghosts, against one context running the whole
periodic system (cacb200_run_nve with a rebuild every 10 steps).  The
two-rank run over torch.distributed is covered on the CPU by
test_halo.py.  Tolerance: the FP64 bar, 1e-10 relative."""
import numpy as np
import pytest

from cac_b200 import gen, halo
from helpers import LJ, SKIN, rel_err, setfl_path

pytestmark = pytest.mark.gpu

TOL = 1e-10
NSTEPS = 20


def system():
    return gen.build_slab(3, 1, 2, 12, temperature=300.0, seed=21, strain=0.01)


@pytest.mark.parametrize("pair", ["lj", "eam"])
@pytest.mark.parametrize("nranks", [2, 3])
def test_device_ranks_equal_one_context(pair, nranks, tmp_path):
    from cac_b200.api import Engine
    s = system()
    setfl = setfl_path(tmp_path)
    cutneigh = (LJ[2] if pair == "lj" else 5.0) + SKIN
    backends = [halo.EngineBackend(0, pair, setfl, LJ, SKIN) for _ in range(nranks)]
    run = halo.HaloRun(halo.LocalComm(nranks), backends, s, cutneigh, every=10, hops=1 if pair == "lj" else 2)
    run.run(NSTEPS, 0.001)
    x, v, nx, nv, f, nf = run.gather()
    for b in backends:
        b.close()
    e = Engine(0)
    e.upload(s)
    if pair == "lj":
        e.pair_lj(*LJ)
    else:
        e.pair_eam(setfl)
    e.neighbor(SKIN, 10)
    e.setup()
    e.run_nve(NSTEPS, 0.001)
    rx, rv, rnx, rnv = e.state()
    rf, rnf, _ = e.forces()
    e.close()
    L = np.asarray(s.boxhi) - np.asarray(s.boxlo)
    for a, b in ((x, rx), (nx, rnx)):
        d = (a - b).reshape(-1, 3)
        d -= np.round(d / L) * L
        assert np.abs(d).max() < 1e-10
    assert rel_err(v, rv) < TOL
    assert rel_err(nv, rnv) < TOL
    assert rel_err(f, rf) < TOL
    assert rel_err(nf, rnf) < TOL
