"""Neighbour windows of the mixed form (cacb200_set_windows): the density and
force passes reading neighbours from a block's window in shared memory give
the forces, energies and trajectory of the direct gathers bit for bit (the
same integer separations and the same sums in the same order), over steps
with list rebuilds."""
import numpy as np
import pytest

from cac_b200 import gen
from helpers import SKIN, setfl_path

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("strain", [0.0, 0.03])
def test_windows_equal_direct_gathers(strain, tmp_path):
    from cac_b200.api import ENERGY_GLOBAL, MIXED, VIRIAL_GLOBAL, Engine
    s = gen.build_slab(4, 2, 2, 12, temperature=300.0, strain=strain, seed=17)
    out = []
    for on in (True, False):
        e = Engine(0)
        e.upload(s)
        e.pair_eam(setfl_path(tmp_path))
        e.set_precision(MIXED)
        e.neighbor(SKIN, 10)
        e.windows(on)
        e.setup()
        f0, nf0, _ = e.forces()
        e.run_nve(25, 0.001, eflag=ENERGY_GLOBAL, vflag=VIRIAL_GLOBAL)
        f, nf, gf = e.forces()
        ev = e.energy(peratom=False)
        x, v, nx, nv = e.state()
        out.append((f0, nf0, f, nf, gf, ev["energy"], ev["virial"], x, v, nx, nv))
        e.close()
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(np.asarray(a), np.asarray(b))
