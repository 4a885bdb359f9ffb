"""The inner prefix of the neighbour lists (cacb200_set_list_prefix): entries
within the cutoff plus a margin at the build come first, and a site's pair
loop stops after them while its own displacement since the build plus the
largest one cannot close the margin.

* Same state, same lists: forces with the prefix and with the whole lists
  are equal bit for bit (the prefix is walked on its own either way).
* A hot system whose atoms outrun half the margin within a rebuild cycle:
  the drift's displacements switch sites to their whole lists, and the
  trajectory follows the one with the prefix off to rounding (1e-9 A after
  20 steps; a neighbour missed near the cutoff would move atoms ~1e-4 A)."""
import numpy as np
import pytest

from cac_b200 import gen
from helpers import LJ, SKIN, rel_err, setfl_path

pytestmark = pytest.mark.gpu


def make(system, pair, tmp_path, margin, form=0):
    from cac_b200.api import Engine
    e = Engine(0)
    e.upload(system)
    e.pair_lj(*LJ) if pair == "lj" else e.pair_eam(setfl_path(tmp_path))
    e.neighbor(SKIN, 10)
    e.set_precision(form)
    e.list_prefix(margin)
    return e


@pytest.mark.parametrize("pair,form", [("lj", 0), ("eam", 0), ("eam", 1)])
def test_prefix_and_whole_lists_equal_at_one_state(pair, form, tmp_path):
    s = gen.replica(3000, 60, temperature=300.0, strain=0.01, seed=91)
    e = make(s, pair, tmp_path, -1.0, form)
    e.setup()
    e.compute(0, 0)
    f1, nf1, gf1 = e.forces()
    x, v, nx, nv = e.state()
    x2 = x.copy()
    x2[0, 0] = np.nextafter(x2[0, 0], 1e9)
    e.set_state(x2, v, nx, nv)      # moved: the whole lists from now on ...
    e.set_state(x, v, nx, nv)       # ... at the same positions
    e.compute(0, 0)
    f2, nf2, gf2 = e.forces()
    e.close()
    assert np.array_equal(f1, f2) and np.array_equal(nf1, nf2) and np.array_equal(gf1, gf2)


@pytest.mark.parametrize("pair,form,tol,temp", [("lj", 0, 1e-9, 3000.0), ("eam", 0, 1e-9, 3000.0),
                                                ("eam", 1, 1e-5, 3000.0), ("eam", 0, 1e-9, 900.0),
                                                ("lj", 0, 1e-9, 1500.0)])
def test_hot_system_switches_to_whole_lists(pair, form, tol, temp, tmp_path):
    """(mixed form: FP32 sums in another order differ by FP32 rounding.)
    At 900 K and 1500 K the fastest sites pass half the margin while most
    do not: each site's own displacement decides whether it walks its whole
    list, and the trajectory still follows the prefix-off one."""
    s = gen.replica(3000, 60, temperature=temp, strain=0.0, seed=92)
    out = []
    for margin in (-1.0, 0.0):
        e = make(s, pair, tmp_path, margin, form)
        e.setup()
        e.run_nve(20, 0.002)
        out.append(e.state())
        e.close()
    (x1, v1, nx1, nv1), (x2, v2, nx2, nv2) = out
    assert np.abs(x1 - x2).max() < tol
    assert np.abs(nx1 - nx2).max() < tol
    assert rel_err(v1, v2) < tol
