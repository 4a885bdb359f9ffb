"""neigh_modify delay / check on the device (cacb200_set_neighbor_modify),
the rule of Neighbor::decide (neighbor.cpp:1584-1683)."""
import numpy as np
import pytest

from cac_b200 import gen
from helpers import LJ, SKIN

pytestmark = pytest.mark.gpu


def engine(system, every, delay=0, check=False, profile=True):
    from cac_b200.api import Engine
    e = Engine(0)
    e.upload(system)
    e.pair_lj(*LJ)
    e.neighbor(SKIN, every)
    e.neighbor_modify(delay, check)
    if profile:
        e.profile(True)
    return e


def builds(e):
    return e.profile_read().get("build_atoms", (0.0, 0))[1]


def test_delay_moves_rebuilds_to_its_multiples():
    """every 1 delay 5 rebuilds on the steps every 5 delay 0 does: the same
    trajectory bit for bit (graph replay of the latter included)."""
    s = gen.tiny(seed=31, temperature=600.0)
    out = []
    for every, delay, prof in ((1, 5, True), (5, 0, False)):
        e = engine(s, every, delay, profile=prof)
        e.setup()
        e.run_nve(40)
        out.append((e.state(), builds(e) if prof else None))
        e.close()
    (a, nb), (b, _) = out
    for u, w in zip(a, b):
        assert np.array_equal(u, w)
    assert nb == 1 + 40 // 5


def test_check_yes_rebuilds_only_after_a_move_past_half_the_skin():
    """every 1 check yes on a hot system: fewer builds than every 1 check no,
    at least one after the first, and the same trajectory within round-off
    (the lists differ only in entries beyond the cutoff and their order)."""
    s = gen.tiny(seed=32, temperature=1500.0)
    out = []
    for check in (True, False):
        e = engine(s, 1, 0, check)
        e.setup()
        e.run_nve(150)
        out.append((e.state(), builds(e)))
        e.close()
    ((x1, v1, nx1, nv1), b1), ((x0, v0, nx0, nv0), b0) = out
    assert b0 == 151
    assert 2 <= b1 < b0
    assert np.abs(x1 - x0).max() < 1e-9
    assert np.abs(nx1 - nx0).max() < 1e-9
    assert np.abs(v1 - v0).max() < 1e-9 * max(1.0, np.abs(v0).max())


def test_neighbor_modify_arguments():
    from cac_b200.api import CacB200Error
    s = gen.tiny(seed=33, temperature=10.0)
    e = engine(s, 1, profile=False)
    with pytest.raises(CacB200Error):
        e.neighbor_modify(-1, False)
    e.close()
