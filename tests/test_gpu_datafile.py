"""Data files through a context: a file read with cacb200_read_data gives the
same forces as the same system uploaded from arrays (bit for bit), and the
state written with cacb200_write_data after some steps reads back exactly."""
import os

import numpy as np
import pytest

from cac_b200 import api, gen
from helpers import LJ, SKIN

pytestmark = pytest.mark.gpu


def test_read_data_equals_upload_and_write_data_round_trips(tmp_path):
    s = gen.tiny(seed=12, temperature=80.0)
    p = os.path.join(str(tmp_path), "in.data")
    gen.write_data(s, p)
    out = []
    for via_file in (True, False):
        e = api.Engine(0)
        if via_file:
            e.read_data(p)
        else:
            e.upload(s)
        e.pair_lj(*LJ)
        e.neighbor(SKIN, 10)
        e.compute()
        out.append(e.forces())
        if via_file:
            e.setup()
            e.run_nve(15, 0.001)
            q = os.path.join(str(tmp_path), "out.data")
            e.write_data(q)
            r = api.read_data_file(q)
            for a, b in zip((r.x, r.v, r.nodex, r.nodev), e.state()):
                assert np.array_equal(a, b)
        e.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)
