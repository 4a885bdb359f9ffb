"""Data files in the reference's read_data format, host side (no device):
what the generator writes for the reference is read back exactly, written
again and read back exactly, and malformed files are refused with a message."""
import os

import numpy as np
import pytest

from cac_b200 import api, gen


def test_generator_file_reads_back_exactly(tmp_path):
    s = gen.tiny(seed=9, temperature=120.0)
    p = os.path.join(str(tmp_path), "in.data")
    gen.write_data(s, p)
    r = api.read_data_file(p)
    assert (r.natoms, r.nelements) == (s.natoms, s.nelements)
    assert np.array_equal(r.boxlo, s.boxlo) and np.array_equal(r.boxhi, s.boxhi)
    assert r.mass == s.mass
    for a, b in ((r.x, s.x), (r.v, s.v), (r.nodex, s.nodex), (r.nodev, s.nodev)):
        assert np.array_equal(a, b)


def test_write_then_read_round_trip(tmp_path):
    s = gen.replica(2000, 40, temperature=300.0, strain=0.02, seed=4)
    p = os.path.join(str(tmp_path), "out.data")
    api.write_data_file(p, s)
    r = api.read_data_file(p)
    for a, b in ((r.x, s.x), (r.v, s.v), (r.nodex, s.nodex), (r.nodev, s.nodev)):
        assert np.array_equal(a, b)


def test_malformed_files_are_refused(tmp_path):
    s = gen.tiny()
    p = os.path.join(str(tmp_path), "bad.data")
    gen.write_data(s, p)
    text = open(p).read()
    cases = {
        "2 atom types": text.replace("1 atom types", "2 atom types"),
        "element type": text.replace("1 Hex 1 9 9 9 2 2 2", "1 Hex 1 5 5 5 2 2 2"),
        "tag out of range": text.replace("\n1 1 ", f"\n{s.natoms + 5} 1 ", 1),
    }
    for what, body in cases.items():
        with open(p, "w") as f:
            f.write(body)
        with pytest.raises(api.CacB200Error):
            api.read_data_file(p)
    with pytest.raises(api.CacB200Error):
        api.read_data_file(os.path.join(str(tmp_path), "missing.data"))
