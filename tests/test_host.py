"""Host-side checks that need no GPU: the C ABI library and its exports, the
Python bindings, the generator and the setfl reader."""
import ctypes
import os
import re

import numpy as np
import pytest

from cac_b200 import api, build, gen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "cacb200.h")).read()
    return sorted(set(re.findall(r"\b(cacb200_[a-z0-9_]+)\s*\(", text)))


def test_library_builds_and_exports_every_declared_symbol():
    lib = api.load()
    names = header_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n


def test_bindings_cover_the_header():
    bound = {s[0] for s in api.SIGNATURES}
    assert bound == set(header_functions())


def test_no_gpu_means_loud_failure():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(api.CacB200Error):
        api.Engine(0)


@pytest.mark.parametrize("builder,na,ne", [
    (lambda: gen.tiny(), 1458, 12),
    (lambda: gen.lj_small(), 4374, 216),
])
def test_generator_counts_and_no_overlaps(builder, na, ne):
    s = builder()
    assert (s.natoms, s.nelements) == (na, ne)
    L = s.boxhi - s.boxlo
    assert np.all(s.x >= s.boxlo) and np.all(s.x < s.boxhi)
    c = s.centers()
    assert np.all(c >= s.boxlo) and np.all(c < s.boxhi)
    # all lattice sites (atoms + every element site) are distinct: min image distance > 2 A
    shape = np.zeros((gen.NUCELL, 8))
    for u in range(gen.NUCELL):
        i, j, k = u // 81, (u // 9) % 9, u % 9
        px, py, pz = 0.25 * i - 1, 0.25 * j - 1, 0.25 * k - 1
        for n, (a, b, cc) in enumerate(gen.HEX_CORNERS // 8):
            shape[u, n] = 0.125 * (1 + (2 * a - 1) * px) * (1 + (2 * b - 1) * py) * (1 + (2 * cc - 1) * pz)
    sites = np.einsum("un,end->eud", shape, s.nodex).reshape(-1, 3)
    pts = np.concatenate([s.x, sites])
    assert pts.shape[0] == na + ne * 729
    # grid-hash check of nearest neighbours
    cell = 2.0
    keys = np.floor((pts - s.boxlo) / cell).astype(np.int64)
    order = np.lexsort(keys.T[::-1])
    p = pts[order]
    d = np.diff(p, axis=0)
    d -= np.round(d / L) * L
    assert np.linalg.norm(d, axis=1).min() > 0.5


def test_setfl_roundtrip(tmp_path):
    p = str(tmp_path / "cu.setfl")
    prm = gen.EamParams()
    gen.write_setfl(prm, p)
    t = api.read_setfl(p)
    frho, rhor, z2r = prm.tables()
    assert t["nrho"] == prm.nrho and t["nr"] == prm.nr
    assert np.array_equal(t["frho"], frho)
    assert np.array_equal(t["rhor"], rhor)
    assert np.array_equal(t["z2r"], z2r)
    assert t["cut"] == prm.cut


def test_named_workload_sizes():
    """The scale workloads keep the counts their docstrings state (sizes only,
    without building the arrays)."""
    for fn, nx, ny, le, la, na, ne in [
        (gen.eam_1m, 8, 5, 125, 162, 1_049_760, 20_000),
        (gen.eam_4m_strained, 20, 10, 125, 129, 4_179_600, 100_000),
    ]:
        assert 162 * nx * ny * la == na
        assert 2 * 2 * nx * ny * le == ne


def _noalloc_call(lib, device, n, natoms, nelements, out, eatom=None, enode=None):
    ip = ctypes.POINTER(ctypes.c_int)
    return lib.cacb200_replica_energy_noalloc(
        device, eatom, enode, n, natoms.ctypes.data_as(ip) if natoms is not None else None,
        nelements.ctypes.data_as(ip) if nelements is not None else None, 1.0,
        out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if out is not None else None, None)


def test_noalloc_rejects_bad_arguments_before_any_device_work():
    """cacb200_replica_energy_noalloc checks its arguments before it touches a
    device (so these run without one): each bad argument returns
    CACB200_EINVAL with its own message in cacb200_noalloc_last_error."""
    lib = api.load()
    lib.cacb200_noalloc_last_error.restype = ctypes.c_char_p
    ok = np.zeros(4, dtype=np.int32)
    out = np.zeros(4)
    cases = [
        ((0, 4097, np.zeros(4097, np.int32), np.zeros(4097, np.int32), np.zeros(4097)), b"4097 replicas"),
        ((0, 0, ok, ok, out), b"0 replicas"),
        ((0, 4, None, ok, out), b"null count or output array"),
        ((0, 4, ok, ok, None), b"null count or output array"),
        ((-1, 4, ok, ok, out), b"device index out of range"),
        ((0, 4, np.array([1, -2, 0, 0], np.int32), ok, out), b"negative site count"),
        ((0, 4, np.array([1, 0, 0, 0], np.int32), ok, out), b"null per-site energy array"),
    ]
    for args, msg in cases:
        assert _noalloc_call(lib, *args) == -1, msg
        assert msg in lib.cacb200_noalloc_last_error(), (msg, lib.cacb200_noalloc_last_error())


def test_noalloc_error_message_is_per_thread():
    """The last-error message belongs to the calling thread: two threads that
    fail differently each read back their own message."""
    import threading
    lib = api.load()
    lib.cacb200_noalloc_last_error.restype = ctypes.c_char_p
    got = {}

    def worker(name, n, natoms, gate_in, gate_out):
        out = np.zeros(max(n, 1))
        zeros = np.zeros(max(n, 1), np.int32)
        _noalloc_call(lib, 0, n, natoms if natoms is not None else zeros, zeros, out)
        gate_out.set()
        gate_in.wait(10)
        got[name] = lib.cacb200_noalloc_last_error()

    a_done, b_done = threading.Event(), threading.Event()
    ta = threading.Thread(target=worker, args=("a", 5000, None, b_done, a_done))
    tb = threading.Thread(target=worker, args=("b", 2, np.array([3, -1], np.int32), a_done, b_done))
    ta.start()
    tb.start()
    ta.join(20)
    tb.join(20)
    assert b"5000 replicas" in got["a"]
    assert b"negative site count" in got["b"]
