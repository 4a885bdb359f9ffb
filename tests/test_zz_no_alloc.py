"""The allocation-free per-replica energy against the context's own.

cacb200_replica_energy_noalloc serves callers that may not allocate device
memory (their GPU memory belongs to another framework's pool, or a cudaFree
would stall other running streams); it keeps its scratch in one fixed device
array of the library.  Here it must give the per-replica energies that
cacb200_replica_energy gives for the same per-site energies, within 1e-12
relative (the same terms in the same order), on two calls in a row (the
second call reuses the scratch the first one left behind).  The test calls
the C ABI directly with device pointers held by torch tensors; this file is
collected last so that a stop at its first failure comes after every other
test has run."""
import ctypes as C

import numpy as np
import pytest

from cac_b200 import gen
from helpers import LJ, SKIN

pytestmark = pytest.mark.gpu

NODE_WEIGHT = 729.0 / 8.0   # UNIFORM node weight of the 9x9x9 Hex element


def test_noalloc_energy_matches_context_energy():
    import torch
    from cac_b200.api import ENERGY_ATOM, ENERGY_GLOBAL, VIRIAL_ATOM, VIRIAL_GLOBAL, Engine

    reps = [gen.replica(2000, 40, temperature=150.0, strain=0.0, seed=201),
            gen.replica(4000, 80, temperature=300.0, strain=0.03, seed=202),
            gen.replica(1500, 30, temperature=50.0, strain=0.01, seed=203)]
    b = Engine(0)
    b.upload_batch(reps)
    b.pair_lj(*LJ)
    b.neighbor(SKIN, 10)
    b.setup()
    b.run_nve(12, 0.001)
    b.compute(ENERGY_GLOBAL | ENERGY_ATOM, VIRIAL_GLOBAL | VIRIAL_ATOM)
    want = b.replica_energy()
    per_site = b.energy(peratom=True)
    eatom = torch.tensor(per_site["eatom"], dtype=torch.float64, device="cuda:0")
    enode = torch.tensor(per_site["enode"], dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()

    na = np.array([r.natoms for r in reps], dtype=np.int32)
    ne = np.array([r.nelements for r in reps], dtype=np.int32)
    ip = C.POINTER(C.c_int)
    lib = b.lib
    for call in range(2):
        got = np.zeros(len(reps))
        rc = lib.cacb200_replica_energy_noalloc(0, C.c_void_p(eatom.data_ptr()), C.c_void_p(enode.data_ptr()),
                                                len(reps), na.ctypes.data_as(ip), ne.ctypes.data_as(ip),
                                                NODE_WEIGHT, got.ctypes.data_as(C.POINTER(C.c_double)), None)
        assert rc == 0, f"call {call} failed ({rc})"
        assert np.all(np.abs(got - want) <= 1e-12 * np.abs(want)), (call, got, want)
    b.close()


def test_noalloc_rejects_more_replicas_than_its_scratch():
    from cac_b200.api import load
    lib = load()
    n = 4097
    counts = np.zeros(n, dtype=np.int32)
    out = np.zeros(n)
    ip = C.POINTER(C.c_int)
    rc = lib.cacb200_replica_energy_noalloc(0, None, None, n, counts.ctypes.data_as(ip), counts.ctypes.data_as(ip),
                                            1.0, out.ctypes.data_as(C.POINTER(C.c_double)), None)
    assert rc != 0
    lib.cacb200_noalloc_last_error.restype = C.c_char_p
    assert b"4097 replicas" in lib.cacb200_noalloc_last_error()
