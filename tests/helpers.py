"""Shared helpers for the tests: canonical list digests, force-error norms and
the seeded systems of the golden fixtures."""
import hashlib

import numpy as np

from cac_b200 import gen

LJ = (0.4093, 2.338, 5.5)
SKIN = 1.0

# golden case -> (system builder, pair, neighbour cutoff)
CASES = {
    "tiny_lj": (lambda: gen.tiny(seed=7, temperature=50.0), "lj", 6.5),
    "tiny_eam": (lambda: gen.tiny(seed=11, temperature=300.0), "eam", 6.0),
    "lj_small": (lambda: gen.lj_small(seed=1), "lj", 6.5),
}

# Gauss point g of an element sits on node G2N[g]; dumps list nodes in node order
G2N = np.array([0, 4, 3, 7, 1, 5, 2, 6])
N2G = np.argsort(G2N)


def digest(rows: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(rows, dtype="<i8").tobytes()).hexdigest()


def counts(rows: np.ndarray, nsites: int) -> np.ndarray:
    return np.bincount(rows[:, 0], minlength=nsites).astype(np.int32)


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    """max_i |a_i - b_i| / max_i |b_i| over whole vectors (per-site norms)."""
    a = np.asarray(a, dtype=np.float64).reshape(-1, 3) if np.asarray(a).size % 3 == 0 else np.asarray(a).reshape(-1, 1)
    b = np.asarray(b, dtype=np.float64).reshape(a.shape)
    scale = np.linalg.norm(b, axis=1).max()
    return float(np.linalg.norm(a - b, axis=1).max() / scale) if scale > 0 else float(np.abs(a - b).max())


def setfl_path(tmpdir) -> str:
    import os
    p = os.path.join(str(tmpdir), "cu.setfl")
    if not os.path.exists(p):
        gen.write_setfl(gen.EamParams(), p)
    return p
