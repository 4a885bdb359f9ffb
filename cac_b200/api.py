"""Python host layer over the C ABI of ``libcacb200.so`` (declared in
``include/cacb200.h``).

It mirrors the reference's style commands for the per-timestep path:

    pair_style lj/cut/b200 CUT ; pair_coeff 1 1 EPS SIGMA  -> Engine.pair_lj
    pair_style eam/alloy/b200 ; pair_coeff * * FILE El     -> Engine.pair_eam
    neighbor SKIN bin ; neigh_modify every N delay 0 check no -> Engine.neighbor
    fix ID all nve/b200 ; run N                            -> Engine.run_nve

There is no CPU fallback: without the library or a CUDA device every call
raises ``CacB200Error``.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from . import build as _build

ENERGY_GLOBAL = 1
ENERGY_ATOM = 2
VIRIAL_GLOBAL = 1
VIRIAL_ATOM = 4
FP64 = 0
MIXED = 1

_dp = C.POINTER(C.c_double)


class CacB200Error(RuntimeError):
    pass


_lib = None

# (name, restype, argtypes) of every entry point in include/cacb200.h
SIGNATURES = [
    ("cacb200_ctx_create", C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    ("cacb200_ctx_destroy", C.c_int, [C.c_void_p]),
    ("cacb200_last_error", C.c_char_p, [C.c_void_p]),
    ("cacb200_stream", C.c_void_p, [C.c_void_p]),
    ("cacb200_set_precision", C.c_int, [C.c_void_p, C.c_int]),
    ("cacb200_upload_system", C.c_int, [C.c_void_p, _dp, _dp, C.c_int, _dp, _dp, C.c_int, _dp, _dp, C.c_double]),
    ("cacb200_get_box", C.c_int, [C.c_void_p, _dp, _dp, _dp]),
    ("cacb200_set_box", C.c_int, [C.c_void_p, _dp, _dp]),
    ("cacb200_data_last_error", C.c_char_p, []),
    ("cacb200_data_counts", C.c_int, [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), _dp, _dp, _dp]),
    ("cacb200_data_read", C.c_int, [C.c_char_p, _dp, _dp, _dp, _dp]),
    ("cacb200_data_write", C.c_int, [C.c_char_p, C.c_int, C.c_int, _dp, _dp, C.c_double, _dp, _dp, _dp, _dp]),
    ("cacb200_read_data", C.c_int, [C.c_void_p, C.c_char_p]),
    ("cacb200_write_data", C.c_int, [C.c_void_p, C.c_char_p]),
    ("cacb200_upload_batch", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), _dp, _dp,
                                       _dp, _dp, _dp, _dp, C.c_double]),
    ("cacb200_replica_energy", C.c_int, [C.c_void_p, _dp]),
    ("cacb200_thermo", C.c_int, [C.c_void_p, C.c_int, _dp]),
    ("cacb200_set_langevin", C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int]),
    ("cacb200_set_langevin_stream", C.c_int, [C.c_void_p, C.c_longlong]),
    ("cacb200_unset_langevin", C.c_int, [C.c_void_p]),
    ("cacb200_set_deform", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), _dp, _dp, C.c_int]),
    ("cacb200_unset_deform", C.c_int, [C.c_void_p]),
    ("cacb200_set_graphs", C.c_int, [C.c_void_p, C.c_int]),
    ("cacb200_set_list_prefix", C.c_int, [C.c_void_p, C.c_double]),
    ("cacb200_set_neighbor_modify", C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    ("cacb200_run_begin", C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_int]),
    ("cacb200_run_steps", C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_int]),
    ("cacb200_device_array", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_int64)]),
    ("cacb200_replica_energy_noalloc", C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int),
                                                 C.POINTER(C.c_int), C.c_double, _dp, C.c_void_p]),
    ("cacb200_noalloc_last_error", C.c_char_p, []),
    ("cacb200_server_create", C.c_int, [C.c_int, C.c_int, C.c_double, C.c_int, C.POINTER(C.c_void_p)]),
    ("cacb200_server_set_lj", C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double]),
    ("cacb200_server_set_eam", C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_double, C.c_double,
                                         _dp, _dp, _dp]),
    ("cacb200_server_set_neighbor", C.c_int, [C.c_void_p, C.c_double, C.c_int]),
    ("cacb200_server_set_segment", C.c_int, [C.c_void_p, C.c_int]),
    ("cacb200_server_start", C.c_int, [C.c_void_p]),
    ("cacb200_server_submit", C.c_int, [C.c_void_p, C.c_int, _dp, _dp, C.c_int, _dp, _dp, C.c_int, _dp, _dp,
                                        C.c_double, C.c_int, C.c_double, C.c_double, C.c_double,
                                        C.POINTER(C.c_int64)]),
    ("cacb200_server_submit_nvt", C.c_int, [C.c_void_p, _dp, _dp, C.c_int, _dp, _dp, C.c_int, _dp, _dp,
                                            C.c_double, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                            C.c_int, C.c_int, C.POINTER(C.c_int64)]),
    ("cacb200_server_thermo", C.c_int, [C.c_void_p, C.c_int64, _dp]),
    ("cacb200_server_wait", C.c_int, [C.c_void_p, C.c_int64, C.c_double]),
    ("cacb200_server_result", C.c_int, [C.c_void_p, C.c_int64, _dp, _dp, _dp, _dp, _dp, C.POINTER(C.c_int),
                                        C.POINTER(C.c_int), _dp]),
    ("cacb200_server_release", C.c_int, [C.c_void_p, C.c_int64]),
    ("cacb200_server_last_error", C.c_char_p, [C.c_void_p]),
    ("cacb200_server_destroy", C.c_int, [C.c_void_p]),
    ("cacb200_graph_launches", C.c_int, [C.c_void_p, C.POINTER(C.c_longlong)]),
    ("cacb200_pair_blocks", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("cacb200_work_queue", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
    ("cacb200_set_state", C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp]),
    ("cacb200_get_state", C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp]),
    ("cacb200_get_forces", C.c_int, [C.c_void_p, _dp, _dp, _dp]),
    ("cacb200_get_energy", C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp]),
    ("cacb200_counts", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("cacb200_set_lj", C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double]),
    ("cacb200_set_eam", C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_double, C.c_double, _dp, _dp, _dp]),
    ("cacb200_set_nodal_energy_weight", C.c_int, [C.c_void_p, C.c_double]),
    ("cacb200_set_neighbor", C.c_int, [C.c_void_p, C.c_double, C.c_int]),
    ("cacb200_build_lists", C.c_int, [C.c_void_p, C.c_int]),
    ("cacb200_list_size", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int)]),
    ("cacb200_get_list", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int8),
                                   C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int8)]),
    ("cacb200_interpolate", C.c_int, [C.c_void_p]),
    ("cacb200_compute_pair", C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    ("cacb200_assemble_nodef", C.c_int, [C.c_void_p]),
    ("cacb200_compute_forces", C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    ("cacb200_nve_initial", C.c_int, [C.c_void_p, C.c_double]),
    ("cacb200_nve_final", C.c_int, [C.c_void_p, C.c_double]),
    ("cacb200_setup", C.c_int, [C.c_void_p]),
    ("cacb200_run_nve", C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_int]),
    ("cacb200_run_nve_host", C.c_int, [C.c_void_p, C.c_int, C.c_double, C.POINTER(C.c_double),
                                      C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    ("cacb200_set_fire_params", C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double,
                                          C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                          C.c_int, C.c_int]),
    ("cacb200_minimize_fire", C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_double, C.c_int,
                                        C.POINTER(C.c_int), C.POINTER(C.c_int), _dp, _dp]),
    ("cacb200_snapshot", C.c_int, [C.c_void_p]),
    ("cacb200_restore", C.c_int, [C.c_void_p]),
    ("cacb200_profile", C.c_int, [C.c_void_p, C.c_int]),
    ("cacb200_profile_read", C.c_int, [C.c_void_p, C.c_int, C.c_char_p, _dp, C.POINTER(C.c_int64),
                                       C.POINTER(C.c_int)]),
]


def library_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load ``libcacb200.so`` (building it with nvcc when missing or stale)."""
    global _lib
    if _lib is not None:
        return _lib
    if build_if_missing and _build.needs_build():
        _build.build()
    if not os.path.exists(_build.LIB):
        raise CacB200Error("libcacb200.so is not built")
    lib = C.CDLL(_build.LIB)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _p(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def read_setfl(path: str):
    """Parse a one-element setfl file (pair_eam_alloy.cpp:100-190)."""
    with open(path) as f:
        lines = f.read().split("\n")
    nel = int(lines[3].split()[0])
    if nel != 1:
        raise CacB200Error("only one-element setfl files are supported")
    w = lines[4].split()
    nrho, drho, nr, dr, cut = int(w[0]), float(w[1]), int(w[2]), float(w[3]), float(w[4])
    mass = float(lines[5].split()[1])
    vals = np.array([float(t) for t in " ".join(lines[6:]).split()], dtype=np.float64)
    need = nrho + 2 * nr
    if vals.size < need:
        raise CacB200Error("setfl file is truncated")
    return dict(nrho=nrho, drho=drho, nr=nr, dr=dr, cut=cut, mass=mass,
                frho=vals[:nrho].copy(), rhor=vals[nrho:nrho + nr].copy(),
                z2r=vals[nrho + nr:nrho + 2 * nr].copy())


class Engine:
    """One device-resident CAC system (a ``cacb200_ctx``)."""

    def __init__(self, device: int = 0):
        self.lib = load()
        h = C.c_void_p()
        rc = self.lib.cacb200_ctx_create(device, C.byref(h))
        if rc != 0:
            raise CacB200Error(f"cacb200_ctx_create failed ({rc}): no usable CUDA device")
        self.h = h
        self.device = device
        self.na = self.ne = 0
        self._cut = None

    def close(self):
        if getattr(self, "h", None):
            self.lib.cacb200_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str):
        if rc != 0:
            msg = self.lib.cacb200_last_error(self.h)
            raise CacB200Error(f"{what} failed ({rc}): {msg.decode() if msg else ''}")

    @property
    def stream(self) -> int:
        return int(self.lib.cacb200_stream(self.h) or 0)

    # ------------------------------------------------------------- system
    def upload(self, system) -> None:
        x = np.ascontiguousarray(system.x, dtype=np.float64)
        v = np.ascontiguousarray(system.v, dtype=np.float64)
        nx = np.ascontiguousarray(system.nodex, dtype=np.float64)
        nv = np.ascontiguousarray(system.nodev, dtype=np.float64)
        lo = np.ascontiguousarray(system.boxlo, dtype=np.float64)
        hi = np.ascontiguousarray(system.boxhi, dtype=np.float64)
        self.na, self.ne = x.shape[0], nx.shape[0]
        self.rep_na, self.rep_ne = np.array([self.na]), np.array([self.ne])
        self._check(self.lib.cacb200_upload_system(self.h, _p(lo), _p(hi), self.na, _p(x), _p(v),
                                                   self.ne, _p(nx), _p(nv), float(system.mass)),
                    "upload_system")

    def upload_batch(self, systems) -> None:
        """Upload independent replicas (one periodic box each) as one batch."""
        if not systems:
            raise CacB200Error("empty batch")
        mass = float(systems[0].mass)
        if any(float(s.mass) != mass for s in systems):
            raise CacB200Error("replicas of a batch share one mass")
        cat = lambda key, shape: np.ascontiguousarray(
            np.concatenate([np.asarray(getattr(s, key), dtype=np.float64).reshape(shape) for s in systems]))
        x, v = cat("x", (-1, 3)), cat("v", (-1, 3))
        nx, nv = cat("nodex", (-1, 8, 3)), cat("nodev", (-1, 8, 3))
        na = np.array([s.x.shape[0] for s in systems], dtype=np.int32)
        ne = np.array([s.nodex.shape[0] for s in systems], dtype=np.int32)
        lo = np.ascontiguousarray(np.stack([np.asarray(s.boxlo, dtype=np.float64) for s in systems]))
        hi = np.ascontiguousarray(np.stack([np.asarray(s.boxhi, dtype=np.float64) for s in systems]))
        self.na, self.ne = int(na.sum()), int(ne.sum())
        self.rep_na, self.rep_ne = na.copy(), ne.copy()
        ip = C.POINTER(C.c_int)
        self._check(self.lib.cacb200_upload_batch(self.h, len(systems), na.ctypes.data_as(ip),
                                                  ne.ctypes.data_as(ip), _p(lo), _p(hi), _p(x), _p(v),
                                                  _p(nx), _p(nv), mass), "upload_batch")

    def replica_energy(self) -> np.ndarray:
        n = len(getattr(self, "rep_na", [0]))
        out = np.zeros(n)
        self._check(self.lib.cacb200_replica_energy(self.h, _p(out)), "replica_energy")
        return out

    THERMO_FIELDS = ("temp", "ke", "pe", "etotal", "press", "pxx", "pyy", "pzz", "pxy", "pxz", "pyz", "vol")

    def thermo(self, units: str = "metal"):
        """Thermo read-out reduced on the device (``thermo_style custom temp ke
        pe etotal press pxx pyy pzz pxy pxz pyz vol``, norm no): a dict of
        floats for one system (or a batch of one), of arrays (one entry per
        replica) for a batch.  ``units`` is ``metal`` (bar) or ``metalgpa`` (GPa).  Energies
        and pressures not tallied at the current step read NaN."""
        u = {"metal": 0, "metalgpa": 1}.get(units)
        if u is None:
            raise ValueError(f"unknown unit style {units!r}")
        n = len(getattr(self, "rep_na", [0]))
        out = np.zeros((n, len(self.THERMO_FIELDS)))
        self._check(self.lib.cacb200_thermo(self.h, u, _p(out)), "thermo")
        if n == 1:
            return {k: float(out[0, i]) for i, k in enumerate(self.THERMO_FIELDS)}
        return {k: out[:, i].copy() for i, k in enumerate(self.THERMO_FIELDS)}

    ARRAYS = {"x": (0, 4), "v": (1, 3), "f": (2, 3), "nodex": (3, 3), "nodev": (4, 3), "nodef": (5, 3),
              "eatom": (6, 1), "enode": (7, 1), "vatom": (8, 6), "vnode": (9, 6)}

    def device_array(self, name: str):
        """A context array as a torch CUDA tensor sharing the device memory
        (no copy): ``x`` (natoms, 4), ``v``/``f`` (natoms, 3), ``nodex``/
        ``nodev``/``nodef`` (nelements*8, 3), ``eatom`` (natoms,), ``enode``
        (nelements*8,), ``vatom``/``vnode`` (n, 6).  Synchronises the
        context's stream first; valid until the next upload or list plan."""
        import torch
        which, width = self.ARRAYS[name]
        ptr, n = C.c_void_p(), C.c_int64()
        self._check(self.lib.cacb200_device_array(self.h, which, C.byref(ptr), C.byref(n)), "device_array")
        torch.cuda.ExternalStream(self.stream, device=torch.device("cuda", self.device)).synchronize()
        shape = (n.value // width, width) if width > 1 else (n.value,)

        class _View:
            __cuda_array_interface__ = {"shape": shape, "typestr": "<f8", "data": (ptr.value or 0, False),
                                        "version": 3, "strides": None}
        return torch.as_tensor(_View(), device=torch.device("cuda", self.device))

    def neighbor_modify(self, delay: int = 0, check: bool = False) -> None:
        """neigh_modify delay D check yes|no (the every of ``neighbor`` stays)."""
        self._check(self.lib.cacb200_set_neighbor_modify(self.h, delay, 1 if check else 0),
                    "set_neighbor_modify")

    def list_prefix(self, margin: float) -> None:
        """Inner-prefix margin of the lists (< 0: default 0.5 x skin, 0: off)."""
        self._check(self.lib.cacb200_set_list_prefix(self.h, margin), "set_list_prefix")

    def graphs(self, enable: bool) -> None:
        self._check(self.lib.cacb200_set_graphs(self.h, 1 if enable else 0), "set_graphs")

    def pair_blocks(self):
        """(rho, force) block sizes the context chose for its force-only EAM passes."""
        r, f = C.c_int(), C.c_int()
        self._check(self.lib.cacb200_pair_blocks(self.h, C.byref(r), C.byref(f)), "pair_blocks")
        return r.value, f.value

    def work_queue(self, enable=None):
        """Batches (mixed form): turn the persistent work-queue launches on or
        off (None: unchanged); returns the tiles chosen per size class."""
        t = (C.c_int * 3)()
        self._check(self.lib.cacb200_work_queue(self.h, -1 if enable is None else int(bool(enable)), t),
                    "work_queue")
        return list(t)

    def graph_launches(self) -> int:
        n = C.c_longlong()
        self._check(self.lib.cacb200_graph_launches(self.h, C.byref(n)), "graph_launches")
        return n.value

    def read_data(self, path: str) -> None:
        """Upload a data file in the reference's format (read_data)."""
        na, ne = C.c_int(), C.c_int()
        self._check(self.lib.cacb200_read_data(self.h, path.encode()), "read_data")
        self._check(self.lib.cacb200_counts(self.h, C.byref(na), C.byref(ne), None), "counts")
        self.na, self.ne = na.value, ne.value
        self.rep_na, self.rep_ne = np.array([self.na]), np.array([self.ne])

    def write_data(self, path: str) -> None:
        """Write the current state as a data file in the reference's format."""
        self._check(self.lib.cacb200_write_data(self.h, path.encode()), "write_data")

    def set_precision(self, form: int) -> None:
        self._check(self.lib.cacb200_set_precision(self.h, form), "set_precision")

    def pair_lj(self, epsilon: float, sigma: float, cut: float) -> None:
        self._check(self.lib.cacb200_set_lj(self.h, epsilon, sigma, cut), "set_lj")

    def pair_eam(self, setfl) -> None:
        t = read_setfl(setfl) if isinstance(setfl, str) else setfl
        self._check(self.lib.cacb200_set_eam(self.h, t["nrho"], t["drho"], t["nr"], t["dr"], t["cut"],
                                             _p(t["frho"]), _p(t["rhor"]), _p(t["z2r"])), "set_eam")

    def nodal_energy_weight(self, w: float) -> None:
        self._check(self.lib.cacb200_set_nodal_energy_weight(self.h, w), "set_nodal_energy_weight")

    def neighbor(self, skin: float, every: int) -> None:
        self._check(self.lib.cacb200_set_neighbor(self.h, skin, every), "set_neighbor")

    # ------------------------------------------------------------- lists
    def build_lists(self, half: bool = False) -> None:
        self._check(self.lib.cacb200_build_lists(self.h, 1 if half else 0), "build_lists")

    def neighbor_list(self, half: bool = False) -> np.ndarray:
        """Sorted int64 rows (i_site, kind, idx, site, sx, sy, sz)."""
        n = C.c_int64()
        ns = C.c_int()
        self._check(self.lib.cacb200_list_size(self.h, 1 if half else 0, C.byref(n), C.byref(ns)), "list_size")
        n, ns = n.value, ns.value
        off = np.zeros(ns + 1, dtype=np.int64)
        kind = np.zeros(max(n, 1), dtype=np.int8)
        idx = np.zeros(max(n, 1), dtype=np.int32)
        site = np.zeros(max(n, 1), dtype=np.int32)
        img = np.zeros(max(n, 1) * 3, dtype=np.int8)
        self._check(self.lib.cacb200_get_list(
            self.h, 1 if half else 0, off.ctypes.data_as(C.POINTER(C.c_int64)),
            kind.ctypes.data_as(C.POINTER(C.c_int8)), idx.ctypes.data_as(C.POINTER(C.c_int32)),
            site.ctypes.data_as(C.POINTER(C.c_int32)), img.ctypes.data_as(C.POINTER(C.c_int8))), "get_list")
        isite = np.repeat(np.arange(ns, dtype=np.int64), np.diff(off))
        img = img[:3 * n].reshape(n, 3).astype(np.int64)
        rows = np.stack([isite, kind[:n].astype(np.int64), idx[:n].astype(np.int64),
                         site[:n].astype(np.int64), img[:, 0], img[:, 1], img[:, 2]], axis=1)
        return rows[np.lexsort(rows.T[::-1])]

    # ------------------------------------------------------------- steps
    def compute(self, eflag: int = ENERGY_GLOBAL | ENERGY_ATOM, vflag: int = VIRIAL_GLOBAL | VIRIAL_ATOM) -> None:
        self._check(self.lib.cacb200_compute_forces(self.h, eflag, vflag), "compute_forces")

    def setup(self) -> None:
        self._check(self.lib.cacb200_setup(self.h), "setup")

    def langevin(self, t_start: float, t_stop: float, t_period: float, seed: int, zero: bool = False) -> None:
        """``fix ID all langevin t_start t_stop t_period seed [zero yes]``, applied by run_nve."""
        self._check(self.lib.cacb200_set_langevin(self.h, t_start, t_stop, t_period, seed, 1 if zero else 0),
                    "set_langevin")

    DEFORM_STYLES = {"none": 0, "final": 1, "delta": 2, "scale": 3, "vel": 4, "erate": 5, "trate": 6,
                     "wiggle": 7, "volume": 8}

    def deform(self, nevery: int, remap: str = "x", **dims) -> None:
        """``fix ID all deform N dim style args ... remap x|none units box``:
        ``deform(1, x=("erate", 0.5), y=("volume",), z=("final", lo, hi))``."""
        style = (C.c_int * 3)()
        a, b = np.zeros(3), np.zeros(3)
        for d, name in enumerate("xyz"):
            spec = dims.pop(name, ("none",))
            style[d] = self.DEFORM_STYLES[spec[0]]
            args = list(spec[1:]) + [0.0, 0.0]
            a[d], b[d] = float(args[0]), float(args[1])
        if dims:
            raise ValueError(f"unknown dimensions {sorted(dims)}")
        if remap not in ("x", "none"):
            raise ValueError("remap must be x or none")
        self._check(self.lib.cacb200_set_deform(self.h, nevery, style, _p(a), _p(b), 1 if remap == "x" else 0),
                    "set_deform")

    def set_box(self, boxlo, boxhi) -> None:
        """New periodic box of a single system, sites left where they are."""
        lo = np.ascontiguousarray(boxlo, dtype=np.float64)
        hi = np.ascontiguousarray(boxhi, dtype=np.float64)
        self._check(self.lib.cacb200_set_box(self.h, _p(lo), _p(hi)), "set_box")

    def unset_deform(self) -> None:
        self._check(self.lib.cacb200_unset_deform(self.h), "unset_deform")

    def box(self):
        """(boxlo, boxhi) of a single system."""
        lo, hi, m = np.zeros(3), np.zeros(3), C.c_double()
        self._check(self.lib.cacb200_get_box(self.h, _p(lo), _p(hi), C.byref(m)), "get_box")
        return lo, hi

    def langevin_stream(self, draws: int) -> None:
        """Continue the thermostat's RanMars streams after ``draws`` uniform() calls."""
        self._check(self.lib.cacb200_set_langevin_stream(self.h, int(draws)), "set_langevin_stream")

    def unset_langevin(self) -> None:
        self._check(self.lib.cacb200_unset_langevin(self.h), "unset_langevin")

    def run_begin(self, nsteps: int, dt: float = 0.001, eflag: int = 0, vflag: int = 0) -> None:
        """Verlet::setup of a run of ``nsteps`` (see run_steps)."""
        self._check(self.lib.cacb200_run_begin(self.h, nsteps, dt, eflag, vflag), "run_begin")

    def run_steps(self, nsteps: int, dt: float = 0.001, eflag: int = 0, vflag: int = 0) -> None:
        """Advance the run begun by run_begin by ``nsteps`` of its steps."""
        self._check(self.lib.cacb200_run_steps(self.h, nsteps, dt, eflag, vflag), "run_steps")

    def run_nve(self, nsteps: int, dt: float = 0.001, eflag: int = 0, vflag: int = 0) -> None:
        self._check(self.lib.cacb200_run_nve(self.h, nsteps, dt, eflag, vflag), "run_nve")

    def run_nve_host(self, nsteps: int, x, v, nodex, nodev, dt: float = 0.001) -> None:
        """State in from host arrays, nsteps of NVE, state back into the same
        arrays (float64, C order; pinned memory lets the position copy run
        beside the last step's forces)."""
        arrs = []
        for a in (x, v, nodex, nodev):
            if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous
                    and a.flags.writeable):
                raise ValueError("run_nve_host needs writable C-contiguous float64 arrays")
            arrs.append(_p(a))
        self._check(self.lib.cacb200_run_nve_host(self.h, nsteps, dt, *arrs), "run_nve_host")

    def fire_params(self, delaystep=20, dtgrow=1.1, dtshrink=0.5, alpha0=0.25, alphashrink=0.99,
                    tmax=10.0, tmin=0.02, dmax=0.1, halfstepback=True, delaystep_start=True,
                    max_vdotf_negatif=2000) -> None:
        self._check(self.lib.cacb200_set_fire_params(self.h, delaystep, dtgrow, dtshrink, alpha0, alphashrink,
                                                     tmax, tmin, dmax, int(halfstepback), int(delaystep_start),
                                                     max_vdotf_negatif), "set_fire_params")

    def minimize_fire(self, etol: float = 0.0, ftol: float = 1e-6, maxiter: int = 5000, dt: float = 0.001,
                      norm: str = "max"):
        """min_style fire/b200; minimize etol ftol maxiter.  Returns
        (stop_code, iterations, energy, fnorm)."""
        ns = {"two": 0, "max": 1, "inf": 2}[norm]
        code, it = C.c_int(), C.c_int()
        e, fn = C.c_double(), C.c_double()
        self._check(self.lib.cacb200_minimize_fire(self.h, etol, ftol, maxiter, dt, ns, C.byref(code),
                                                   C.byref(it), C.byref(e), C.byref(fn)), "minimize_fire")
        return code.value, it.value, e.value, fn.value

    def snapshot(self) -> None:
        self._check(self.lib.cacb200_snapshot(self.h), "snapshot")

    def restore(self) -> None:
        self._check(self.lib.cacb200_restore(self.h), "restore")

    def counts(self):
        a, e, s = C.c_int(), C.c_int(), C.c_int()
        self._check(self.lib.cacb200_counts(self.h, C.byref(a), C.byref(e), C.byref(s)), "counts")
        return a.value, e.value, s.value

    # ------------------------------------------------------------- read-outs
    def state(self):
        x = np.zeros((self.na, 3))
        v = np.zeros((self.na, 3))
        nx = np.zeros((self.ne, 8, 3))
        nv = np.zeros((self.ne, 8, 3))
        self._check(self.lib.cacb200_get_state(self.h, _p(x), _p(v), _p(nx), _p(nv)), "get_state")
        return x, v, nx, nv

    def set_state(self, x=None, v=None, nodex=None, nodev=None) -> None:
        conv = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        x, v, nodex, nodev = conv(x), conv(v), conv(nodex), conv(nodev)
        self._check(self.lib.cacb200_set_state(self.h, _p(x), _p(v), _p(nodex), _p(nodev)), "set_state")

    def forces(self):
        f = np.zeros((self.na, 3))
        nf = np.zeros((self.ne, 8, 3))
        gf = np.zeros((self.ne, 8, 3))
        self._check(self.lib.cacb200_get_forces(self.h, _p(f), _p(nf), _p(gf)), "get_forces")
        return f, nf, gf

    def energy(self, peratom: bool = True):
        e = C.c_double()
        vir = np.zeros(6)
        out = {}
        if peratom:
            out["eatom"] = np.zeros(self.na)
            out["vatom"] = np.zeros((self.na, 6))
            out["enode"] = np.zeros((self.ne, 8))
            out["vnode"] = np.zeros((self.ne, 8, 6))
            self._check(self.lib.cacb200_get_energy(self.h, C.byref(e), _p(vir), _p(out["eatom"]),
                                                    _p(out["vatom"]), _p(out["enode"]), _p(out["vnode"])),
                        "get_energy")
        else:
            self._check(self.lib.cacb200_get_energy(self.h, C.byref(e), _p(vir), None, None, None, None),
                        "get_energy")
        out["energy"] = e.value
        out["virial"] = vir
        return out

    # ------------------------------------------------------------- profiling
    def profile(self, enable: bool) -> None:
        self._check(self.lib.cacb200_profile(self.h, 1 if enable else 0), "profile")

    def profile_read(self):
        maxn = 64
        names = C.create_string_buffer(32 * maxn)
        ms = np.zeros(maxn)
        la = np.zeros(maxn, dtype=np.int64)
        cnt = C.c_int()
        self._check(self.lib.cacb200_profile_read(self.h, maxn, names, _p(ms),
                                                  la.ctypes.data_as(C.POINTER(C.c_int64)), C.byref(cnt)),
                    "profile_read")
        out = {}
        raw = names.raw
        for k in range(min(cnt.value, maxn)):
            nm = raw[32 * k:32 * k + 32].split(b"\0", 1)[0].decode()
            out[nm] = (float(ms[k]), int(la[k]))
        return out


JOB_NVE = 0
JOB_FIRE = 1


class Server:
    """A ``cacb200_server``: jobs (one system each, ``run N`` under NVE or a
    FIRE minimisation) served concurrently by worker threads that each own a
    device context, admitted first come first served under a memory budget."""

    def __init__(self, device: int = 0, workers: int = 8, budget_gb: float = 120.0, precision: int = FP64):
        self.lib = load()
        h = C.c_void_p()
        rc = self.lib.cacb200_server_create(device, workers, budget_gb * 1e9, precision, C.byref(h))
        if rc != 0:
            raise CacB200Error(f"cacb200_server_create failed ({rc})")
        self.h = h
        self._shapes = {}

    def _check(self, rc: int, what: str):
        if rc != 0:
            raise CacB200Error(f"{what} failed ({rc}): {self.last_error()}")

    def last_error(self) -> str:
        msg = self.lib.cacb200_server_last_error(self.h)
        return msg.decode() if msg else ""

    def pair_lj(self, epsilon: float, sigma: float, cut: float) -> None:
        self._check(self.lib.cacb200_server_set_lj(self.h, epsilon, sigma, cut), "server_set_lj")

    def pair_eam(self, setfl) -> None:
        t = read_setfl(setfl) if isinstance(setfl, str) else setfl
        self._check(self.lib.cacb200_server_set_eam(self.h, t["nrho"], t["drho"], t["nr"], t["dr"], t["cut"],
                                                    _p(t["frho"]), _p(t["rhor"]), _p(t["z2r"])), "server_set_eam")

    def neighbor(self, skin: float, every: int) -> None:
        self._check(self.lib.cacb200_server_set_neighbor(self.h, skin, every), "server_set_neighbor")

    def segment(self, steps: int) -> None:
        self._check(self.lib.cacb200_server_set_segment(self.h, steps), "server_set_segment")

    def start(self) -> None:
        self._check(self.lib.cacb200_server_start(self.h), "server_start")

    def submit(self, system, kind: int, steps: int, dt: float = 0.001, etol: float = 0.0,
               ftol: float = 0.0) -> int:
        x = np.ascontiguousarray(system.x, dtype=np.float64)
        v = np.ascontiguousarray(system.v, dtype=np.float64)
        nx = np.ascontiguousarray(system.nodex, dtype=np.float64)
        nv = np.ascontiguousarray(system.nodev, dtype=np.float64)
        lo = np.ascontiguousarray(system.boxlo, dtype=np.float64)
        hi = np.ascontiguousarray(system.boxhi, dtype=np.float64)
        job = C.c_int64()
        self._check(self.lib.cacb200_server_submit(self.h, kind, _p(lo), _p(hi), x.shape[0], _p(x), _p(v),
                                                   nx.shape[0], _p(nx), _p(nv), float(system.mass), steps, dt,
                                                   etol, ftol, C.byref(job)), "server_submit")
        self._shapes[job.value] = (x.shape[0], nx.shape[0])
        return job.value

    def submit_nvt(self, system, steps: int, dt: float, t_start: float, t_stop: float, damp: float, seed: int,
                   zero: bool = False) -> int:
        """An NVE job under ``fix langevin t_start t_stop damp seed [zero yes]``."""
        x = np.ascontiguousarray(system.x, dtype=np.float64)
        v = np.ascontiguousarray(system.v, dtype=np.float64)
        nx = np.ascontiguousarray(system.nodex, dtype=np.float64)
        nv = np.ascontiguousarray(system.nodev, dtype=np.float64)
        lo = np.ascontiguousarray(system.boxlo, dtype=np.float64)
        hi = np.ascontiguousarray(system.boxhi, dtype=np.float64)
        job = C.c_int64()
        self._check(self.lib.cacb200_server_submit_nvt(self.h, _p(lo), _p(hi), x.shape[0], _p(x), _p(v),
                                                       nx.shape[0], _p(nx), _p(nv), float(system.mass), steps, dt,
                                                       t_start, t_stop, damp, seed, 1 if zero else 0,
                                                       C.byref(job)), "server_submit_nvt")
        self._shapes[job.value] = (x.shape[0], nx.shape[0])
        return job.value

    def thermo(self, job: int) -> dict:
        """The job's thermo line at its end (Engine.THERMO_FIELDS, metal units)."""
        out = np.zeros(len(Engine.THERMO_FIELDS))
        self._check(self.lib.cacb200_server_thermo(self.h, job, _p(out)), "server_thermo")
        return {k: float(out[i]) for i, k in enumerate(Engine.THERMO_FIELDS)}

    def wait(self, job: int, timeout: float = -1.0) -> int:
        """The job's status once it ends (0 = done), or CACB200_ETIMEDOUT."""
        return self.lib.cacb200_server_wait(self.h, job, timeout)

    def times(self, job: int) -> np.ndarray:
        """[queued, running, submit to end] seconds of an ended job, failed or not."""
        t = np.zeros(3)
        self.lib.cacb200_server_result(self.h, job, None, None, None, None, None, None, None, _p(t))
        return t

    def result(self, job: int):
        """(x, v, nodex, nodev, energy, iterations, stop_code, times[queued, running, total])"""
        na, ne = self._shapes[job]
        x, v = np.zeros((na, 3)), np.zeros((na, 3))
        nx, nv = np.zeros((ne, 8, 3)), np.zeros((ne, 8, 3))
        e = np.zeros(1)
        it, code = C.c_int(), C.c_int()
        t = np.zeros(3)
        self._check(self.lib.cacb200_server_result(self.h, job, _p(x), _p(v), _p(nx), _p(nv), _p(e),
                                                   C.byref(it), C.byref(code), _p(t)), "server_result")
        return x, v, nx, nv, float(e[0]), it.value, code.value, t

    def release(self, job: int) -> None:
        self._check(self.lib.cacb200_server_release(self.h, job), "server_release")
        self._shapes.pop(job, None)

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.cacb200_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _data_check(lib, rc: int, what: str):
    if rc != 0:
        msg = lib.cacb200_data_last_error()
        raise CacB200Error(f"{what} failed ({rc}): {msg.decode() if msg else ''}")


def read_data_file(path: str):
    """Host-only read of a data file in the reference's format: a ``gen.System``
    with the file's box, mass and state (tags in file order)."""
    from cac_b200 import gen
    lib = load()
    na, ne = C.c_int(), C.c_int()
    lo, hi, m = np.zeros(3), np.zeros(3), np.zeros(1)
    _data_check(lib, lib.cacb200_data_counts(path.encode(), C.byref(na), C.byref(ne), _p(lo), _p(hi), _p(m)),
                "data_counts")
    x, v = np.zeros((na.value, 3)), np.zeros((na.value, 3))
    nx, nv = np.zeros((ne.value, 8, 3)), np.zeros((ne.value, 8, 3))
    _data_check(lib, lib.cacb200_data_read(path.encode(), _p(x), _p(v), _p(nx), _p(nv)), "data_read")
    return gen.System(boxlo=lo, boxhi=hi, x=x, v=v, nodex=nx, nodev=nv, mass=float(m[0]), lattice_a=0.0, meta={})


def write_data_file(path: str, system) -> None:
    """Host-only write of ``system`` in the reference's data-file format."""
    lib = load()
    arr = lambda a, shape: np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(shape))
    x, v = arr(system.x, (-1, 3)), arr(system.v, (-1, 3))
    nx, nv = arr(system.nodex, (-1, 8, 3)), arr(system.nodev, (-1, 8, 3))
    lo, hi = arr(system.boxlo, (3,)), arr(system.boxhi, (3,))
    _data_check(lib, lib.cacb200_data_write(path.encode(), x.shape[0], nx.shape[0], _p(lo), _p(hi),
                                            float(system.mass), _p(x), _p(v), _p(nx), _p(nv)), "data_write")
