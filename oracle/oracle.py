"""ctypes bindings for the C restatement (``_ref/liboracle.so``) and readers for
the reference executable's ``oracle_dump`` / ``oracle_dump_neigh`` output.

TEST INFRASTRUCTURE, NOT PRODUCT CODE.  Only the tests, the smoke check and
the benchmark's CPU-baseline leg import this module, and only as the checker.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
LIB_PATH = os.path.join(REF_DIR, "liboracle.so")
REF_EXE = os.path.join(REF_DIR, "cac")
REF_EXE_EAMFIX = os.path.join(REF_DIR, "cac_eamfix")

_dp = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)
_i32p = C.POINTER(C.c_int32)
_i8p = C.POINTER(C.c_int8)


class _State(C.Structure):
    _fields_ = [("boxlo", C.c_double * 3), ("boxhi", C.c_double * 3),
                ("natoms", C.c_int), ("nelements", C.c_int),
                ("x", _dp), ("v", _dp), ("f", _dp),
                ("nodex", _dp), ("nodev", _dp), ("nodef", _dp), ("gaussf", _dp),
                ("mass", C.c_double)]


class _List(C.Structure):
    _fields_ = [("nsites", C.c_int), ("nentries", C.c_int64), ("offset", _i64p),
                ("jidx", _i32p), ("jsite", _i32p), ("jkind", _i8p), ("img", _i8p)]


class _Ev(C.Structure):
    _fields_ = [("energy", C.c_double), ("virial", C.c_double * 6),
                ("eatom", _dp), ("vatom", _dp), ("enode", _dp), ("vnode", _dp)]


class _Eam(C.Structure):
    _fields_ = [("nrho", C.c_int), ("nr", C.c_int), ("drho", C.c_double), ("dr", C.c_double),
                ("cut", C.c_double), ("rhomax", C.c_double),
                ("frho_spline", _dp), ("rhor_spline", _dp), ("z2r_spline", _dp)]


_lib = None


def build() -> None:
    """Compile the restatement (and, where the reference tree exists, the reference)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-s", "-C", HERE, "restatement"], check=True)
        L = C.CDLL(LIB_PATH)
        L.oracle_build_list.argtypes = [C.POINTER(_State), C.c_double, C.c_int, C.POINTER(_List)]
        L.oracle_free_list.argtypes = [C.POINTER(_List)]
        L.oracle_lj_compute.argtypes = [C.POINTER(_State), C.POINTER(_List), C.c_double,
                                        C.c_double, C.c_double, C.POINTER(_Ev)]
        L.oracle_eam_load_setfl.argtypes = [C.c_char_p, C.POINTER(_Eam)]
        L.oracle_eam_free.argtypes = [C.POINTER(_Eam)]
        L.oracle_eam_compute.argtypes = [C.POINTER(_State), C.POINTER(_List), C.POINTER(_Eam),
                                         C.POINTER(_Ev), _dp, _dp]
        L.oracle_compute_nodef.argtypes = [C.POINTER(_State)]
        L.oracle_nve_initial.argtypes = [C.POINTER(_State), C.c_double]
        L.oracle_nve_final.argtypes = [C.POINTER(_State), C.c_double]
        L.oracle_pbc.argtypes = [C.POINTER(_State)]
        L.oracle_run_nve.argtypes = [C.POINTER(_State), C.c_int, C.c_double, C.c_double,
                                     C.c_double, C.POINTER(_Eam), C.c_double, C.c_double,
                                     C.c_int, C.c_int]
        L.oracle_minimize_fire.argtypes = [C.POINTER(_State), C.c_int, C.c_double, C.c_double, C.c_double,
                                           C.POINTER(_Eam), C.c_double, C.c_double, C.c_double, C.c_double,
                                           C.c_int, C.c_int, C.c_int, _dp, C.POINTER(C.c_int),
                                           C.POINTER(C.c_int), _dp, _dp]
        L.oracle_set_neighbor_check.argtypes = [C.c_int]
        L.oracle_shape_array.argtypes = [_dp]
        L.oracle_gauss_tables.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int), _dp, _dp]
        L.oracle_inverse_mass_hex.argtypes = [_dp]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class OracleState:
    """Owns contiguous float64 copies of a system's arrays."""

    def __init__(self, system):
        self.x = np.ascontiguousarray(system.x, dtype=np.float64).copy()
        self.v = np.ascontiguousarray(system.v, dtype=np.float64).copy()
        self.nodex = np.ascontiguousarray(system.nodex, dtype=np.float64).copy()
        self.nodev = np.ascontiguousarray(system.nodev, dtype=np.float64).copy()
        self.f = np.zeros_like(self.x)
        self.nodef = np.zeros_like(self.nodex)
        self.gaussf = np.zeros_like(self.nodex)
        self.boxlo = np.array(system.boxlo, dtype=np.float64)
        self.boxhi = np.array(system.boxhi, dtype=np.float64)
        self.mass = float(system.mass)
        self._s = _State()
        self._s.boxlo[:] = list(self.boxlo)
        self._s.boxhi[:] = list(self.boxhi)
        self._s.natoms = self.x.shape[0]
        self._s.nelements = self.nodex.shape[0]
        for name in ("x", "v", "f", "nodex", "nodev", "nodef", "gaussf"):
            setattr(self._s, name, _ptr(getattr(self, name)))
        self._s.mass = self.mass

    @property
    def ref(self):
        return C.byref(self._s)


class NeighList:
    def __init__(self, offset, jkind, jidx, jsite, img):
        self.offset, self.jkind, self.jidx, self.jsite, self.img = offset, jkind, jidx, jsite, img

    @property
    def nsites(self):
        return len(self.offset) - 1

    def canonical(self, natoms: int):
        """Sorted int64 rows (i_site, kind, idx, site, sx, sy, sz)."""
        counts = np.diff(self.offset)
        isite = np.repeat(np.arange(self.nsites, dtype=np.int64), counts)
        rows = np.stack([isite, self.jkind.astype(np.int64), self.jidx.astype(np.int64),
                         self.jsite.astype(np.int64), self.img[:, 0].astype(np.int64),
                         self.img[:, 1].astype(np.int64), self.img[:, 2].astype(np.int64)], axis=1)
        order = np.lexsort(rows.T[::-1])
        return rows[order]


def build_list(state: OracleState, cutneigh: float, half: bool) -> NeighList:
    L = _List()
    rc = lib().oracle_build_list(state.ref, cutneigh, 1 if half else 0, C.byref(L))
    if rc:
        raise RuntimeError(f"oracle_build_list failed ({rc})")
    n = L.nentries
    ns = L.nsites
    out = NeighList(
        np.ctypeslib.as_array(L.offset, shape=(ns + 1,)).copy(),
        np.ctypeslib.as_array(L.jkind, shape=(max(n, 1),))[:n].copy(),
        np.ctypeslib.as_array(L.jidx, shape=(max(n, 1),))[:n].copy(),
        np.ctypeslib.as_array(L.jsite, shape=(max(n, 1),))[:n].copy(),
        np.ctypeslib.as_array(L.img, shape=(max(n, 1) * 3,))[:3 * n].reshape(n, 3).copy())
    out._c = L
    return out


def _c_list(nl: NeighList) -> _List:
    return nl._c


def free_list(nl: NeighList) -> None:
    if getattr(nl, "_c", None) is not None:
        lib().oracle_free_list(C.byref(nl._c))
        nl._c = None


class EvResult:
    def __init__(self, natoms, nelements):
        self.eatom = np.zeros(natoms)
        self.vatom = np.zeros((natoms, 6))
        self.enode = np.zeros((nelements, 8))
        self.vnode = np.zeros((nelements, 8, 6))
        self._ev = _Ev()
        self._ev.eatom = _ptr(self.eatom)
        self._ev.vatom = _ptr(self.vatom)
        self._ev.enode = _ptr(self.enode)
        self._ev.vnode = _ptr(self.vnode)

    @property
    def energy(self):
        return self._ev.energy

    @property
    def virial(self):
        return np.array(list(self._ev.virial))


def lj_forces(state: OracleState, half_list: NeighList, eps: float, sigma: float, cut: float):
    ev = EvResult(state.x.shape[0], state.nodex.shape[0])
    lib().oracle_lj_compute(state.ref, C.byref(half_list._c), eps, sigma, cut, C.byref(ev._ev))
    lib().oracle_compute_nodef(state.ref)
    return ev


class Eam:
    def __init__(self, path: str):
        self._e = _Eam()
        rc = lib().oracle_eam_load_setfl(path.encode(), C.byref(self._e))
        if rc:
            raise RuntimeError(f"cannot read setfl {path} ({rc})")

    @property
    def cut(self):
        return self._e.cut

    def __del__(self):
        try:
            lib().oracle_eam_free(C.byref(self._e))
        except Exception:
            pass


def eam_forces(state: OracleState, half_list: NeighList, eam: Eam):
    ev = EvResult(state.x.shape[0], state.nodex.shape[0])
    rho_a = np.zeros(state.x.shape[0])
    rho_n = np.zeros((state.nodex.shape[0], 8))
    lib().oracle_eam_compute(state.ref, C.byref(half_list._c), C.byref(eam._e), C.byref(ev._ev),
                             _ptr(rho_a), _ptr(rho_n))
    lib().oracle_compute_nodef(state.ref)
    ev.rho_atom, ev.rho_node = rho_a, rho_n
    return ev


def run_nve(state: OracleState, pair: str, *, lj=None, eam: Optional[Eam] = None,
            skin: float = 1.0, dt: float = 0.001, nsteps: int = 10, every: int = 10) -> None:
    if pair == "lj":
        eps, sig, cut = lj
        rc = lib().oracle_run_nve(state.ref, 0, eps, sig, cut, None, skin, dt, nsteps, every)
    else:
        rc = lib().oracle_run_nve(state.ref, 1, 0.0, 0.0, 0.0, C.byref(eam._e), skin, dt, nsteps, every)
    if rc:
        raise RuntimeError("oracle_run_nve failed")


FIRE_DEFAULTS = (20, 1.1, 0.5, 0.25, 0.99, 10.0, 0.02, 0.1, 1, 1, 2000)


def minimize_fire(state: OracleState, pair: str, *, lj=None, eam: Optional[Eam] = None,
                  skin: float = 1.0, dt: float = 0.001, etol: float = 0.0, ftol: float = 1e-6,
                  maxiter: int = 5000, norm: str = "max", every: int = 10, check: bool = False,
                  params=FIRE_DEFAULTS):
    """FIRE restated in C; returns (stop_code, iterations, energy, fnorm).
    check: neigh_modify check yes (a rebuild due by ``every`` only after a
    move past half the skin, as the reference's Min runs its lists)."""
    par = np.array(params, dtype=np.float64)
    lib().oracle_set_neighbor_check(1 if check else 0)
    code, it = C.c_int(), C.c_int()
    e, fn = C.c_double(), C.c_double()
    ns = {"two": 0, "max": 1, "inf": 2}[norm]
    if pair == "lj":
        eps, sig, cut = lj
        rc = lib().oracle_minimize_fire(state.ref, 0, eps, sig, cut, None, skin, dt, etol, ftol, maxiter, ns,
                                        every, _ptr(par), C.byref(code), C.byref(it), C.byref(e), C.byref(fn))
    else:
        rc = lib().oracle_minimize_fire(state.ref, 1, 0.0, 0.0, 0.0, C.byref(eam._e), skin, dt, etol, ftol,
                                        maxiter, ns, every, _ptr(par), C.byref(code), C.byref(it), C.byref(e),
                                        C.byref(fn))
    lib().oracle_set_neighbor_check(0)
    if rc:
        raise RuntimeError("oracle_minimize_fire failed")
    return code.value, it.value, e.value, fn.value


# ------------------------------------------------------------------ thermo

THERMO_FIELDS = ("temp", "ke", "pe", "etotal", "press", "pxx", "pyy", "pzz", "pxy", "pxz", "pyz", "vol")
THERMO_COLUMNS = ("Temp", "KinEng", "PotEng", "TotEng", "Press", "Pxx", "Pyy", "Pzz", "Pxy", "Pxz", "Pyz",
                  "Volume")
BOLTZ, MVV2E = 8.617343e-5, 1.0364269e-4          # update.cpp:160-164 (metal)
NKTV2P = {"metal": 1.6021765e6, "metalgpa": 1.6021765e2}   # update.cpp:166-170


def hex_mass_matrix() -> np.ndarray:
    """Element::define_mass_matrices, HEXAHEDRON (element.cpp:1993-2056), as
    the listed literals: 1/27, 1/54, 1/108, 1/216 by the number of natural
    coordinates in which two nodes differ."""
    corner = np.array([(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)])
    d = (corner[:, None, :] != corner[None, :, :]).sum(-1)
    return np.array([1.0 / 27.0, 1.0 / 54.0, 1.0 / 108.0, 1.0 / 216.0])[d]


def thermo(v, nodev, mass, boxlo, boxhi, energy, virial, units: str = "metal", nucell: int = 729) -> dict:
    """Thermo keywords temp ke pe etotal press pxx..pyz vol (norm no) of one
    system, restated with Python loops in the reference's order of terms:
    ComputeTemp::dof_compute / compute_scalar / compute_vector
    (compute_temp.cpp:74-158, 160-243; CONSISTENT branch, apc 1), virtual
    atoms nucell per element (group.cpp:1160-1175), ComputePressure
    (compute_pressure.cpp:140-220), Thermo::compute_ke / compute_etotal
    (thermo.cpp:1913-1936).  ``energy`` / ``virial`` are the pair's tallies."""
    v = np.asarray(v, dtype=np.float64).reshape(-1, 3)
    nodev = np.asarray(nodev, dtype=np.float64).reshape(-1, 8, 3)
    M = hex_mass_matrix()
    t = 0.0
    tv = [0.0] * 6
    for i in range(v.shape[0]):
        vx, vy, vz = v[i]
        t += mass * (vx * vx + vy * vy + vz * vz)
        for q, (a, b) in enumerate(((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))):
            tv[q] += mass * v[i, a] * v[i, b]
    for e in range(nodev.shape[0]):
        nv = nodev[e]
        s = 0.0
        for k in range(8):
            for l in range(8):
                s += M[k, l] * (nv[k, 0] * nv[l, 0] + nv[k, 1] * nv[l, 1] + nv[k, 2] * nv[l, 2])
        t += s * mass * nucell
        massone = mass * nucell
        for k in range(8):
            for l in range(8):
                for q, (a, b) in enumerate(((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))):
                    tv[q] += massone * M[k, l] * nv[k, a] * nv[l, b]
    dof = 3.0 * (v.shape[0] + nucell * nodev.shape[0])
    tfactor = MVV2E / (dof * BOLTZ) if dof > 0 else 0.0
    temp = t * tfactor
    ke = temp * (0.5 * dof * BOLTZ)
    prd = np.asarray(boxhi, dtype=np.float64) - np.asarray(boxlo, dtype=np.float64)
    vol = prd[0] * prd[1] * prd[2]
    inv_volume = 1.0 / vol
    nk = NKTV2P[units]
    w = np.asarray(virial, dtype=np.float64)
    out = {"temp": temp, "ke": ke, "pe": float(energy), "etotal": float(energy) + ke,
           "press": (dof * BOLTZ * temp + w[0] + w[1] + w[2]) / 3.0 * inv_volume * nk, "vol": vol}
    for q, k in enumerate(("pxx", "pyy", "pzz", "pxy", "pxz", "pyz")):
        out[k] = (tv[q] * MVV2E + w[q]) * inv_volume * nk
    return out


# ------------------------------------------------------------------ langevin

FTM2V = 1.0 / 1.0364269e-4    # update.cpp:164 (metal)


class RanMars:
    """The reference's uniform generator (random_mars.cpp:23-90): F. James's
    RANMAR (Comp. Phys. Comm. 60, 329 (1990)), a lagged subtractive Fibonacci
    sequence (lags 97 and 33) combined with an arithmetic sequence, restated
    in integers: every value the reference handles is a multiple of 2^-24,
    so u[] holds 24-bit integers and ``uniform`` returns integer / 2^24, the
    same doubles exactly.  The constructor's warm-up draw is kept."""

    C0, CD, CM = 362436, 7654321, 16777213
    MASK = (1 << 24) - 1

    def __init__(self, seed: int):
        if seed <= 0 or seed > 900000000:
            raise ValueError("Invalid seed for Marsaglia random # generator")
        ij = (seed - 1) // 30082
        kl = (seed - 1) - 30082 * ij
        i = (ij // 177) % 177 + 2
        j = ij % 177 + 2
        k = (kl // 169) % 178 + 1
        l = kl % 169
        self.u = [0] * 98
        for ii in range(1, 98):
            s = 0
            for jj in range(1, 25):
                m = ((i * j) % 179) * k % 179
                i, j, k = j, k, m
                l = (53 * l + 1) % 169
                if (l * m) % 64 >= 32:
                    s += 1 << (24 - jj)
            self.u[ii] = s
        self.c = self.C0
        self.i97, self.j97 = 97, 33
        self.uniform()

    def uniform_int(self) -> int:
        uni = (self.u[self.i97] - self.u[self.j97]) & self.MASK
        self.u[self.i97] = uni
        self.i97 = 97 if self.i97 == 1 else self.i97 - 1
        self.j97 = 97 if self.j97 == 1 else self.j97 - 1
        self.c -= self.CD
        if self.c < 0:
            self.c += self.CM
        return (uni - self.c) & self.MASK

    def uniform(self) -> float:
        return self.uniform_int() / 16777216.0


def langevin_post_force(f, nodef, v, nodev, rng: RanMars, mass: float, t_target: float, t_period: float,
                        dt: float, zero: bool, nucell: int = 729, npe: int = 8) -> None:
    """FixLangevin::post_force on one system, in place (fix_langevin.cpp:
    gfactors 266-273, atoms 538-612, element nodes 614-646, zero 650-672),
    with the reference's order of draws (atoms x y z, then each element's
    nodes x y z) and of floating-point operations.  ``count`` for ``zero``
    is atoms + elements (group.cpp:1068-1104), as in the reference."""
    gfactor1 = -mass / t_period / FTM2V
    gfactor2 = math.sqrt(mass) * math.sqrt(24.0 * BOLTZ / t_period / dt / MVV2E) / FTM2V
    gfactor1 *= 1.0 / 1.0
    gfactor2 *= 1.0 / math.sqrt(1.0)
    tsqrt = math.sqrt(t_target)
    fsum = [0.0, 0.0, 0.0]
    gamma1, gamma2 = gfactor1, gfactor2 * tsqrt
    for i in range(f.shape[0]):
        fran = [gamma2 * (rng.uniform() - 0.5) for _ in range(3)]
        for d in range(3):
            f[i, d] += gamma1 * v[i, d] + fran[d]
            fsum[d] += fran[d]
    gamma2 = gfactor2 * tsqrt / math.sqrt(nucell / npe)
    for e in range(nodef.shape[0]):
        for k in range(npe):
            fran = [gamma2 * (rng.uniform() - 0.5) for _ in range(3)]
            for d in range(3):
                nodef[e, k, d] += gamma1 * nodev[e, k, d] + fran[d]
                fsum[d] += fran[d]
    if zero:
        count = f.shape[0] + nodef.shape[0]
        fs = [s / count for s in fsum]
        for d in range(3):
            f[:, d] -= fs[d]
            nodef[:, :, d] -= fs[d]


def langevin_target(t_start: float, t_stop: float, step: int, begin: int, end: int) -> float:
    """FixLangevin::compute_target, CONSTANT style (fix_langevin.cpp:683-694)."""
    delta = float(step - begin)
    if delta != 0.0:
        delta /= end - begin
    return t_start + delta * (t_stop - t_start)


# ------------------------------------------------------------------ deform

DEFORM_STYLES = ("none", "final", "delta", "scale", "vel", "erate", "trate", "wiggle", "volume")
MY_2PI = 6.28318530717958647692


def deform_boxes(boxlo, boxhi, nevery: int, style, a, b, runs, dt: float = 0.001, first_step: int = 0):
    """Box edges under ``fix deform`` (orthogonal, units box) after the given
    consecutive runs, in the reference's order of operations: FixDeform::init
    per run (fix_deform.cpp:417-487), apply_strain / apply_volume /
    update_domain on steps divisible by N (fix_deform.cpp:698-707,
    1020-1240).  Returns (lo, hi) as lists."""
    lo, hi = [float(v) for v in boxlo], [float(v) for v in boxhi]
    st = [DEFORM_STYLES[int(s)] for s in style]
    link = {}
    for i in range(3):
        if st[i] != "volume":
            continue
        o1, o2 = (i + 1) % 3, (i + 2) % 3
        if st[o1] == "none":
            link[i] = ("one_from_one", o1, o2, None)
        elif st[o2] == "none":
            link[i] = ("one_from_one", o2, o1, None)
        elif st[o1] == "volume":
            link[i] = ("two_from_one", o1, o2, None)
        elif st[o2] == "volume":
            link[i] = ("two_from_one", o2, o1, None)
        else:
            link[i] = ("one_from_two", None, o1, o2)
    step = first_step
    for n in runs:
        begin, end = step, step + n
        delt = (end - begin) * dt
        los, his = lo[:], hi[:]
        vol0 = (hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2])
        lstop, hstop = lo[:], hi[:]
        for i in range(3):
            s, x, y = st[i], float(a[i]), float(b[i])
            if s == "final":
                lstop[i], hstop[i] = x, y
            elif s == "delta":
                lstop[i], hstop[i] = los[i] + x, his[i] + y
            elif s == "scale":
                lstop[i] = 0.5 * (los[i] + his[i]) - 0.5 * x * (his[i] - los[i])
                hstop[i] = 0.5 * (los[i] + his[i]) + 0.5 * x * (his[i] - los[i])
            elif s == "vel":
                lstop[i], hstop[i] = los[i] - 0.5 * delt * x, his[i] + 0.5 * delt * x
            elif s == "erate":
                lstop[i] = los[i] - 0.5 * delt * x * (his[i] - los[i])
                hstop[i] = his[i] + 0.5 * delt * x * (his[i] - los[i])
        for _ in range(n):
            step += 1
            if step % nevery:
                continue
            delta = float(step - begin)
            if delta != 0.0:
                delta /= end - begin
            t = (step - begin) * dt
            lt, ht = lo[:], hi[:]
            for i in range(3):
                s, x, y = st[i], float(a[i]), float(b[i])
                if s == "trate":
                    shift = 0.5 * ((his[i] - los[i]) * math.exp(x * t))
                    lt[i], ht[i] = 0.5 * (los[i] + his[i]) - shift, 0.5 * (los[i] + his[i]) + shift
                elif s == "wiggle":
                    shift = 0.5 * x * math.sin(MY_2PI * t / y)
                    lt[i], ht[i] = los[i] - shift, his[i] + shift
                elif s in ("final", "delta", "scale", "vel", "erate"):
                    lt[i] = los[i] + delta * (lstop[i] - los[i])
                    ht[i] = his[i] + delta * (hstop[i] - his[i])
            for i in range(3):
                if i not in link:
                    continue
                kind, fixed, d1, d2 = link[i]
                if kind == "one_from_one":
                    shift = 0.5 * (vol0 / (ht[d1] - lt[d1]) / (his[fixed] - los[fixed]))
                elif kind == "one_from_two":
                    shift = 0.5 * (vol0 / (ht[d1] - lt[d1]) / (ht[d2] - lt[d2]))
                else:
                    shift = 0.5 * math.sqrt(vol0 * (his[i] - los[i]) / (ht[d1] - lt[d1]) / (his[fixed] - los[fixed]))
                lt[i], ht[i] = 0.5 * (los[i] + his[i]) - shift, 0.5 * (los[i] + his[i]) + shift
            for i in range(3):
                if st[i] != "none":
                    lo[i], hi[i] = lt[i], ht[i]
    return lo, hi


def read_thermo(log: str, columns=THERMO_COLUMNS) -> np.ndarray:
    """Rows of the reference's thermo output (``Step`` plus ``columns``) from
    a run's screen log, one row per printed step."""
    rows = []
    lines = log.splitlines()
    for n, line in enumerate(lines):
        head = line.split()
        if head[:1] != ["Step"] or tuple(head[1:]) != tuple(columns):
            continue
        for row in lines[n + 1:]:
            parts = row.split()
            if len(parts) != len(columns) + 1:
                break
            try:
                rows.append([float(p) for p in parts])
            except ValueError:
                break
    return np.array(rows, dtype=np.float64).reshape(-1, len(columns) + 1)


# ------------------------------------------------------- reference read-outs

def read_dump(path: str) -> dict:
    """Parse ``oracle_dump`` output: atoms sorted by tag, nodes by (tag, node)."""
    out = {}
    with open(path) as f:
        lines = f.read().splitlines()
    i = 0
    while i < len(lines):
        ln = lines[i]
        if ln.startswith("#"):
            i += 1
            continue
        w = ln.split()
        if w[0] == "step":
            out["step"] = int(w[1])
        elif w[0] == "box":
            out["box"] = np.array([float(t) for t in w[1:]])
        elif w[0] == "natoms":
            out["natoms"], out["nelements"] = int(w[1]), int(w[3])
        elif w[0] == "energy":
            out["energy"] = float(w[1])
        elif w[0] == "virial":
            out["virial"] = np.array([float(t) for t in w[1:]])
        elif w[0] == "atoms":
            n = out["natoms"]
            a = np.array(" ".join(lines[i + 1:i + 1 + n]).split(), dtype=np.float64).reshape(n, 17)
            out["atoms"] = a
            i += n
        elif w[0] == "nodes":
            n = out["nelements"] * 8
            a = np.array(" ".join(lines[i + 1:i + 1 + n]).split(), dtype=np.float64).reshape(n, 21)
            out["nodes"] = a
            i += n
        i += 1
    a = out["atoms"]
    out["x"], out["v"], out["f"] = a[:, 1:4], a[:, 4:7], a[:, 7:10]
    out["eatom"], out["vatom"] = a[:, 10], a[:, 11:17]
    nd = out["nodes"]
    ne = out["nelements"]
    out["nodex"] = nd[:, 2:5].reshape(ne, 8, 3)
    out["nodev"] = nd[:, 5:8].reshape(ne, 8, 3)
    out["nodef"] = nd[:, 8:11].reshape(ne, 8, 3)
    out["gaussf_at_node"] = nd[:, 11:14].reshape(ne, 8, 3)
    out["enode"] = nd[:, 14].reshape(ne, 8)
    out["vnode"] = nd[:, 15:21].reshape(ne, 8, 6)
    return out


def read_dump_binary(path: str) -> dict:
    """Parse ``oracle_dump FILE state|compute binary`` (oracle_dump.cpp: the
    magic, 16 float64 header values, then 17-value atom rows and 21-value
    node rows) into the dictionary of :func:`read_dump`."""
    raw = np.fromfile(path, dtype=np.uint8)
    if raw[:8].tobytes() != b"CACODMP1":
        raise ValueError(f"{path}: not a binary oracle dump")
    v = raw[8:].view(np.float64)
    out = {"step": int(v[0]), "box": v[1:7].copy(), "natoms": int(v[7]), "nelements": int(v[8]),
           "energy": float(v[9]), "virial": v[10:16].copy()}
    na, ne = out["natoms"], out["nelements"]
    a = v[16:16 + 17 * na].reshape(na, 17)
    nd = v[16 + 17 * na:16 + 17 * na + 21 * 8 * ne].reshape(8 * ne, 21)
    out["atoms"], out["nodes"] = a, nd
    out["x"], out["v"], out["f"] = a[:, 1:4], a[:, 4:7], a[:, 7:10]
    out["eatom"], out["vatom"] = a[:, 10], a[:, 11:17]
    out["nodex"] = nd[:, 2:5].reshape(ne, 8, 3)
    out["nodev"] = nd[:, 5:8].reshape(ne, 8, 3)
    out["nodef"] = nd[:, 8:11].reshape(ne, 8, 3)
    out["gaussf_at_node"] = nd[:, 11:14].reshape(ne, 8, 3)
    out["enode"] = nd[:, 14].reshape(ne, 8)
    out["vnode"] = nd[:, 15:21].reshape(ne, 8, 6)
    return out


def read_neigh(path: str, natoms: int) -> np.ndarray:
    """Parse ``oracle_dump_neigh`` output into sorted int64 rows
    (i_site, kind, idx, site, sx, sy, sz) in the restatement's numbering:
    atoms by tag-1, Gauss points at natoms + 8*(etag-1) + igcell."""
    rows = []
    cur = None
    with open(path) as f:
        for ln in f:
            if ln[0] == "I":
                _, kind, tag, site, _n = ln.split()
                kind, tag, site = int(kind), int(tag), int(site)
                cur = tag - 1 if kind == 0 else natoms + 8 * (tag - 1) + site
            elif ln[0] == "J":
                _, kind, tag, site, sx, sy, sz = ln.split()
                rows.append((cur, int(kind), int(tag) - 1, int(site), int(sx), int(sy), int(sz)))
    a = np.array(rows, dtype=np.int64).reshape(-1, 7)
    order = np.lexsort(a.T[::-1])
    return a[order]


def read_neigh_binary(path: str) -> np.ndarray:
    """Parse ``oracle_dump_neigh FILE binary`` output (rows of 7 int32 written
    in sorted order) into the int64 rows of ``read_neigh``."""
    a = np.fromfile(path, dtype="<i4").reshape(-1, 7).astype(np.int64)
    order = np.lexsort(a.T[::-1])
    return a[order]


def run_reference(workdir: str, script: str, exe: str = REF_EXE, timeout: float = 900.0) -> str:
    """Run the reference executable on ``script`` (a file in ``workdir``)."""
    r = subprocess.run([exe, "-in", script], cwd=workdir, capture_output=True, text=True,
                       timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"reference run failed ({r.returncode}):\n{r.stdout[-3000:]}\n{r.stderr[-3000:]}")
    return r.stdout
