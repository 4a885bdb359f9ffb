"""Seeded builder for synthetic CAC systems (atoms + 8-node rhombohedral elements).

Geometry
--------
All sites lie on one FCC lattice in the orientation of the reference's
``lattice pri/fcc`` (``lattice.cpp:46,144,213``): nearest-neighbour distance
``b = a/sqrt(2)`` and primitive vectors

    A1 = b (1, 0, 0)
    A2 = b (1/2, sqrt(3)/2, 0)
    A3 = b (1/2, sqrt(3)/6, sqrt(2/3))

so x is [1-10], y is [11-2] and z is [111]; atomic layers are ``b*sqrt(2/3)``
apart along z and stack ABC.

An element spans 8 primitive vectors per edge (``ncell = 9`` lattice sites per
edge, 729 sites), with nodes in the Hex order of the reference
(``element_vec_cac.cpp:1740-1770``): node 0 at the origin, 1 = +8A1,
2 = +8A1+8A2, 3 = +8A2, 4..7 = 0..3 shifted by +8A3.  Elements do not share
sites; their origins form the superlattice 9A1, 9A2, 9A3.

The periodic box is ``Lx = 9 b nx``, ``Ly = 9 sqrt(3) b ny`` and
``Lz = NL b sqrt(2/3)`` with ``NL`` a multiple of 3, which makes atoms and
elements commensurate: a layer of ``2 nx ny`` elements covers 9 atomic layers
exactly, so the system is a perfect crystal with no gaps and no overlaps.
Along z the box holds ``[coarse region: le element layers]
[atomistic slab: la atomic layers][coarse region: le element layers]``.

Perturbations: every atom and node coordinate gets an independent seeded
uniform displacement in ``[-disp, +disp]`` (default ``0.01 a``); velocities
are Maxwell-Boltzmann at ``T`` per component; an optional affine strain
``x -> (1 + strain) x`` is applied to positions and the box along x.

Output is the CAC data-file format read by ``read_data``
(``read_data.cpp:339-367``; element lines ``element_vec_cac.cpp:300-336``,
node lines ``:354-395``, node velocity lines ``:337-352``) and the setfl
format read by ``pair_style eam/alloy`` (``pair_eam_alloy.cpp:100-240``).
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np

# metal units (update.cpp:161-164)
BOLTZ = 8.617343e-5
MVV2E = 1.0364269e-4
FTM2V = 1.0 / 1.0364269e-4

NCELL = 9
NUCELL = NCELL ** 3
NPE = 8

# Hex node corners in (i, j, k) lattice steps along (A1, A2, A3)
HEX_CORNERS = np.array(
    [[0, 0, 0], [8, 0, 0], [8, 8, 0], [0, 8, 0],
     [0, 0, 8], [8, 0, 8], [8, 8, 8], [0, 8, 8]], dtype=np.int64)


@dataclasses.dataclass
class System:
    """A CAC system in the reference's own ordering (atoms, then elements)."""

    boxlo: np.ndarray            # (3,)
    boxhi: np.ndarray            # (3,)
    x: np.ndarray                # (na, 3) atom positions
    v: np.ndarray                # (na, 3) atom velocities
    nodex: np.ndarray            # (ne, 8, 3) node positions (unwrapped, near the centre)
    nodev: np.ndarray            # (ne, 8, 3) node velocities
    mass: float = 63.546
    lattice_a: float = 3.615
    meta: dict = dataclasses.field(default_factory=dict)

    @property
    def natoms(self) -> int:
        return int(self.x.shape[0])

    @property
    def nelements(self) -> int:
        return int(self.nodex.shape[0])

    @property
    def nsites(self) -> int:
        """Force sites: atoms plus the 8 Gauss points (= nodes) of each element."""
        return self.natoms + NPE * self.nelements

    def centers(self) -> np.ndarray:
        """Element centres as the reference computes them
        (``ElementVecCAC::update_center_coord``, ``element_vec_cac.cpp:3740-3765``):
        a sequential sum over nodes divided by npe then by apc."""
        c = np.zeros((self.nelements, 3))
        for k in range(NPE):
            c = c + self.nodex[:, k, :]
        return c / NPE / 1


def primitive_vectors(a: float) -> np.ndarray:
    b = a / math.sqrt(2.0)
    return np.array([[b, 0.0, 0.0],
                     [0.5 * b, math.sqrt(3.0 / 4.0) * b, 0.0],
                     [0.5 * b, math.sqrt(1.0 / 12.0) * b, math.sqrt(2.0 / 3.0) * b]])


def build_slab(nx: int, ny: int, le: int, la: int, *, a: float = 3.615,
               mass: float = 63.546, temperature: float = 10.0,
               disp: Optional[float] = None, strain: float = 0.0,
               seed: int = 0) -> System:
    """Build ``[le element layers][la atomic layers][le element layers]``.

    ``la`` must be a multiple of 3 (ABC stacking across the periodic boundary).
    Elements: ``2*nx*ny*le`` per coarse region.  Atoms: ``162*nx*ny*la``.
    """
    if la % 3 != 0:
        raise ValueError("la (atomic layers) must be a multiple of 3")
    if nx < 1 or ny < 1 or le < 0 or la < 0:
        raise ValueError("invalid slab dimensions")
    A = primitive_vectors(a)
    b = a / math.sqrt(2.0)
    dz = b * math.sqrt(2.0 / 3.0)
    Lx = NCELL * b * nx
    Ly = NCELL * math.sqrt(3.0) * b * ny
    NL = 2 * NCELL * le + la
    Lz = NL * dz
    # keep lattice planes away from the box faces
    origin = np.array([0.25 * b, 0.25 * b * math.sqrt(3.0) / 2.0, 0.5 * dz])
    boxlo = np.zeros(3)
    boxhi = np.array([Lx, Ly, Lz])

    def wrap_xy(p):
        q = p.copy()
        q[..., 0] -= np.floor((q[..., 0] - 0.0) / Lx) * Lx
        q[..., 1] -= np.floor((q[..., 1] - 0.0) / Ly) * Ly
        return q

    # ---- atoms: every lattice site of layers [9 le, 9 le + la)
    na_layer = 2 * (NCELL * nx) * (NCELL * ny)
    ii, jj = np.meshgrid(np.arange(NCELL * nx), np.arange(2 * NCELL * ny), indexing="ij")
    ii = ii.ravel()
    jj = jj.ravel()
    atoms = []
    for k in range(NCELL * le, NCELL * le + la):
        p = origin + ii[:, None] * A[0] + jj[:, None] * A[1] + k * A[2]
        atoms.append(wrap_xy(p))
    x = np.concatenate(atoms) if atoms else np.zeros((0, 3))
    assert x.shape[0] == na_layer * la

    # ---- elements: superlattice points 9(p A1 + q A2) + k0 A3
    pp, qq = np.meshgrid(np.arange(nx), np.arange(2 * ny), indexing="ij")
    pp = pp.ravel()
    qq = qq.ravel()
    corner_off = HEX_CORNERS @ A  # (8, 3)
    elems = []
    layer_starts = [NCELL * m for m in range(le)] + \
                   [NCELL * le + la + NCELL * m for m in range(le)]
    for k0 in layer_starts:
        o = origin + NCELL * (pp[:, None] * A[0] + qq[:, None] * A[1]) + k0 * A[2]
        o = wrap_xy(o)
        nodes = o[:, None, :] + corner_off[None, :, :]
        elems.append(nodes)
    nodex = np.concatenate(elems) if elems else np.zeros((0, 8, 3))

    rng = np.random.default_rng(seed)
    if disp is None:
        disp = 0.01 * a
    x = x + rng.uniform(-disp, disp, size=x.shape)
    nodex = nodex + rng.uniform(-disp, disp, size=nodex.shape)

    sigma = math.sqrt(BOLTZ * temperature / (mass * MVV2E)) if temperature > 0 else 0.0
    v = rng.normal(0.0, sigma, size=x.shape)
    nodev = rng.normal(0.0, sigma, size=nodex.shape)

    if strain != 0.0:
        s = 1.0 + strain
        x[:, 0] *= s
        nodex[:, :, 0] *= s
        boxhi[0] = boxlo[0] + (boxhi[0] - boxlo[0]) * s

    meta = dict(nx=nx, ny=ny, le=le, la=la, a=a, temperature=temperature,
                disp=disp, strain=strain, seed=seed, layers=NL)
    s = System(boxlo=boxlo, boxhi=boxhi, x=x, v=v, nodex=nodex, nodev=nodev,
               mass=mass, lattice_a=a, meta=meta)
    wrap_into_box(s)
    return s


def wrap_into_box(s: System) -> None:
    """Canonical periodic representation: atoms inside ``[lo, hi)``; each
    element moved as a whole so that its centre is inside the box.  This is
    the state the reference holds after ``read_data`` remaps element centres
    and shifts nodes with them (``element.cpp:533-700``, ``domain.cpp:1453``)."""
    L = s.boxhi - s.boxlo
    s.x[:] = s.x - np.floor((s.x - s.boxlo) / L) * L
    if s.nelements:
        c = s.centers()
        shift = -np.floor((c - s.boxlo) / L) * L
        s.nodex[:] = s.nodex + shift[:, None, :]


# -------------------------------------------------------------- named shapes

def lj_small(seed: int = 1) -> System:
    """LJ workload at the CPU-runnable scale: 4,374 atoms (9 layers of 486)
    between two coarse regions of 108 elements each (18 layers of 6; 216 total,
    6,102 atom+IP sites), 10 K."""
    return build_slab(3, 1, 18, 9, temperature=10.0, seed=seed)


def eam_1m(seed: int = 2) -> System:
    """EAM workload at scale: 1,049,760 atoms (162 layers of 6,480) plus 20,000
    elements (2 regions x 125 layers x 80), 1,209,760 atom+IP sites, 300 K."""
    return build_slab(8, 5, 125, 162, temperature=300.0, seed=seed)


def eam_small(seed: int = 5) -> System:
    """A quarter-height EAM slab for profiling captures: 272,160 atoms (42
    layers of 6,480) plus 5,120 elements (2 regions x 32 layers x 80), 313,120
    atom+IP sites, 300 K; still larger than the 126 MB L2 once lists exist."""
    return build_slab(8, 5, 32, 42, temperature=300.0, seed=seed)


def eam_4m_strained(seed: int = 3) -> System:
    """Mixed-precision workload: 4,179,600 atoms plus 100,000 elements under 3 %
    x-strain (nx=20, ny=10: 32,400 atoms per layer, 129 layers; 125 layers of
    400 elements per region; 4,979,600 atom+IP sites), 300 K."""
    return build_slab(20, 10, 125, 129, temperature=300.0, strain=0.03, seed=seed)


def replica(target_atoms: int, target_elements: int, *, temperature: float, strain: float,
            seed: int) -> System:
    """A slab with about ``target_atoms`` atoms and ``target_elements``
    elements: the cross-section (nx, ny >= 2, 1) is chosen so that at least
    3 atomic layers and 1 element layer per region fit both targets; the
    realised counts are multiples of the layer sizes."""
    nxy = max(2, min(target_atoms // 486, target_elements // 4))
    nx = max(2, int(math.ceil(math.sqrt(nxy))))
    ny = max(1, int(round(nxy / nx)))
    per_layer = 162 * nx * ny
    la = max(3, 3 * int(round(target_atoms / per_layer / 3.0)))
    le = max(1, int(round(target_elements / (4.0 * nx * ny))))
    return build_slab(nx, ny, le, la, temperature=temperature, strain=strain, seed=seed)


def replica_specs(n: int = 256, seed: int = 11, atoms=(2000, 64000), elements=(50, 2000),
                  temperature=(10.0, 500.0), strain=(0.0, 0.05)) -> List[tuple]:
    """(atom target, element target, temperature, x-strain, seed) of the
    replicas of ``replica_set``: targets log-uniform in the given ranges,
    temperature and strain uniform, every draw from one seeded generator in
    replica order (the first k specs of a longer set are the k of a shorter)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        ta = int(round(math.exp(rng.uniform(math.log(atoms[0]), math.log(atoms[1])))))
        te = int(round(math.exp(rng.uniform(math.log(elements[0]), math.log(elements[1])))))
        t = float(rng.uniform(*temperature))
        st = float(rng.uniform(*strain))
        out.append((ta, te, t, st, int(rng.integers(1 << 30))))
    return out


def replica_from_spec(spec: tuple) -> System:
    ta, te, t, st, s = spec
    return replica(ta, te, temperature=t, strain=st, seed=s)


def replica_set(n: int = 256, seed: int = 11, **ranges) -> List[System]:
    """Independent replicas for batched runs (``replica_specs``)."""
    return [replica_from_spec(sp) for sp in replica_specs(n, seed, **ranges)]


def tiny(seed: int = 7, temperature: float = 50.0) -> System:
    """1,458 atoms and 12 elements: fast parity cases.  ``nx = 3`` keeps the
    box wider than 1.5x the element bounding box in x, the reference's own
    condition for complete neighbour lists (``comm_brick.cpp:273-296``)."""
    return build_slab(3, 1, 1, 3, temperature=temperature, seed=seed)


# ------------------------------------------------------------------ writers

def _fmt(v: float) -> str:
    return repr(float(v))


def write_data(system: System, path: str, *, atom_type: int = 1) -> None:
    """Write ``system`` in the reference's data-file format (tags from 1)."""
    s = system
    lines = ["CAC data file written by cac_b200.gen", ""]
    lines.append(f"{s.natoms} atoms")
    lines.append(f"{s.nelements} elements")
    lines.append("1 atom types")
    lines.append("1 element types")
    lines.append("")
    for d, name in enumerate("xyz"):
        lines.append(f"{_fmt(s.boxlo[d])} {_fmt(s.boxhi[d])} {name}lo {name}hi")
    lines += ["", "Masses", "", f"1 {_fmt(s.mass)}", ""]
    lines += ["Element Types", "", f"1 Hex 1 {NCELL} {NCELL} {NCELL} 2 2 2", ""]
    if s.natoms:
        lines += ["Atoms", ""]
        lines += [f"{i + 1} {atom_type} {_fmt(p[0])} {_fmt(p[1])} {_fmt(p[2])}"
                  for i, p in enumerate(s.x)]
        lines += ["", "Velocities", ""]
        lines += [f"{i + 1} {_fmt(p[0])} {_fmt(p[1])} {_fmt(p[2])}"
                  for i, p in enumerate(s.v)]
        lines.append("")
    if s.nelements:
        c = s.centers()
        lines += ["Elements", ""]
        lines += [f"{e + 1} 1 {_fmt(p[0])} {_fmt(p[1])} {_fmt(p[2])}"
                  for e, p in enumerate(c)]
        lines += ["", "Nodes", ""]
        for e in range(s.nelements):
            for k in range(NPE):
                p = s.nodex[e, k]
                lines.append(f"{e + 1} {k + 1} 1 {atom_type} {_fmt(p[0])} {_fmt(p[1])} {_fmt(p[2])}")
        lines += ["", "Node Velocities", ""]
        for e in range(s.nelements):
            for k in range(NPE):
                p = s.nodev[e, k]
                lines.append(f"{e + 1} {k + 1} 1 {_fmt(p[0])} {_fmt(p[1])} {_fmt(p[2])}")
        lines.append("")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


# -------------------------------------------------------------- EAM tables

@dataclasses.dataclass
class EamParams:
    """Analytic EAM tabulated into a setfl file.

    phi(r) = A exp(-alpha (r/re - 1)) - B exp(-beta (r/re - 1))
    f(r)   = exp(-beta (r/re - 1))
    F(rho) = -E0 sqrt(rho)
    """

    A: float = 0.1
    B: float = 0.25
    alpha: float = 9.0
    beta: float = 4.5
    re: float = 2.556
    E0: float = 1.5
    cut: float = 5.0
    nr: int = 10000
    nrho: int = 10000
    rhomax: float = 50.0
    mass: float = 63.546

    @property
    def dr(self) -> float:
        return self.cut / (self.nr - 1)

    @property
    def drho(self) -> float:
        return self.rhomax / (self.nrho - 1)

    def tables(self):
        r = np.arange(self.nr) * self.dr
        rho = np.arange(self.nrho) * self.drho
        t = r / self.re - 1.0
        phi = self.A * np.exp(-self.alpha * t) - self.B * np.exp(-self.beta * t)
        frho = -self.E0 * np.sqrt(rho)
        rhor = np.exp(-self.beta * t)
        z2r = r * phi
        return frho, rhor, z2r


def write_setfl(params: EamParams, path: str, element: str = "Cu") -> None:
    """Write a one-element setfl file (values printed with full precision so that
    every reader parses the same doubles)."""
    frho, rhor, z2r = params.tables()
    out = ["analytic EAM tabulated by cac_b200.gen",
           f"phi=A exp(-alpha(r/re-1))-B exp(-beta(r/re-1)); f=exp(-beta(r/re-1)); F=-E0 sqrt(rho)",
           f"A={params.A} B={params.B} alpha={params.alpha} beta={params.beta} re={params.re} E0={params.E0}",
           f"1 {element}",
           f"{params.nrho} {_fmt(params.drho)} {params.nr} {_fmt(params.dr)} {_fmt(params.cut)}",
           f"29 {_fmt(params.mass)} 3.615 fcc"]
    for arr in (frho, rhor, z2r):
        for i in range(0, len(arr), 5):
            out.append(" ".join(_fmt(v) for v in arr[i:i + 5]))
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


@dataclasses.dataclass
class LjParams:
    epsilon: float = 0.4093
    sigma: float = 2.338
    cut: float = 5.5
