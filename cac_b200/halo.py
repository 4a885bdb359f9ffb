"""Spatial decomposition of one CAC system over ranks: slabs along one box
axis, one context per rank, a forward halo of positions every step.

The reference decomposes space over MPI ranks and exchanges halos by
messages (comm_brick.cpp:561-740: forward x and nodex of ghosts before the
force evaluation, reverse f and gaussf of ghosts after it with newton on;
pair_eam.cpp:1036-1158: reverse rho and forward F' between its two passes).
Here each rank holds its own sites plus ghost copies of every site its
force evaluation needs, and evaluates forces over full lists:

* the force on an owned site is the sum over its full list, so it is
  complete on the owning rank and nothing is folded back (no reverse halo
  of f or gaussf);
* for EAM the ghost shell is two neighbour radii deep: the density, and so
  F', of every ghost that an owned site's force reads is complete on the
  rank itself (the sites within one radius of the owned ones have their
  whole neighbourhood locally), so the two EAM messages between the passes
  become one deeper shell;
* one forward message per step carries the owners' new positions (atoms and
  element nodes) to the ghosts' holders after the drift, before the forces;
  a ghost's velocity and force are never used.

Every `every` steps (the list rebuild of ``neigh_modify every N check no``)
the owned states are gathered, wrapped into the box as Domain::pbc wraps them
(domain.cpp:526-720) and split again, so sites that crossed a slab boundary
change owner (the reference's exchange, comm_brick.cpp:758-944).  Each
rank's context holds a box that is the real box across the slab axis and
open along it (wide enough that no periodic image along the axis comes
within a neighbour radius), so ghosts beyond the global periodic boundary
are carried as shifted copies, as the reference's ghosts are.

Ranks talk through a communicator object: ``TorchComm`` over
torch.distributed (NCCL between GPUs, gloo on the CPU) or ``LocalComm``
(ranks in one process, stepped one after another).  Force evaluation and
integration run in a backend: ``EngineBackend`` (a cacb200 context on the
rank's GPU; the product path) or any object with the same methods.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np


# ------------------------------------------------------------ periodic wrap

def wrap_atoms(x: np.ndarray, lo, hi) -> None:
    """Domain::pbc for atoms (domain.cpp:562-630), in place, in the same
    floating-point steps as the device's wrap."""
    for d in range(3):
        L = hi[d] - lo[d]
        c = x[:, d]
        below = c < lo[d]
        c[below] = c[below] + L
        above = c >= hi[d]
        c[above] = np.maximum(c[above] - L, lo[d])


def element_centres(nodex: np.ndarray) -> np.ndarray:
    """Element centres as ElementVecCAC::update_center_coord forms them
    (element_vec_cac.cpp:3740-3765): nodes summed in order, divided by 8."""
    s = nodex[:, 0, :].copy()
    for k in range(1, 8):
        s = s + nodex[:, k, :]
    return s / 8.0


def wrap_elements(nodex: np.ndarray, lo, hi) -> None:
    """Domain::pbc for elements (domain.cpp:645-720 with
    update_node_coord): an element whose centre left the box moves with all
    its nodes by the centre's shift, in place."""
    if nodex.shape[0] == 0:
        return
    for d in range(3):
        L = hi[d] - lo[d]
        s = nodex[:, 0, d].copy()
        for k in range(1, 8):
            s = s + nodex[:, k, d]
        c = s / 8.0
        c2 = c.copy()
        below = c2 < lo[d]
        c2[below] = c2[below] + L
        above = c2 >= hi[d]
        c2[above] = np.maximum(c2[above] - L, lo[d])
        moved = below | above
        if moved.any():
            sh = c2[moved] - s[moved] / 8.0
            nodex[moved, :, d] = nodex[moved, :, d] + sh[:, None]


# ------------------------------------------------------------------- plan

@dataclass
class RankPart:
    """One rank's share: owned sites and ghost copies (global index and
    periodic shift along the slab axis), and the rank's context box."""
    own_atoms: np.ndarray
    own_elems: np.ndarray
    ghost_atoms: np.ndarray        # global indices
    ghost_atom_shift: np.ndarray   # -1, 0, +1 box lengths along the axis
    ghost_elems: np.ndarray
    ghost_elem_shift: np.ndarray
    boxlo: np.ndarray
    boxhi: np.ndarray

    @property
    def natoms(self) -> int:
        return len(self.own_atoms) + len(self.ghost_atoms)

    @property
    def nelements(self) -> int:
        return len(self.own_elems) + len(self.ghost_elems)


class SlabPlan:
    """Slabs of equal width along `axis`; ghosts within `hops` neighbour
    radii (cutneigh = cutoff + skin) of a rank's owned sites, with a margin
    of `margin` (default: the skin) for the moves between re-splits."""

    def __init__(self, boxlo, boxhi, nranks: int, cutneigh: float, hops: int = 1, axis: Optional[int] = None,
                 margin: float = 0.0):
        self.lo = np.asarray(boxlo, dtype=np.float64).copy()
        self.hi = np.asarray(boxhi, dtype=np.float64).copy()
        L = self.hi - self.lo
        self.axis = int(np.argmax(L)) if axis is None else int(axis)
        self.n = int(nranks)
        self.cut = float(cutneigh)
        self.hops = int(hops)
        self.margin = float(margin)
        self.L = float(L[self.axis])
        self.edges = self.lo[self.axis] + self.L * np.arange(self.n + 1) / self.n
        self.edges[-1] = self.hi[self.axis]

    def owner(self, z: np.ndarray) -> np.ndarray:
        """Rank owning a coordinate along the axis (inside the box)."""
        r = np.searchsorted(self.edges, z, side="right") - 1
        return np.clip(r, 0, self.n - 1)

    def split(self, x: np.ndarray, nodex: np.ndarray) -> List[RankPart]:
        """Every rank's share of the wrapped global state (every rank
        computes all shares, so no message is needed to agree on them)."""
        a = self.axis
        za = x[:, a] if len(x) else np.zeros(0)
        cen = element_centres(nodex)[:, a] if len(nodex) else np.zeros(0)
        emin = nodex[:, :, a].min(axis=1) if len(nodex) else np.zeros(0)
        emax = nodex[:, :, a].max(axis=1) if len(nodex) else np.zeros(0)
        aown = self.owner(za)
        eown = self.owner(cen)
        parts = []
        for r in range(self.n):
            s_lo, s_hi = self.edges[r], self.edges[r + 1]
            reg_lo, reg_hi = s_lo, s_hi
            sel_a = {}
            sel_e = {}
            for _ in range(self.hops):
                A0, A1 = reg_lo - self.cut - self.margin, reg_hi + self.cut + self.margin
                nlo, nhi = reg_lo, reg_hi
                for sh in (-1, 0, 1):
                    zs = za + sh * self.L
                    ma = (zs >= A0) & (zs < A1)
                    sel_a[sh] = ma if sh not in sel_a else (sel_a[sh] | ma)
                    me = (emax + sh * self.L >= A0) & (emin + sh * self.L <= A1)
                    sel_e[sh] = me if sh not in sel_e else (sel_e[sh] | me)
                    if ma.any():
                        nlo, nhi = min(nlo, zs[ma].min()), max(nhi, zs[ma].max())
                    if me.any():
                        nlo = min(nlo, (emin[me] + sh * self.L).min())
                        nhi = max(nhi, (emax[me] + sh * self.L).max())
                reg_lo, reg_hi = nlo, nhi
            own_a = np.nonzero(aown == r)[0]
            own_e = np.nonzero(eown == r)[0]
            ga, gas, ge, ges = [], [], [], []
            for sh in (-1, 0, 1):
                ia = np.nonzero(sel_a[sh])[0]
                ie = np.nonzero(sel_e[sh])[0]
                if sh == 0:
                    ia = ia[aown[ia] != r]
                    ie = ie[eown[ie] != r]
                ga.append(ia)
                gas.append(np.full(len(ia), sh, dtype=np.int64))
                ge.append(ie)
                ges.append(np.full(len(ie), sh, dtype=np.int64))
            ga, gas = np.concatenate(ga), np.concatenate(gas)
            ge, ges = np.concatenate(ge), np.concatenate(ges)
            # the context's box: the real box across the axis, open along it
            # (no periodic image along the axis within a neighbour radius of
            # any site the rank holds, for the moves until the next split)
            ext_lo, ext_hi = s_lo, s_hi
            if len(ga):
                zg = za[ga] + gas * self.L
                ext_lo, ext_hi = min(ext_lo, zg.min()), max(ext_hi, zg.max())
            if len(ge):
                ext_lo = min(ext_lo, (emin[ge] + ges * self.L).min())
                ext_hi = max(ext_hi, (emax[ge] + ges * self.L).max())
            if len(own_e):
                ext_lo = min(ext_lo, emin[own_e].min())
                ext_hi = max(ext_hi, emax[own_e].max())
            pad = 2.0 * self.cut + self.margin + 1.0
            blo, bhi = self.lo.copy(), self.hi.copy()
            blo[a], bhi[a] = ext_lo - pad, ext_hi + pad
            parts.append(RankPart(own_a, own_e, ga, gas, ge, ges, blo, bhi))
        return parts


# ----------------------------------------------------------- communicators

class LocalComm:
    """All ranks in one process: messages are array copies."""

    def __init__(self, nranks: int):
        self.size = nranks

    def exchange(self, sends):
        """sends[src][dst] -> arrays; returns recvs[dst][src]."""
        return [[sends[src][dst] for src in range(self.size)] for dst in range(self.size)]


class TorchComm:
    """One rank of a torch.distributed group (NCCL between GPUs, gloo on the
    CPU); arrays travel as float64 tensors on `device`, in point-to-point
    messages whose sizes both sides know from the shared plan."""

    def __init__(self, dist, device=None):
        self.dist = dist
        self.rank = dist.get_rank()
        self.size = dist.get_world_size()
        self.device = device

    def exchange_rank(self, sends, recv_sizes):
        """sends[dst] -> this rank's arrays for dst; recv_sizes[src] -> the
        number of float64 values arriving from src; returns recvs[src]."""
        import torch
        dist = self.dist
        reqs, bufs = [], [None] * self.size
        for peer in range(self.size):
            if peer == self.rank:
                continue
            if recv_sizes[peer]:
                bufs[peer] = torch.empty(recv_sizes[peer], dtype=torch.float64, device=self.device)
                reqs.append(dist.irecv(bufs[peer], src=peer))
        for peer in range(self.size):
            if peer == self.rank or sends[peer] is None or sends[peer].size == 0:
                continue
            t = torch.from_numpy(np.ascontiguousarray(sends[peer], dtype=np.float64).ravel())
            if self.device is not None:
                t = t.to(self.device)
            reqs.append(dist.isend(t, dst=peer))
        for q in reqs:
            q.wait()
        out = [None] * self.size
        for peer in range(self.size):
            if bufs[peer] is not None:
                out[peer] = bufs[peer].cpu().numpy()
        return out

    def all_gather(self, obj):
        res = [None] * self.size
        self.dist.all_gather_object(res, obj)
        return res


# ---------------------------------------------------------------- backend

class EngineBackend:
    """A rank's force evaluation and integration on its GPU: one cacb200
    context holding the rank's owned sites and ghosts."""

    def __init__(self, device: int, pair: str, setfl: Optional[str] = None, lj=(0.4093, 2.338, 5.5),
                 skin: float = 1.0):
        from cac_b200 import api
        self.api = api
        self.eng = api.Engine(device)
        self.pair, self.setfl, self.lj, self.skin = pair, setfl, lj, skin

    def upload(self, boxlo, boxhi, x, v, nodex, nodev, mass):
        from cac_b200.gen import System
        s = System(x=x, v=v, nodex=nodex, nodev=nodev, boxlo=np.asarray(boxlo), boxhi=np.asarray(boxhi),
                   mass=mass, meta={})
        self.eng.upload(s)
        if self.pair == "eam":
            self.eng.pair_eam(self.setfl)
        else:
            self.eng.pair_lj(*self.lj)
        self.eng.neighbor(self.skin, 0)

    def nve_initial(self, dt):
        self.eng._check(self.eng.lib.cacb200_nve_initial(self.eng.h, dt), "nve_initial")

    def nve_final(self, dt):
        self.eng._check(self.eng.lib.cacb200_nve_final(self.eng.h, dt), "nve_final")

    def forces(self):
        self.eng._check(self.eng.lib.cacb200_compute_forces(self.eng.h, 0, 0), "compute_forces")

    def positions(self):
        x, _, nx, _ = self.eng.state()
        return x, nx

    def set_positions(self, x, nodex):
        self.eng.set_state(x=x, nodex=nodex)

    def state(self):
        x, v, nx, nv = self.eng.state()
        f, nf, _ = self.eng.forces()
        return x, v, nx, nv, f, nf

    def close(self):
        self.eng.close()


# ------------------------------------------------------------------- run

@dataclass
class _Maps:
    """Forward-halo maps of one rank: what it sends to each peer (indices
    of its owned sites, in the order of the peer's ghosts) and where what it
    receives goes (its ghost slots), with the periodic shift to apply."""
    send_atoms: list = field(default_factory=list)   # [peer] -> owned local atom indices
    send_elems: list = field(default_factory=list)
    recv_atoms: list = field(default_factory=list)   # [peer] -> (ghost local indices, shifts)
    recv_elems: list = field(default_factory=list)


class HaloRun:
    """Velocity Verlet of one system split over ranks (see the module
    docstring).  `comm` is a LocalComm (then `backends` lists one backend per
    rank and `rank` is ignored) or a TorchComm (one backend, this rank's)."""

    def __init__(self, comm, backends, system, cutneigh: float, every: int = 10, hops: int = 1,
                 axis: Optional[int] = None, margin: Optional[float] = None, skin: float = 1.0):
        self.comm = comm
        self.local = isinstance(comm, LocalComm)
        self.backends = backends if self.local else [backends]
        self.nr = comm.size
        self.rank = None if self.local else comm.rank
        self.every = every
        self.mass = float(system.mass)
        self.lo = np.asarray(system.boxlo, dtype=np.float64).copy()
        self.hi = np.asarray(system.boxhi, dtype=np.float64).copy()
        self.plan = SlabPlan(self.lo, self.hi, self.nr, cutneigh, hops, axis, skin if margin is None else margin)
        self.step_count = 0
        g = (np.array(system.x, dtype=np.float64), np.array(system.v, dtype=np.float64),
             np.array(system.nodex, dtype=np.float64).reshape(-1, 8, 3),
             np.array(system.nodev, dtype=np.float64).reshape(-1, 8, 3))
        self._split(*g)
        for k in self._ranks():
            self.backends[self._bi(k)].forces()

    # ranks this process drives
    def _ranks(self):
        return range(self.nr) if self.local else [self.rank]

    def _bi(self, r):
        return r if self.local else 0

    def _split(self, x, v, nodex, nodev):
        wrap_atoms(x, self.lo, self.hi)
        wrap_elements(nodex, self.lo, self.hi)
        self.parts = self.plan.split(x, nodex)
        a = self.plan.axis
        L = self.plan.L
        for r in self._ranks():
            p = self.parts[r]
            xs = np.concatenate([x[p.own_atoms], x[p.ghost_atoms]])
            if len(p.ghost_atoms):
                xs[len(p.own_atoms):, a] += p.ghost_atom_shift * L
            nxs = np.concatenate([nodex[p.own_elems], nodex[p.ghost_elems]])
            if len(p.ghost_elems):
                nxs[len(p.own_elems):, :, a] += (p.ghost_elem_shift * L)[:, None]
            vs = np.concatenate([v[p.own_atoms], v[p.ghost_atoms]])
            nvs = np.concatenate([nodev[p.own_elems], nodev[p.ghost_elems]])
            self.backends[self._bi(r)].upload(p.boxlo, p.boxhi, xs, vs, nxs, nvs, self.mass)
        self.maps = {r: self._maps_of(r) for r in self._ranks()}

    def _maps_of(self, r):
        """Send and receive maps of rank r from the shared plan."""
        m = _Maps()
        parts = self.parts
        # local index of each global site within its owner
        aown_pos, eown_pos = {}, {}
        for o, p in enumerate(parts):
            aown_pos.update({int(g): (o, k) for k, g in enumerate(p.own_atoms)})
            eown_pos.update({int(g): (o, k) for k, g in enumerate(p.own_elems)})
        for peer in range(self.nr):
            # what r sends to peer: r's owned sites among peer's ghosts, in peer's ghost order
            q = parts[peer]
            sa = [aown_pos[int(g)][1] for g in q.ghost_atoms if aown_pos[int(g)][0] == r]
            se = [eown_pos[int(g)][1] for g in q.ghost_elems if eown_pos[int(g)][0] == r]
            m.send_atoms.append(np.array(sa, dtype=np.int64))
            m.send_elems.append(np.array(se, dtype=np.int64))
            # what r receives from peer: r's ghosts owned by peer
            p = parts[r]
            na_own, ne_own = len(p.own_atoms), len(p.own_elems)
            ka = [i for i, g in enumerate(p.ghost_atoms) if aown_pos[int(g)][0] == peer]
            ke = [i for i, g in enumerate(p.ghost_elems) if eown_pos[int(g)][0] == peer]
            m.recv_atoms.append((na_own + np.array(ka, dtype=np.int64), p.ghost_atom_shift[ka]))
            m.recv_elems.append((ne_own + np.array(ke, dtype=np.int64), p.ghost_elem_shift[ke]))
        return m

    def _forward(self):
        """Owners' positions to their ghosts (atoms and element nodes)."""
        a, L = self.plan.axis, self.plan.L
        pos = {r: self.backends[self._bi(r)].positions() for r in self._ranks()}
        sends = {}
        for r in self._ranks():
            x, nx = pos[r]
            m = self.maps[r]
            sends[r] = [np.concatenate([x[m.send_atoms[q]].ravel(), nx[m.send_elems[q]].ravel()])
                        for q in range(self.nr)]
        if self.local:
            recvs = {r: [sends[src][r] for src in range(self.nr)] for r in self._ranks()}
        else:
            r = self.rank
            m = self.maps[r]
            sizes = [3 * len(m.recv_atoms[q][0]) + 24 * len(m.recv_elems[q][0]) for q in range(self.nr)]
            got = self.comm.exchange_rank([None if q == r else sends[r][q] for q in range(self.nr)], sizes)
            got[r] = sends[r][r]   # own periodic copies
            recvs = {r: got}
        for r in self._ranks():
            x, nx = pos[r]
            m = self.maps[r]
            for q in range(self.nr):
                ia, sa = m.recv_atoms[q]
                ie, se = m.recv_elems[q]
                buf = recvs[r][q]
                if buf is None or (len(ia) == 0 and len(ie) == 0):
                    continue
                xa = buf[:3 * len(ia)].reshape(-1, 3).copy()
                xe = buf[3 * len(ia):].reshape(-1, 8, 3).copy()
                xa[:, a] += sa * L
                xe[:, :, a] += (se * L)[:, None]
                x[ia] = xa
                nx[ie] = xe
            self.backends[self._bi(r)].set_positions(x, nx)

    def gather(self):
        """The global state of the owned sites (x, v, nodex, nodev, f, nodef),
        in the global order, on every rank."""
        own = {}
        for r in self._ranks():
            p = self.parts[r]
            x, v, nx, nv, f, nf = self.backends[self._bi(r)].state()
            na, ne = len(p.own_atoms), len(p.own_elems)
            own[r] = (p.own_atoms, p.own_elems, x[:na], v[:na], nx[:ne], nv[:ne], f[:na], nf[:ne])
        if self.local:
            pieces = [own[r] for r in range(self.nr)]
        else:
            pieces = self.comm.all_gather(own[self.rank])
        na = sum(len(p[0]) for p in pieces)
        ne = sum(len(p[1]) for p in pieces)
        out = [np.zeros((na, 3)), np.zeros((na, 3)), np.zeros((ne, 8, 3)), np.zeros((ne, 8, 3)),
               np.zeros((na, 3)), np.zeros((ne, 8, 3))]
        for ia, ie, x, v, nx, nv, f, nf in pieces:
            out[0][ia], out[1][ia], out[4][ia] = x, v, f
            out[2][ie], out[3][ie], out[5][ie] = nx, nv, nf
        return tuple(out)

    def step(self, dt: float):
        """One velocity-Verlet step (fix_nve.cpp:62-219) of the whole system."""
        for r in self._ranks():
            self.backends[self._bi(r)].nve_initial(dt)
        self.step_count += 1
        if self.every and self.step_count % self.every == 0:
            # rebuild step: owners gathered, wrapped and split again
            x, v, nx, nv, _, _ = self.gather()
            self._split(x, v, nx, nv)
        else:
            self._forward()
        for r in self._ranks():
            b = self.backends[self._bi(r)]
            b.forces()
            b.nve_final(dt)

    def run(self, nsteps: int, dt: float):
        for _ in range(nsteps):
            self.step(dt)
