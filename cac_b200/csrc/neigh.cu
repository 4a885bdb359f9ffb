// Periodic wrap, cell binning and neighbour-list construction.
//
// Lists hold, for every i-site (atoms, then the 8 Gauss points of each
// element), the atoms and element lattice sites within cutneigh = cut + skin,
// with the periodic image of each neighbour.  Membership is decided in the
// reference's FP64 arithmetic, so the sets equal the reference's bit for bit:
//   atom j:           rsq of xi - (xj + s*L)          (npair_half_bin_newton.cpp:116-120)
//   lattice site j:   xi - sum_k N_k (xnode_k + s*L)  subtracted node by node
//                                                     (npair_half_bin_newton.cpp:194-200)
// with products and differences rounded separately (no FMA).
//
// Candidates come from two periodic cell grids instead of the reference's
// bin/stencil/sub-element walk: atoms from a grid of cell >= cutneigh with a
// 3x3x3 stencil (atoms: one block per chunk of 32 cell-sorted atoms, the
// atoms as lanes sharing broadcast candidate loads; Gauss points: one warp
// each, the lanes over the candidates), element sites
// from a grid over element centres of cell >= cutneigh + (centre-to-node
// radius + affine deviation), and for each candidate element only the lattice
// sites whose affine position can lie within cutneigh (a box in lattice-index
// space).  Both prunings are exact supersets, so they change cost, not
// membership.
//
// Full lists are written in their final form: an entry packs the neighbour's
// pair-table index (atoms by list slot) with its image; a site's entries
// inside the inner radius at build time fill its list from row 0 up, the
// others from row cap-1 down, so no pass reorders them.  Element-site entries
// are first written as lattice-site ids (the pair-table index of a lattice
// site is known only once every list has marked the sites it uses) and
// converted by k_remap_sites.  Half lists (read only by the list download)
// are written as raw entries and compacted by k_remap.
//
// Storage rules (the reference's, restated):
//   full  (npair_full_bin.cpp:23-358): every neighbour except the site itself.
//   half  (npair_half_bin_newton.cpp:25-392): an atom keeps atom j when j's
//         reference bin is in its upper half stencil, or in the same bin when j
//         is owned and later in order, or a ghost "above and to the right";
//         it keeps every lattice site.  A Gauss point keeps no atoms, every
//         non-Gauss lattice site, and a Gauss site once: owned (element i < j,
//         or same element and igcell < jgcell) or ghost with its element
//         centre above and to the right.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <tuple>
#include <type_traits>

#include "ctx.cuh"
#include "device.cuh"

namespace cacb200 {

namespace {

constexpr int KIND_SITE = 1 << 30;  // build-time entry flag: lattice site (gid = e*729+u)

// Replica lookup.  A single system uses OneRep (its descriptor is a kernel
// argument); a batch uses ManyRep (descriptor table plus per-site, per-element
// and per-cell replica indices).  The kernels are written once for both.
struct OneRep {
  Rep r;
  static constexpr bool many = false;
  __device__ __forceinline__ Rep site(int) const { return r; }
  __device__ __forceinline__ Rep elem(int) const { return r; }
  __device__ __forceinline__ Rep acell(int) const { return r; }
  __device__ __forceinline__ int elem_id(int) const { return 0; }
};
struct ManyRep {
  const Rep *reps;
  const int *site_rep, *elem_rep, *acell_rep;
  static constexpr bool many = true;
  __device__ __forceinline__ Rep site(int i) const { return reps[site_rep[i]]; }
  __device__ __forceinline__ Rep elem(int e) const { return reps[elem_rep[e]]; }
  __device__ __forceinline__ Rep acell(int c) const { return reps[acell_rep[c]]; }
  __device__ __forceinline__ int elem_id(int e) const { return elem_rep[e]; }
};

// ------------------------------------------------------------------ pbc

// Domain::pbc for owned atoms (domain.cpp:562-630)
template <class RP>
__global__ void k_pbc_atoms(double4 *xs, int na, RP P) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= na) return;
  const BoxD b = P.site(i).b;
  double4 p = xs[i];
  double *q = &p.x;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    double x = q[d];
    if (x < b.lo[d]) x += b.L[d];
    if (x >= b.hi[d]) {
      x -= b.L[d];
      x = fmax(x, b.lo[d]);
    }
    q[d] = x;
  }
  xs[i] = p;
}

// Element centre (ElementVecCAC::update_center_coord, element_vec_cac.cpp:3740-3765),
// Domain::pbc for elements (domain.cpp:645-720 with update_node_coord,
// element_vec_cac.cpp:3772-3785), then the geometry used by the candidate
// search: affine frame n0 + i a + j b + k c of the lattice sites, its inverse,
// the largest deviation of the trilinear nodes from that frame, and the
// centre-to-node radius.
//   eframe[e*EFR + 0..2]  n0
//   eframe[e*EFR + 3..11] rows of the inverse frame matrix
//   eframe[e*EFR + 12]    dmax
//   eframe[e*EFR + 13..21] frame vectors a, b, c (one lattice step each)
//   eframe[e*EFR + 22..24] norms of the inverse frame's rows (lattice steps
//                         per unit length along each index)
constexpr int EFR = 28;

template <class RP>
__global__ void k_elem_geom(double *nodex, int ne, RP P, double4 *ecenter, double *eframe,
                            unsigned long long *reach_bits, int *grew) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  double reach = 0.0;
  if (e < ne) {
    const Rep rp = P.elem(e);
    const BoxD b = rp.b;
    double *nx = nodex + (size_t)e * 24;
    double c[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      double s = 0.0;
      for (int k = 0; k < NPE; k++) s = __dadd_rn(s, nx[3 * k + d]);
      c[d] = s / NPE / 1;
    }
#pragma unroll
    for (int d = 0; d < 3; d++) {
      bool moved = false;
      if (c[d] < b.lo[d]) {
        c[d] += b.L[d];
        moved = true;
      }
      if (c[d] >= b.hi[d]) {
        c[d] -= b.L[d];
        c[d] = fmax(c[d], b.lo[d]);
        moved = true;
      }
      if (moved) {
        double s = 0.0;
        for (int k = 0; k < NPE; k++) s = __dadd_rn(s, nx[3 * k + d]);
        double sh = c[d] - s / NPE / 1;
        for (int k = 0; k < NPE; k++) nx[3 * k + d] += sh;
      }
    }
    double R = 0.0;
    for (int k = 0; k < NPE; k++) {
      double dx = nx[3 * k] - c[0], dy = nx[3 * k + 1] - c[1], dz = nx[3 * k + 2] - c[2];
      R = fmax(R, sqrt(dx * dx + dy * dy + dz * dz));
    }
    double n0[3], A[3][3];  // columns a, b, c
#pragma unroll
    for (int d = 0; d < 3; d++) {
      n0[d] = nx[d];
      A[d][0] = (nx[3 * 1 + d] - n0[d]) / (NC - 1);
      A[d][1] = (nx[3 * 3 + d] - n0[d]) / (NC - 1);
      A[d][2] = (nx[3 * 4 + d] - n0[d]) / (NC - 1);
    }
    double dmax = 0.0;
    for (int k = 0; k < NPE; k++) {
      double dev2 = 0.0;
#pragma unroll
      for (int d = 0; d < 3; d++) {
        double aff = n0[d] + (NC - 1) * (node_xi(k) * A[d][0] + node_eta(k) * A[d][1] +
                                         node_zeta(k) * A[d][2]);
        double t = nx[3 * k + d] - aff;
        dev2 += t * t;
      }
      dmax = fmax(dmax, sqrt(dev2));
    }
    // inverse of the 3x3 frame
    double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                 A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                 A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
    double id = 1.0 / det;
    double inv[3][3];
    inv[0][0] = (A[1][1] * A[2][2] - A[1][2] * A[2][1]) * id;
    inv[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) * id;
    inv[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) * id;
    inv[1][0] = (A[1][2] * A[2][0] - A[1][0] * A[2][2]) * id;
    inv[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) * id;
    inv[1][2] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) * id;
    inv[2][0] = (A[1][0] * A[2][1] - A[1][1] * A[2][0]) * id;
    inv[2][1] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) * id;
    inv[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) * id;
    double *fr = eframe + (size_t)e * EFR;
    fr[0] = n0[0];
    fr[1] = n0[1];
    fr[2] = n0[2];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
      for (int q = 0; q < 3; q++) fr[3 + 3 * r + q] = inv[r][q];
#pragma unroll
    for (int r = 0; r < 3; r++)
      fr[22 + r] = sqrt(inv[r][0] * inv[r][0] + inv[r][1] * inv[r][1] + inv[r][2] * inv[r][2]);
    fr[12] = dmax;
#pragma unroll
    for (int q = 0; q < 3; q++)
#pragma unroll
      for (int d = 0; d < 3; d++) fr[13 + 3 * q + d] = A[d][q];
    ecenter[e] = make_double4(c[0], c[1], c[2], R);
    reach = R + dmax;
    if (!(reach <= rp.reach_budget)) atomicExch(grew, 1);
    // per-replica maximum (non-negative doubles order like their bit patterns)
    if (RP::many) atomicMax(reach_bits + P.elem_id(e), (unsigned long long)__double_as_longlong(reach));
  }
  if (!RP::many) {
    for (int o = 16; o > 0; o >>= 1) reach = fmax(reach, __shfl_down_sync(0xffffffffu, reach, o));
    if ((threadIdx.x & 31) == 0) atomicMax(reach_bits, (unsigned long long)__double_as_longlong(reach));
  }
}

// ---------------------------------------------------------------- binning

__device__ __forceinline__ int grid_cell(const Grid &g, const BoxD &b, const double *w) {
  int c[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    int v = (int)((w[d] - b.lo[d]) * g.inv[d]);
    c[d] = min(max(v, 0), g.nc[d] - 1);
  }
  return (c[2] * g.nc[1] + c[1]) * g.nc[0] + c[0];
}

template <class RP>
__global__ void k_atom_keys(const double4 *xs, int na, RP P, int *key, int *idx) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= na) return;
  const Rep r = P.site(i);
  double4 p = xs[i];
  double w[3] = {p.x, p.y, p.z};
  key[i] = r.abase + grid_cell(r.ag, r.b, w);
  idx[i] = i;
}

template <class RP>
__global__ void k_elem_keys(const double4 *ecenter, int ne, RP P, int *key, int *idx) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const Rep r = P.elem(e);
  double4 p = ecenter[e];
  double w[3] = {p.x, p.y, p.z};
  key[e] = r.ebase + grid_cell(r.eg, r.b, w);
  idx[e] = e;
}

// near[c]: some cell of the 27-cell block around cell c (a single system's
// grid, periodic) holds an entry (element grid: an element; atom grid: an
// atom)
__global__ void k_ecell_near(const int *start, Grid g, unsigned char *near) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.ncell) return;
  const int cx = c % g.nc[0], cy = (c / g.nc[0]) % g.nc[1], cz = c / (g.nc[0] * g.nc[1]);
  bool any = false;
  for (int oz = -1; oz <= 1 && !any; oz++)
    for (int oy = -1; oy <= 1 && !any; oy++)
      for (int ox = -1; ox <= 1 && !any; ox++) {
        const int x = (cx + ox + g.nc[0]) % g.nc[0], y = (cy + oy + g.nc[1]) % g.nc[1],
                  z = (cz + oz + g.nc[2]) % g.nc[2];
        const int k = (z * g.nc[1] + y) * g.nc[0] + x;
        any = start[k + 1] > start[k];
      }
  near[c] = any ? 1 : 0;
}

// cell_start[c] = first sorted position with key >= c, for c in [0, ncell]
// (lower bound by binary search, one thread per cell)
__global__ void k_cell_start(const int *skey, int n, int ncell, int *start) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c > ncell) return;
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (skey[mid] < c) lo = mid + 1;
    else hi = mid;
  }
  start[c] = lo;
}

__global__ void k_gather_pos(const double4 *xs, const int *sidx, const int *skey, int n, double4 *out,
                             float4 *out32, int *atom_slot, int *slot_cell) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int i = sidx[k];
  atom_slot[i] = k;
  slot_cell[k] = skey[k];
  double4 p = xs[i];
  out32[k] = make_float4((float)p.x, (float)p.y, (float)p.z, __int_as_float(i));
  p.w = __longlong_as_double((long long)i);
  out[k] = p;
}

// -------------------------------------------------------------- the build

struct BuildArgs {
  const double4 *xs;          // atom positions (first na entries)
  const double *nodex;
  const double4 *ecenter;
  const double *eframe;
  const int *acell_start;
  const double4 *acell_pos;
  const float4 *acell_pos32;  // wrapped positions as floats, w = atom index bits
  const int *acell_of;        // [na] cell of each sorted atom (list slot)
  const int *ecell_start;
  const unsigned char *ecell_near;   // single systems: element cell has an element in its 27-cell block (else null)
  const unsigned char *acell_near;   // single systems: atom cell has an atom in its 27-cell block (else null)
  const int *ecell_elems;
  const int *atom_of_slot;    // list slot (cell-sorted position) -> atom index
  int *site_flag;             // [ne * 729] marks the lattice sites some full list references
  int na, ne, nsi, cap;
  RefBins rb;                 // single systems only (half lists)
  double cutneigh, cutneighsq;
  double cutforcesq;          // pairs inside the inner radius (force cutoff + margin) at build time go first
  int want_half;
  int *nbr_full;              // final full-list entries (atoms; element sites after k_remap_sites)
  int *num_in;                // per slot: entries in the front segment
  int2 *site_from;            // per slot: front / back rows before the element-site entries
  int *raw_full, *num_full;   // raw_full / img_full: element-site entries at their final rows
  unsigned char *img_full;
  int *raw_half, *num_half;
  unsigned char *img_half;
  int *overflow;              // [0] flag, [1] max count, [2] bad image
};

__device__ __forceinline__ int ref_bin1(const RefBins &rb, int d, double x) {
  int ix;
  if (x >= rb.hi[d]) ix = (int)((x - rb.hi[d]) * rb.inv[d]) + rb.nbin[d];
  else if (x >= rb.lo[d]) {
    ix = (int)((x - rb.lo[d]) * rb.inv[d]);
    ix = min(ix, rb.nbin[d] - 1);
  } else ix = (int)((x - rb.lo[d]) * rb.inv[d]) - 1;
  return ix;
}

// >0: q's reference bin is in p's upper half stencil; 0: same bin; <0 otherwise
__device__ __forceinline__ int ref_bin_order(const RefBins &rb, const double *p, const double *q) {
#pragma unroll
  for (int d = 2; d >= 0; d--) {
    int a = ref_bin1(rb, d, p[d]), c = ref_bin1(rb, d, q[d]);
    if (c != a) return c > a ? 1 : -1;
  }
  return 0;
}

__device__ __forceinline__ bool above_right(const double *q, const double *p) {
  if (q[2] < p[2]) return false;
  if (q[2] == p[2]) {
    if (q[1] < p[1]) return false;
    if (q[1] == p[1] && q[0] < p[0]) return false;
  }
  return true;
}

__device__ __forceinline__ double rsq_rn(double dx, double dy, double dz) {
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// Stores one entry; the image byte carries IN_CUT when the pair lies inside
// the force cutoff at build time (the compaction puts those entries first).
constexpr unsigned char IN_CUT = 0x80;
__device__ __forceinline__ void emit(const BuildArgs &A, int i, int &n, int *raw, unsigned char *img,
                                     int val, int code) {
  if (n < A.cap) {
    raw[(size_t)n * A.nsi + i] = val;
    img[(size_t)n * A.nsi + i] = (unsigned char)code;
  }
  n++;
}

// One query point (an i-site) of the build.
struct Query {
  Rep r;          // its replica
  int i;          // site-table index (atoms: input order)
  int slot;       // list slot: atoms in cell-sorted order, then Gauss points
  bool iatom;
  int ie, ig, iu;
  double xi[3];   // raw position
  double wi[3];   // wrapped into the box: wi = xi + ti L
  int ti[3];
};

template <class RP>
__device__ __forceinline__ void make_query(const BuildArgs &A, const RP &P, int i, Query &q) {
  q.r = P.site(i);
  q.i = i;
  q.slot = i;
  q.iatom = i < A.na;
  q.ie = q.ig = q.iu = -1;
  if (q.iatom) {
    double4 p = A.xs[i];
    q.xi[0] = p.x;
    q.xi[1] = p.y;
    q.xi[2] = p.z;
  } else {
    q.ie = (i - A.na) / NG;
    q.ig = (i - A.na) % NG;
    q.iu = gauss_site(q.ig);
    const double *nx = A.nodex + (size_t)q.ie * 24 + 3 * gauss_node(q.ig);
    q.xi[0] = nx[0];
    q.xi[1] = nx[1];
    q.xi[2] = nx[2];
  }
  const BoxD &b = q.r.b;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    double f = floor((q.xi[d] - b.lo[d]) / b.L[d]);
    q.ti[d] = -(int)f;
    q.wi[d] = q.xi[d] - f * b.L[d];
    if (q.wi[d] >= b.hi[d]) {
      q.wi[d] -= b.L[d];
      q.ti[d] -= 1;
    }
    if (q.wi[d] < b.lo[d]) {
      q.wi[d] += b.L[d];
      q.ti[d] += 1;
    }
  }
}

// A candidate atom j seen in a cell with wrap count W: exact test and storage
// rules (atoms are inside the box after pbc, so their own wrap is zero).
// Full-list entries go to `full(j, code)`; half-list entries are stored here.
template <class FullSink>
__device__ __forceinline__ void try_atom(const BuildArgs &A, const Query &q, int j, const int W[3], int &nh,
                                         FullSink &&full) {
  int s[3] = {W[0] - q.ti[0], W[1] - q.ti[1], W[2] - q.ti[2]};
  bool zero = (s[0] == 0 && s[1] == 0 && s[2] == 0);
  if (q.iatom && j == q.i && zero) return;
  double4 xj = A.xs[j];
  double qq[3] = {xj.x, xj.y, xj.z};
  if (!zero) {
    qq[0] = s[0] ? __dadd_rn(qq[0], s[0] * q.r.b.L[0]) : qq[0];
    qq[1] = s[1] ? __dadd_rn(qq[1], s[1] * q.r.b.L[1]) : qq[1];
    qq[2] = s[2] ? __dadd_rn(qq[2], s[2] * q.r.b.L[2]) : qq[2];
  }
  double rsq = rsq_rn(__dsub_rn(q.xi[0], qq[0]), __dsub_rn(q.xi[1], qq[1]), __dsub_rn(q.xi[2], qq[2]));
  if (!(rsq <= A.cutneighsq)) return;
  // a neighbour beyond the first periodic image cannot be stored (the box is
  // shorter than twice the cutoff)
  if (s[0] < -1 || s[0] > 1 || s[1] < -1 || s[1] > 1 || s[2] < -1 || s[2] > 1) {
    atomicExch(&A.overflow[2], 1);
    return;
  }
  int code = img_code(s[0], s[1], s[2]) | (rsq < A.cutforcesq ? IN_CUT : 0);
  full(j, code);
  if (A.want_half && q.iatom) {
    int ord = ref_bin_order(A.rb, q.xi, qq);
    bool keep = ord > 0 || (ord == 0 && (zero ? (j > q.i) : above_right(qq, q.xi)));
    if (keep) emit(A, q.slot, nh, A.raw_half, A.img_half, j, code);
  }
}

__device__ __forceinline__ void wrap_cell(int v, int nc, int &cell, int &W) {
  W = 0;
  while (v < 0) {
    v += nc;
    W--;
  }
  while (v >= nc) {
    v -= nc;
    W++;
  }
  cell = v;
}

// Element lattice sites are found in two phases.  Phase A (one thread per
// query) walks the element cells around the query and, for every element
// whose site box in lattice-index space is not empty, writes a work item:
// the element, the periodic image and the box.  Phase B (one warp per query)
// tests the sites of each item with the lanes splitting the box, emitting in
// box order, so the list is the one a serial walk would write.

// work item: x = element | (image + 4 per dimension, 3 bits each) << 21,
// y = box lo/hi in lattice indices (4 bits each)
__device__ __forceinline__ int2 pack_item(int e, const int s[3], const int lo[3], const int hi[3]) {
  int x = e | ((s[0] + 4) << 21) | ((s[1] + 4) << 24) | ((s[2] + 4) << 27);
  int y = lo[0] | (lo[1] << 4) | (lo[2] << 8) | (hi[0] << 12) | (hi[1] << 16) | (hi[2] << 20);
  return make_int2(x, y);
}
__device__ __forceinline__ void unpack_item(int2 it, int &e, int s[3], int lo[3], int hi[3]) {
  e = it.x & ((1 << 21) - 1);
  s[0] = ((it.x >> 21) & 7) - 4;
  s[1] = ((it.x >> 24) & 7) - 4;
  s[2] = ((it.x >> 27) & 7) - 4;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    lo[d] = (it.y >> (4 * d)) & 15;
    hi[d] = (it.y >> (12 + 4 * d)) & 15;
  }
}

// Phase A for one query: the element walk (candidate sphere test, then the
// lattice-index box of the sites whose affine position can lie within
// cutneigh + the element's deviation from affine).  Returns the number of
// items; at most cap are stored.
__device__ int element_items(const BuildArgs &A, const Query &q, int2 *out, int cap) {
  const Grid &eg = q.r.eg;
  int ci[3];
#pragma unroll
  for (int d = 0; d < 3; d++)
    ci[d] = min(max((int)((q.wi[d] - q.r.b.lo[d]) * eg.inv[d]), 0), eg.nc[d] - 1);
  // no element in the 27 cells around: nothing to walk
  if (A.ecell_near && !A.ecell_near[q.r.ebase + (ci[2] * eg.nc[1] + ci[1]) * eg.nc[0] + ci[0]]) return 0;
  int n = 0;
  for (int oz = -1; oz <= 1; oz++) {
    int cz, Wz;
    wrap_cell(ci[2] + oz, eg.nc[2], cz, Wz);
    for (int oy = -1; oy <= 1; oy++) {
      int cy, Wy;
      wrap_cell(ci[1] + oy, eg.nc[1], cy, Wy);
      for (int ox = -1; ox <= 1; ox++) {
        int cx, Wx;
        wrap_cell(ci[0] + ox, eg.nc[0], cx, Wx);
        int cell = q.r.ebase + (cz * eg.nc[1] + cy) * eg.nc[0] + cx;
        int beg = A.ecell_start[cell], end = A.ecell_start[cell + 1];
        if (beg == end) continue;
        int s[3] = {Wx - q.ti[0], Wy - q.ti[1], Wz - q.ti[2]};
        double sL[3] = {s[0] * q.r.b.L[0], s[1] * q.r.b.L[1], s[2] * q.r.b.L[2]};
        for (int kk = beg; kk < end; kk++) {
          int e = A.ecell_elems[kk];
          double4 ce = A.ecenter[e];
          // sphere test in the element's raw frame: |xi - s L - centre| <= cutneigh + R
          double p[3] = {q.xi[0] - sL[0], q.xi[1] - sL[1], q.xi[2] - sL[2]};
          const double *fr = A.eframe + (size_t)e * EFR;
          double dmax = fr[12];
          double R = ce.w + dmax + A.cutneigh + 1e-6;
          double dcx = p[0] - ce.x, dcy = p[1] - ce.y, dcz = p[2] - ce.z;
          if (dcx * dcx + dcy * dcy + dcz * dcz > R * R) continue;
          double rel[3] = {p[0] - fr[0], p[1] - fr[1], p[2] - fr[2]};
          int lo[3], hi[3];
          bool empty = false;
#pragma unroll
          for (int r = 0; r < 3; r++) {
            double a0 = fr[3 + 3 * r], a1 = fr[4 + 3 * r], a2 = fr[5 + 3 * r];
            double fidx = a0 * rel[0] + a1 * rel[1] + a2 * rel[2];
            double rho = (A.cutneigh + dmax + 1e-6) * fr[22 + r] + 1e-6;
            lo[r] = max(0, (int)ceil(fidx - rho));
            hi[r] = min(NC - 1, (int)floor(fidx + rho));
            if (lo[r] > hi[r]) empty = true;
          }
          if (empty) continue;
          // a box shorter than the candidate sphere's diameter shows an element
          // under two images; images beyond +-2 cannot be encoded (and are far
          // beyond any cutoff in such a box)
          if (s[0] < -3 || s[0] > 3 || s[1] < -3 || s[1] > 3 || s[2] < -3 || s[2] > 3) {
            atomicExch(&A.overflow[2], 1);
            continue;
          }
          if (n < cap) out[n] = pack_item(e, s, lo, hi);
          n++;
        }
      }
    }
  }
  return n;
}

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Warp-wide emission: the lanes' accepted candidates are stored in lane
// order after the entries already written, so a warp walking candidates in
// chunks of 32 writes exactly the order of a serial walk.  Every lane keeps
// the same count n.
__device__ __forceinline__ void warp_emit(const BuildArgs &A, int slot, int &n, int *raw, unsigned char *img,
                                          bool pass, int val, int code) {
  const unsigned m = __ballot_sync(0xffffffffu, pass);
  if (pass) {
    const int at = n + __popc(m & lanemask_lt());
    if (at < A.cap) {
      raw[(size_t)at * A.nsi + slot] = val;
      img[(size_t)at * A.nsi + slot] = (unsigned char)code;
    }
  }
  n += __popc(m);
}

// The same for full lists: accepted entries go to the front segment (inside
// the inner radius) or the back segment, each in lane order; dst gets the
// entry and img (when given) the image code at the same place.  Rows
// outside [0, cap) are not written (the count still grows and flags the
// overflow).
__device__ __forceinline__ void warp_emit_full(const BuildArgs &A, int slot, int &nin, int &nout, int *dst,
                                               unsigned char *img, bool pass, bool incut, int val, int code) {
  const unsigned mi = __ballot_sync(0xffffffffu, pass && incut);
  const unsigned mo = __ballot_sync(0xffffffffu, pass && !incut);
  if (pass) {
    const int row = incut ? nin + __popc(mi & lanemask_lt()) : A.cap - 1 - (nout + __popc(mo & lanemask_lt()));
    if (row >= 0 && row < A.cap) {
      dst[(size_t)row * A.nsi + slot] = val;
      if (img) img[(size_t)row * A.nsi + slot] = (unsigned char)code;
    }
  }
  nin += __popc(mi);
  nout += __popc(mo);
}

// Phase B for one query: its items in groups of up to 16.  Lane k stages
// item k of a group in the warp's shared scratch (the 24 ghost node
// coordinates and the FP32 affine frame relative to the query), then the
// lanes walk the group's sites flattened in (item, a, bb, cc) order -- the
// serial order -- so small boxes do not leave lanes idle.  Each site takes the
// FP32 affine screen; the sites that pass are queued in that order and take
// the reference's exact FP64 distance 32 at a time, so the FP64 work runs on
// full warps and the entries are emitted in the serial order.
constexpr int ITEM_GROUP = 16;   // items staged at a time (a query has a few)
struct ItemStage {
  double g[ITEM_GROUP][24];   // ghost node coordinates nodex + s L
  float fr[ITEM_GROUP][13];   // frame columns a, b, c; query minus frame origin; screen radius^2
  int mg[ITEM_GROUP][2];      // ceil(2^16 / n) of the box's z and y extents (division by multiply-shift)
  int2 item[ITEM_GROUP];      // the group's items
  int queue[64];              // screened sites: item lane << 10 | lattice site
};

// The exact test of one queued site (active lanes only) and the warp's
// emission of the accepted ones.
__device__ __forceinline__ void items_exact(const BuildArgs &A, const Query &q, const ItemStage &st, bool active,
                                            int entry, int &nin, int &nout, int &nh) {
  bool pf = false, ph = false;
  int val = 0, codef = 0, code = 0;
  if (active) {
    const int m = entry >> 10, u = entry & 1023;
    int e, sv[3], lo[3], hi[3];
    unpack_item(st.item[m], e, sv, lo, hi);
    const bool zero = (sv[0] == 0 && sv[1] == 0 && sv[2] == 0);
    const bool far_image = sv[0] < -1 || sv[0] > 1 || sv[1] < -1 || sv[1] > 1 || sv[2] < -1 || sv[2] > 1;
    code = far_image ? 0 : img_code(sv[0], sv[1], sv[2]);
    const double *g = st.g[m];
    double dx = q.xi[0], dy = q.xi[1], dz = q.xi[2];
#pragma unroll
    for (int k = 0; k < 8; k++) {
      double N = shape_val(u, k);
      dx = __dsub_rn(dx, __dmul_rn(N, g[3 * k]));
      dy = __dsub_rn(dy, __dmul_rn(N, g[3 * k + 1]));
      dz = __dsub_rn(dz, __dmul_rn(N, g[3 * k + 2]));
    }
    double rsq = rsq_rn(dx, dy, dz);
    if (rsq <= A.cutneighsq) {
      if (far_image) {
        atomicExch(&A.overflow[2], 1);
      } else {
        pf = true;
        val = KIND_SITE | (e * NU + u);
        codef = code | (rsq < A.cutforcesq ? IN_CUT : 0);
        if (site_gauss(u) < 0) A.site_flag[e * NU + u] = 1;   // to be interpolated
        ph = true;
        if (A.want_half && !q.iatom) {
          int jg = site_gauss(u);
          if (jg >= 0) {
            if (zero) {
              ph = (q.ie < e) || (q.ie == e && q.ig < jg);
            } else {
              const double4 ce = A.ecenter[e], ci = A.ecenter[q.ie];
              const double sL[3] = {sv[0] * q.r.b.L[0], sv[1] * q.r.b.L[1], sv[2] * q.r.b.L[2]};
              double qcen[3] = {sv[0] ? __dadd_rn(ce.x, sL[0]) : ce.x, sv[1] ? __dadd_rn(ce.y, sL[1]) : ce.y,
                                sv[2] ? __dadd_rn(ce.z, sL[2]) : ce.z};
              double icen[3] = {ci.x, ci.y, ci.z};
              ph = above_right(qcen, icen);
            }
          }
        }
      }
    }
  }
  warp_emit_full(A, q.slot, nin, nout, A.raw_full, A.img_full, pf, (codef & IN_CUT) != 0, val, code);
  if (A.want_half) warp_emit(A, q.slot, nh, A.raw_half, A.img_half, ph, val, code);
}

__device__ void items_warp(const BuildArgs &A, const Query &q, const int2 *items, int n, ItemStage &st, int &nin,
                           int &nout, int &nh) {
  const int lane = threadIdx.x & 31;
  for (int g0 = 0; g0 < n; g0 += ITEM_GROUP) {
    const int gi = g0 + lane;
    int2 it = make_int2(0, 0);
    int nbox = 0;
    __syncwarp();
    if (lane < ITEM_GROUP && gi < n) {
      it = items[gi];
      st.item[lane] = it;
      int e, sv[3], lo[3], hi[3];
      unpack_item(it, e, sv, lo, hi);
      nbox = (hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
      const double sL[3] = {sv[0] * q.r.b.L[0], sv[1] * q.r.b.L[1], sv[2] * q.r.b.L[2]};
      const double *nx = A.nodex + (size_t)e * 24;
#pragma unroll
      for (int k = 0; k < 24; k++) st.g[lane][k] = sv[k % 3] ? __dadd_rn(nx[k], sL[k % 3]) : nx[k];
      const double *fr = A.eframe + (size_t)e * EFR;
#pragma unroll
      for (int k = 0; k < 9; k++) st.fr[lane][k] = (float)fr[13 + k];
#pragma unroll
      for (int d = 0; d < 3; d++) st.fr[lane][9 + d] = (float)(q.xi[d] - sL[d] - fr[d]);
      const float lim = (float)(A.cutneigh + fr[12]) + 1e-3f;
      st.fr[lane][12] = lim * lim;
      const int n1s = hi[1] - lo[1] + 1, n2s = hi[2] - lo[2] + 1;
      st.mg[lane][0] = (65536 + n2s - 1) / n2s;
      st.mg[lane][1] = (65536 + n1s - 1) / n1s;
    }
    __syncwarp();
    // exclusive prefix of the box sizes over the group's lanes
    int incl = nbox;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    const int excl = incl - nbox;
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    const int ng = min(ITEM_GROUP, n - g0);
    int qn = 0;   // queued sites (warp-uniform)
    for (int base = 0; base < total; base += 32) {
      const int f = base + lane;
      // item of flattened site f: the last lane m < ng with excl[m] <= f
      int m = 0;
#pragma unroll
      for (int step = ITEM_GROUP / 2; step > 0; step >>= 1) {
        const int cand = m + step;
        const int v = __shfl_sync(0xffffffffu, excl, cand & 31);
        if (cand < ng && v <= f) m = cand;
      }
      const int exm = __shfl_sync(0xffffffffu, excl, m);
      bool pass = false;
      int u = 0;
      if (f < total) {
        const int y = st.item[m].y;
        const int lo0 = y & 15, lo1 = (y >> 4) & 15, lo2 = (y >> 8) & 15;
        const int n1 = ((y >> 16) & 15) - lo1 + 1, n2 = ((y >> 20) & 15) - lo2 + 1;
        // (a, bb, cc) of the t-th site of the box in (a, bb, cc) order; the
        // multiply-shift quotients are exact for t < 729 and extents <= 9
        const int t = f - exm;
        const int q2 = (t * st.mg[m][0]) >> 16, q12 = (q2 * st.mg[m][1]) >> 16;
        const int cc = lo2 + (t - q2 * n2), bb = lo1 + (q2 - q12 * n1), a = lo0 + q12;
        const float *F = st.fr[m];
        const float ex = F[9] - (a * F[0] + bb * F[3] + cc * F[6]);
        const float ey = F[10] - (a * F[1] + bb * F[4] + cc * F[7]);
        const float ez = F[11] - (a * F[2] + bb * F[5] + cc * F[8]);
        u = (a * NC + bb) * NC + cc;
        pass = ex * ex + ey * ey + ez * ez <= F[12];
        if (pass && !q.iatom && u == q.iu) {
          // the query's own site (same element, zero image)
          const int x = st.item[m].x;
          pass = !((x & ((1 << 21) - 1)) == q.ie && (x >> 21) == ((4 << 6) | (4 << 3) | 4));
        }
      }
      const unsigned mask = __ballot_sync(0xffffffffu, pass);
      if (pass) st.queue[qn + __popc(mask & lanemask_lt())] = (m << 10) | u;
      qn += __popc(mask);
      __syncwarp();
      if (qn >= 32) {
        items_exact(A, q, st, true, st.queue[lane], nin, nout, nh);
        qn -= 32;
        const int rest = lane < qn ? st.queue[32 + lane] : 0;
        __syncwarp();
        if (lane < qn) st.queue[lane] = rest;
        __syncwarp();
      }
    }
    if (qn > 0) items_exact(A, q, st, lane < qn, lane < qn ? st.queue[lane] : 0, nin, nout, nh);
  }
}

// An atom candidate j of a Gauss point seen in a cell with wrap count W:
// the exact distance test; code gets the image and the in-cutoff mark
// (Gauss points keep no atoms in half lists).
__device__ __forceinline__ bool gauss_atom_test(const BuildArgs &A, const Query &q, int j, const int W[3],
                                                int &code) {
  int s[3] = {W[0] - q.ti[0], W[1] - q.ti[1], W[2] - q.ti[2]};
  double4 xj = A.xs[j];
  double qq[3] = {xj.x, xj.y, xj.z};
  qq[0] = s[0] ? __dadd_rn(qq[0], s[0] * q.r.b.L[0]) : qq[0];
  qq[1] = s[1] ? __dadd_rn(qq[1], s[1] * q.r.b.L[1]) : qq[1];
  qq[2] = s[2] ? __dadd_rn(qq[2], s[2] * q.r.b.L[2]) : qq[2];
  double rsq = rsq_rn(__dsub_rn(q.xi[0], qq[0]), __dsub_rn(q.xi[1], qq[1]), __dsub_rn(q.xi[2], qq[2]));
  if (!(rsq <= A.cutneighsq)) return false;
  if (s[0] < -1 || s[0] > 1 || s[1] < -1 || s[1] > 1 || s[2] < -1 || s[2] > 1) {
    atomicExch(&A.overflow[2], 1);
    return false;
  }
  code = img_code(s[0], s[1], s[2]) | (rsq < A.cutforcesq ? IN_CUT : 0);
  return true;
}

__device__ __forceinline__ void finish_counts(const BuildArgs &A, int i, int nin, int nout, int nh) {
  A.num_full[i] = nin + nout;
  A.num_in[i] = nin;
  if (A.want_half) A.num_half[i] = nh;
  int m = max(nin + nout, nh);
  if (m > A.cap) {
    atomicExch(&A.overflow[0], 1);
    atomicMax(&A.overflow[1], m);
  }
}

// Atoms, atom neighbours: one block (one warp) per chunk of 32 consecutive
// sorted atoms (list slots).  Cells (>= cutneigh) are sorted x fastest, so a
// chunk lies in one row of cells, or in two at a row's end (then the warp
// takes the two parts in turn).  For each of the 9 rows around the part's
// row the lanes walk together the cells from one left of the part's first
// cell to one right of its last, as at most three runs of consecutive cells
// under one image (the left and right wraps and the middle), so every
// candidate is one broadcast load shared by the warp and all 32 lanes hold
// an atom.  A lane meets the cells of its own 27-cell block in the order a
// walk of that block alone would take (ascending x in each row) and the
// others only beyond its reach, so its list is the same entry for entry.
// A conservative FP32 distance test (from a float copy of the wrapped
// positions) decides all but the candidates near the cutoff, which take the
// exact FP64 test.  The image of a run relative to each lane's atom is fixed
// per run.
//
// Full-list entries are written in their final form (the candidate's sorted
// position is its list slot) and staged per lane in two 32-row rings in
// shared memory, one per segment (lane = column, so a lane only ever touches
// its own bank); the warp writes them out row by row: the lanes' list slots
// are consecutive, so each row is one coalesced store across the warp
// instead of one scattered store per entry (the lists are transposed,
// [entry][slot]).  The warp flushes whenever a lane's ring is full and once
// at the end.
constexpr int STAGE_ROWS = 32;
template <class RP>
__device__ __forceinline__ void build_atoms_chunk(BuildArgs A, RP P, const int chunk) {
  const int lane = threadIdx.x & 31;
  const float fcut2 = (float)A.cutforcesq;
  __shared__ int st_in[STAGE_ROWS][32], st_out[STAGE_ROWS][32];   // front / back segment rings
  const int h = chunk * 32 + lane;
  const bool mine = h < A.na;
  const int key = mine ? A.acell_of[h] : -1;
  Query q;
  float wx = 0.f, wy = 0.f, wz = 0.f;
  if (mine) {
    make_query(A, P, (int)__double_as_longlong(A.acell_pos[h].w), q);
    q.slot = h;
    float4 w = A.acell_pos32[h];
    wx = w.x;
    wy = w.y;
    wz = w.z;
  }
  // the chunk's parts, one row of cells each, lowest lanes first
  unsigned todo = __ballot_sync(0xffffffffu, mine);
  while (todo) {
    const int lkey = __shfl_sync(0xffffffffu, key, __ffs(todo) - 1);
    const Rep R = P.acell(lkey);
    const int nc0 = R.ag.nc[0], nc1 = R.ag.nc[1], nc2 = R.ag.nc[2];
    const int row = (lkey - R.abase) / nc0;   // cz * nc1 + cy of the part
    const int hx = key - R.abase - row * nc0;
    const bool active = mine && ((todo >> lane) & 1u) && hx >= 0 && hx < nc0;
    todo &= ~__ballot_sync(0xffffffffu, active);
    const int hy = row % nc1, hz = row / nc1;
    // unwrapped x range of the candidate cells
    const int xlo = __reduce_min_sync(0xffffffffu, active ? hx : 0x7fffffff) - 1;
    const int xhi = __reduce_max_sync(0xffffffffu, active ? hx : -1) + 1;
    // FP32 screen: beyond cutneigh + margin never a neighbour, within
    // cutneigh - margin always one; only the band between takes the FP64 test
    const float pre = (float)A.cutneigh + R.fmargin, sure = (float)A.cutneigh - R.fmargin;
    const float pre2 = pre * pre, sure2 = sure * sure;
    int nin = 0, nout = 0, nh = 0;
    int fin = 0, fout = 0;   // this lane's entries of each segment already written
    // entry = (neighbour's list slot << IMG_BITS) | image code
    auto stage = [&](int val, bool incut) {
      if (incut) st_in[nin++ & (STAGE_ROWS - 1)][lane] = val;
      else st_out[nout++ & (STAGE_ROWS - 1)][lane] = val;
    };
    // every lane writes its staged entries, row by row: front segment
    // entries [fin, nin) to rows fin.., back segment entries [fout, nout)
    // to rows cap-1-fout down
    auto flush = [&]() {
      int lo = __reduce_min_sync(0xffffffffu, active ? fin : 0x7fffffff);
      int hi = __reduce_max_sync(0xffffffffu, active ? nin : 0);
      for (int k = lo; k < hi; k++)
        if (active && k >= fin && k < nin && k < A.cap)
          A.nbr_full[(size_t)k * A.nsi + q.slot] = st_in[k & (STAGE_ROWS - 1)][lane];
      lo = __reduce_min_sync(0xffffffffu, active ? fout : 0x7fffffff);
      hi = __reduce_max_sync(0xffffffffu, active ? nout : 0);
      for (int k = lo; k < hi; k++)
        if (active && k >= fout && k < nout && k < A.cap)
          A.nbr_full[(size_t)(A.cap - 1 - k) * A.nsi + q.slot] = st_out[k & (STAGE_ROWS - 1)][lane];
      fin = nin;
      fout = nout;
    };
    for (int oz = -1; oz <= 1; oz++) {
      int cz, Wz;
      wrap_cell(hz + oz, nc2, cz, Wz);
      for (int oy = -1; oy <= 1; oy++) {
        int cy, Wy;
        wrap_cell(hy + oy, nc1, cy, Wy);
        const int rowbase = R.abase + (cz * nc1 + cy) * nc0;
        // runs: unwrapped x in [xlo, -1] (the cell nc0 - 1 one image left),
        // [0, nc0 - 1], [nc0, xhi] (the cell 0 one image right)
        for (int run = -1; run <= 1; run++) {
          const int u0 = run < 0 ? xlo : (run == 0 ? max(xlo, 0) : max(xlo, nc0));
          const int u1 = run < 0 ? min(xhi, -1) : (run == 0 ? min(xhi, nc0 - 1) : xhi);
          if (u0 > u1) continue;
          const int Wx = run;
          int W[3] = {Wx, Wy, Wz};
          // the lane's position less the run's image shift (once per run)
          const float rx = __fsub_rn(wx, (float)(Wx * R.b.L[0]));
          const float ry = __fsub_rn(wy, (float)(Wy * R.b.L[1]));
          const float rz = __fsub_rn(wz, (float)(Wz * R.b.L[2]));
          // this run's image relative to the lane's atom
          const int s0 = Wx - q.ti[0], s1 = Wy - q.ti[1], s2 = Wz - q.ti[2];
          const bool zero = (s0 == 0 && s1 == 0 && s2 == 0);
          const bool far = s0 < -1 || s0 > 1 || s1 < -1 || s1 > 1 || s2 < -1 || s2 > 1;
          const int code = far ? 0 : img_code(s0, s1, s2);
          const int beg = A.acell_start[rowbase + u0 - Wx * nc0], end = A.acell_start[rowbase + u1 - Wx * nc0 + 1];
          // candidate pj at list slot ks
          // the FP32 distance in explicitly rounded operations: the
          // in-cutoff mark below decides an entry's list segment, so every
          // kernel that builds these lists (grid and SM-local forms) must
          // round it the same way, whatever the compiler would contract
          auto consider = [&](const float4 &pj, int ks) {
            const float ex = __fsub_rn(rx, pj.x);
            const float ey = __fsub_rn(ry, pj.y);
            const float ez = __fsub_rn(rz, pj.z);
            const float r2 = __fmaf_rn(ez, ez, __fmaf_rn(ey, ey, __fmul_rn(ex, ex)));
            if (r2 > pre2) return;
            const int j = __float_as_int(pj.w);
            if (r2 < sure2 && !A.want_half) {
              if (zero && j == q.i) return;
              if (far) {
                atomicExch(&A.overflow[2], 1);
                return;
              }
              stage((ks << IMG_BITS) | code, r2 < fcut2);
            } else {
              try_atom(A, q, j, W, nh, [&](int, int c) {
                stage((ks << IMG_BITS) | (c & (IN_CUT - 1)), (c & IN_CUT) != 0);
              });
            }
          };
          // candidates four at a time: the four broadcast loads are in
          // flight together instead of one load's latency per candidate
          int k = beg;
          for (; k + 4 <= end; k += 4) {
            const float4 p0 = A.acell_pos32[k], p1 = A.acell_pos32[k + 1];
            const float4 p2 = A.acell_pos32[k + 2], p3 = A.acell_pos32[k + 3];
            // room for four more entries in every lane's rings
            if (__any_sync(0xffffffffu, active && (nin - fin > STAGE_ROWS - 4 || nout - fout > STAGE_ROWS - 4)))
              flush();
            if (active) {
              consider(p0, k);
              consider(p1, k + 1);
              consider(p2, k + 2);
              consider(p3, k + 3);
            }
          }
          for (; k < end; k++) {
            const float4 pj = A.acell_pos32[k];
            if (__any_sync(0xffffffffu, active && (nin - fin >= STAGE_ROWS || nout - fout >= STAGE_ROWS)))
              flush();
            if (active) consider(pj, k);
          }
        }
      }
    }
    flush();
    if (active) {
      A.site_from[q.slot] = make_int2(nin, nout);
      finish_counts(A, q.slot, nin, nout, nh);
    }
  }
}

// The single-system forms as the compiler allocates them (96 registers with
// the candidate loads four at a time, 118 in the persistent form: a cap at 20
// resident warps per SM, 88 registers, was 10 % slower); the batch form
// capped at 64 registers (a few bytes spilled) so that 32 warps are resident
// per SM: 10 % faster on a 64-replica batch, where the same cap slowed the
// single-system form.
__global__ void __launch_bounds__(32) k_build_atoms(BuildArgs A, OneRep P) { build_atoms_chunk(A, P, blockIdx.x); }
__global__ void __launch_bounds__(32, 32) k_build_atoms(BuildArgs A, ManyRep P) {
  build_atoms_chunk(A, P, blockIdx.x);
}

// Single systems: persistent warps taking the chunks in SM-local runs (one
// chunk per run, sm_run in device.cuh), so that the warps resident on one SM
// walk neighbouring cells and share their candidates in L1.  The same lists.
__global__ void __launch_bounds__(32) k_build_atoms_sm(BuildArgs A, OneRep P, int nchunk, int *cnt, int nsm) {
  __shared__ int v;
  if (threadIdx.x == 0) v = sm_id() % nsm;
  for (;;) {
    const int chunk = sm_run(cnt, nsm, nchunk, v);
    if (chunk < 0) return;
    build_atoms_chunk(A, P, chunk);
  }
}

// Phase A over every list slot: the element walk of each atom and Gauss
// point; atoms with at least one item go on the work list of phase B (its
// order does not matter: an atom's entries depend on that atom alone).
template <class RP>
__device__ __forceinline__ void elem_items_slot(BuildArgs A, RP P, int2 *items, int *nitems, int icap, int *work,
                                                int *nwork) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= A.nsi) return;
  Query q;
  if (t < A.na) {
    make_query(A, P, A.atom_of_slot[t], q);
    q.slot = t;
  } else {
    make_query(A, P, t, q);
  }
  const int n = element_items(A, q, items + (size_t)t * icap, icap);
  nitems[t] = n;
  if (n > icap) {
    atomicExch(&A.overflow[8], 1);
    atomicMax(&A.overflow[9], n);
  }
  if (t < A.na && n > 0) work[atomicAdd(nwork, 1)] = t;
}

// The single-system form as the compiler allocates it; the batch form capped
// at 64 registers (from 70) for 8 resident blocks per SM: 4 % faster on a
// 64-replica batch, where the same cap slowed the single-system form.
__global__ void __launch_bounds__(128) k_elem_items(BuildArgs A, OneRep P, int2 *items, int *nitems, int icap,
                                                    int *work, int *nwork) {
  elem_items_slot(A, P, items, nitems, icap, work, nwork);
}
__global__ void __launch_bounds__(128, 8) k_elem_items(BuildArgs A, ManyRep P, int2 *items, int *nitems, int icap,
                                                       int *work, int *nwork) {
  elem_items_slot(A, P, items, nitems, icap, work, nwork);
}

// Phase B for atoms: one warp per listed atom, its element sites appended
// after its atom neighbours.
template <class RP>
__global__ void __launch_bounds__(128, 8) k_build_atom_sites(BuildArgs A, RP P, const int2 *items, const int *nitems,
                                                          int icap, const int *work, const int *nwork) {
  __shared__ ItemStage stage[4];
  ItemStage &st = stage[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int nw = *nwork;
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nw; w += (gridDim.x * blockDim.x) >> 5) {
    const int h = work[w];
    Query q;
    make_query(A, P, A.atom_of_slot[h], q);
    q.slot = h;
    int nin = A.num_in[h], nout = A.num_full[h] - nin, nh = A.want_half ? A.num_half[h] : 0;
    items_warp(A, q, items + (size_t)h * icap, min(nitems[h], icap), st, nin, nout, nh);
    if (lane == 0) finish_counts(A, h, nin, nout, nh);
    __syncwarp();
  }
}

// Phase B for Gauss points: one warp each; atoms from the 27 surrounding atom
// cells (full list only), 32 candidates at a time, then the element sites.
template <class RP>
__global__ void __launch_bounds__(128, 8) k_build_gauss(BuildArgs A, RP P, const int2 *items, const int *nitems,
                                                     int icap) {
  __shared__ ItemStage stage[4];
  ItemStage &st = stage[threadIdx.x >> 5];
  const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= NG * A.ne) return;   // whole warps
  Query q;
  make_query(A, P, A.na + t, q);
  const Grid &ag = q.r.ag;
  int nin = 0, nout = 0, nh = 0;
  if (A.na > 0) {
    const double pre = (A.cutneigh + 1e-6) * (A.cutneigh + 1e-6);
    int ci[3];
#pragma unroll
    for (int d = 0; d < 3; d++)
      ci[d] = min(max((int)((q.wi[d] - q.r.b.lo[d]) * ag.inv[d]), 0), ag.nc[d] - 1);
    // no atom in the 27 cells around (most Gauss points of an element
    // region): no atom candidates, the walk below would find none
    const bool atoms_near = !A.acell_near || A.acell_near[q.r.abase + (ci[2] * ag.nc[1] + ci[1]) * ag.nc[0] + ci[0]];
    if (atoms_near)
    for (int oz = -1; oz <= 1; oz++) {
      int cz, Wz;
      wrap_cell(ci[2] + oz, ag.nc[2], cz, Wz);
      for (int oy = -1; oy <= 1; oy++) {
        int cy, Wy;
        wrap_cell(ci[1] + oy, ag.nc[1], cy, Wy);
        for (int ox = -1; ox <= 1; ox++) {
          int cx, Wx;
          wrap_cell(ci[0] + ox, ag.nc[0], cx, Wx);
          int cell = q.r.abase + (cz * ag.nc[1] + cy) * ag.nc[0] + cx;
          int W[3] = {Wx, Wy, Wz};
          double sh[3] = {Wx * q.r.b.L[0], Wy * q.r.b.L[1], Wz * q.r.b.L[2]};
          int beg = A.acell_start[cell], end = A.acell_start[cell + 1];
          for (int base = beg; base < end; base += 32) {
            const int k = base + lane;
            bool pass = false;
            int j = 0, code = 0;
            if (k < end) {
              double4 pj = A.acell_pos[k];
              double ex = q.wi[0] - (pj.x + sh[0]), ey = q.wi[1] - (pj.y + sh[1]), ez = q.wi[2] - (pj.z + sh[2]);
              if (ex * ex + ey * ey + ez * ez <= pre) {
                j = (int)__double_as_longlong(pj.w);
                pass = gauss_atom_test(A, q, j, W, code);
              }
            }
            // the atom's list slot is its sorted position k
            warp_emit_full(A, q.slot, nin, nout, A.nbr_full, nullptr, pass, (code & IN_CUT) != 0,
                           (k << IMG_BITS) | (code & (IN_CUT - 1)), 0);
          }
        }
      }
    }
  }
  const int slot = A.na + t;
  if (lane == 0) A.site_from[slot] = make_int2(nin, nout);
  items_warp(A, q, items + (size_t)slot * icap, min(nitems[slot], icap), st, nin, nout, nh);
  if (lane == 0) finish_counts(A, q.slot, nin, nout, nh);
}

// ------------------------------------------------------------- compaction

__global__ void k_act_table(const int *flag, const int *pref, int ngid, int ne, int nsi, int *act_gid,
                            int *act_off, int *nact, int *too_many) {
  int gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid < ngid && flag[gid]) act_gid[pref[gid]] = gid;
  if (gid < ne) act_off[gid] = pref[gid * NU];
  if (gid == 0) {
    act_off[ne] = pref[ngid];
    *nact = pref[ngid];
    if ((long)nsi + pref[ngid] >= (1L << (31 - IMG_BITS))) *too_many = 1;
  }
}

// Packs each entry as (pair-table index << 5 | image code): atoms by their
// list slot (the pair table holds atoms in cell-sorted order), element sites
// after them as in the site table.  Entries inside the inner radius (the
// force cutoff plus a margin) at build time go first, each group in build
// order, and their number is kept (num_in): while no site has moved half the
// margin since the build, every pair inside the cutoff lies in that prefix,
// in the same order, so the pair loops may stop there with identical sums.
__global__ void k_remap(const int *raw, const unsigned char *img, const int *num, int nsi, int cap,
                        const int *pref, const int *atom_slot, int na, int ne, int *out, int *num_in) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nsi) return;
  int n = min(num[i], cap);
  int nin = 0;
  for (int k = 0; k < n; k++) nin += (img[(size_t)k * nsi + i] & IN_CUT) != 0;
  if (num_in) num_in[i] = nin;
  int a = 0, b = nin;   // next in-cutoff and next other position
  for (int k = 0; k < n; k++) {
    size_t o = (size_t)k * nsi + i;
    unsigned char im = img[o];
    int v = raw[o];
    int sidx;
    if (v & KIND_SITE) {
      int gid = v & ~KIND_SITE;
      int e = gid / NU, u = gid % NU;
      int g = site_gauss(u);
      sidx = (g >= 0) ? na + NG * e + g : na + NG * ne + pref[gid];
    } else {
      sidx = atom_slot[v];
    }
    const int w = (im & IN_CUT) ? a++ : b++;
    out[(size_t)w * nsi + i] = (sidx << IMG_BITS) | (im & (IN_CUT - 1));
  }
}

// Converts the element-site entries of the full lists (rows site_from.x ..
// num_in - 1 of the front segment, cap - back .. cap - 1 - site_from.y of the
// back one) from lattice-site ids to pair-table indices: Gauss points at
// their fixed place, the other sites by their rank among the marked ones.
__global__ void k_remap_sites(const int *raw, const unsigned char *img, const int *num, const int *num_in,
                              const int2 *site_from, int nsi, int cap, const int *pref, int na, int ne, int *out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nsi) return;
  const int nin = num_in[i], nback = num[i] - nin;
  if (nin + nback > cap) return;   // overflow: the build is repeated
  const int2 from = site_from[i];
  auto one = [&](int row) {
    const size_t o = (size_t)row * nsi + i;
    const int gid = raw[o] & ~KIND_SITE;
    const int e = gid / NU, u = gid % NU;
    const int g = site_gauss(u);
    const int sidx = (g >= 0) ? na + NG * e + g : na + NG * ne + pref[gid];
    out[o] = (sidx << IMG_BITS) | img[o];
  };
  for (int k = from.x; k < nin; k++) one(k);
  for (int k = from.y; k < nback; k++) one(cap - 1 - k);
}

inline int nblk(long n, int t) { return (int)((n + t - 1) / t); }

// Reference atom bins of a single system (nbin_standard.cpp:84-128),
// orthogonal box: used only by the half-list storage rule.
void setup_ref_bins(Ctx &c) {
  double binsize_optimal = 0.5 * c.cutneigh;
  double binsizeinv = 1.0 / binsize_optimal;
  for (int d = 0; d < 3; d++) {
    double bbox = c.boxhi[d] - c.boxlo[d];
    c.rbins.lo[d] = c.boxlo[d];
    c.rbins.hi[d] = c.boxhi[d];
    int nb = (int)(bbox * binsizeinv);
    if (nb == 0) nb = 1;
    c.rbins.nbin[d] = nb;
    double bs = bbox / nb;
    c.rbins.inv[d] = 1.0 / bs;
  }
}

// Candidate grids of one replica: atoms in cells >= cutneigh, element
// centres in cells >= cutneigh + element reach.
void setup_grids(const Ctx &c, Rep &r, bool has_elements) {
  for (int d = 0; d < 3; d++) {
    double L = r.b.L[d];
    int na_c = (int)(L / c.cutneigh);
    if (na_c < 1) throw Error(CACB200_EINVAL, "box shorter than the neighbour cutoff");
    r.ag.nc[d] = na_c;
    r.ag.inv[d] = na_c / L;
    double reach = c.cutneigh + r.reach_budget + 1e-6;
    if (has_elements && L < reach)
      throw Error(CACB200_EINVAL, "box shorter than the cutoff plus the element radius in dimension " +
                                      std::to_string(d));
    int ne_c = std::max(1, (int)(L / reach));
    r.eg.nc[d] = ne_c;
    r.eg.inv[d] = ne_c / L;
  }
  r.ag.ncell = r.ag.nc[0] * r.ag.nc[1] * r.ag.nc[2];
  r.eg.ncell = r.eg.nc[0] * r.eg.nc[1] * r.eg.nc[2];
}

// Launch a rebuild kernel for a single system or a batch.
template <class F>
void with_reps(const Ctx &c, F &&f) {
  if (c.nrep == 1) {
    OneRep P{c.rep_h[0]};
    f(P);
  } else {
    ManyRep P{c.rep_d.p, c.site_rep.p, c.elem_rep.p, c.acell_rep.p};
    f(P);
  }
}

}  // namespace

// Capacity plan: sizes every buffer of a rebuild for the current system (site
// table for the worst case of every lattice site active, candidate grids with
// room for elements to grow, list slots of `cap` per site), so that rebuilds
// afterwards neither allocate nor synchronise and can be queued or captured
// in a CUDA graph.  Synchronises once to read the element radii.
void neigh_plan(Ctx &c, bool want_half) {
  c.check_system();
  if (c.pp.style == CACB200_PAIR_NONE) throw Error(CACB200_ESTATE, "no pair style set");
  if (want_half && c.nrep > 1) throw Error(CACB200_EINVAL, "half lists are built for single systems only");
  double cutoff = std::sqrt(c.pp.cut * c.pp.cut);
  c.cutneigh = cutoff + c.skin;
  c.cutneighsq = c.cutneigh * c.cutneigh;
  c.ecenter.reserve(std::max(c.ne, 1));
  c.eframe.reserve((size_t)std::max(c.ne, 1) * EFR);
  c.overflow.reserve(16);
  c.dev_nact.reserve(1);
  c.inner_margin = c.inner_margin_set >= 0.0 ? c.inner_margin_set : 0.5 * c.skin;
  c.inner_ok.reserve(c.nrep);
  c.disp.reserve(std::max(c.na, 1));
  c.edisp.reserve(std::max(c.ne, 1));
  c.dmax.reserve(c.nrep);
  c.xbuild.reserve(std::max(c.na, 1));
  c.nodex_build.reserve(24 * (size_t)std::max(c.ne, 1));
  c.num_in.reserve(std::max(c.nsite_i(), 1));
  c.reach_bits.reserve(c.nrep);
  c.rep_d.reserve(c.nrep);
  c.sm_counter.reserve(2 * c.num_sms);
  CACB200_CUDA(cudaMemsetAsync(c.overflow.p, 0, 16 * sizeof(int), c.stream));
  CACB200_CUDA(cudaMemsetAsync(c.dev_nact.p, 0, sizeof(int), c.stream));
  CACB200_CUDA(cudaMemsetAsync(c.reach_bits.p, 0, sizeof(unsigned long long) * c.nrep, c.stream));
  // element geometry with no reach limit, to measure each replica's radius
  for (Rep &r : c.rep_h) r.reach_budget = 1e300;
  stream_copy(c, c.rep_d.p, c.rep_h.data(), sizeof(Rep) * c.nrep, cudaMemcpyHostToDevice);
  std::vector<unsigned long long> bits(c.nrep, 0);
  if (c.ne) {
    with_reps(c, [&](auto P) {
      if (c.na) k_pbc_atoms<<<nblk(c.na, 256), 256, 0, c.stream>>>(c.xs.p, c.na, P);
      k_elem_geom<<<nblk(c.ne, 128), 128, 0, c.stream>>>(c.nodex.p, c.ne, P, c.ecenter.p, c.eframe.p,
                                                         c.reach_bits.p, c.overflow.p + 3);
    });
    stream_copy(c, bits.data(), c.reach_bits.p, sizeof(unsigned long long) * c.nrep, cudaMemcpyDeviceToHost);
  }
  int abase = 0, ebase = 0;
  for (int r = 0; r < c.nrep; r++) {
    Rep &R = c.rep_h[r];
    double ereach = 0.0;
    std::memcpy(&ereach, &bits[r], sizeof(double));
    if (!(ereach < 1e30)) throw Error(CACB200_EUNSTABLE, "non-finite element geometry");
    // elements may grow by 20 % (and 2 A) before the grid is planned again,
    // as far as the box allows
    R.reach_budget = 0.0;
    if (c.rep_ne[r]) {
      double room = std::min(R.b.L[0], std::min(R.b.L[1], R.b.L[2])) - c.cutneigh - 2e-6;
      R.reach_budget = std::max(ereach, std::min(std::max(1.2 * ereach, ereach + 2.0), room));
    }
    setup_grids(c, R, c.rep_ne[r] > 0);
    // FP32 separations (a wrapped position less an image shift, |.| <= 2X
    // with X = |lo| + |hi| + L, minus a wrapped candidate) carry at most ~4
    // ulp(X) of rounding per distance; 16 ulp of 2X bounds it with room to
    // spare
    {
      double X = 1.0;
      for (int d = 0; d < 3; d++) X = std::max(X, std::fabs(R.b.lo[d]) + std::fabs(R.b.hi[d]) + R.b.L[d]);
      R.fmargin = (float)(16.0 * std::ldexp(1.0, std::ilogb(2.0 * X) - 23));
    }
    // fixed-point frame of the mixed form: quantum 2^-26 A, box length in
    // quanta modulo 2^32 (pair separations are taken modulo 2^32 as well)
    for (int d = 0; d < 3; d++) {
      R.qscale[d] = std::ldexp(1.0, 26);
      R.qinv[d] = std::ldexp(1.0f, -26);
      R.Lq[d] = (int)(uint32_t)(uint64_t)std::llrint(R.b.L[d] * R.qscale[d]);
    }
    R.abase = abase;
    R.ebase = ebase;
    abase += R.ag.ncell;
    ebase += R.eg.ncell;
  }
  stream_copy(c, c.rep_d.p, c.rep_h.data(), sizeof(Rep) * c.nrep, cudaMemcpyHostToDevice);
  c.agrid.ncell = abase;
  c.egrid.ncell = ebase;
  if (c.nrep > 1) {
    std::vector<int> cr(abase);
    for (int r = 0; r < c.nrep; r++)
      std::fill(cr.begin() + c.rep_h[r].abase, cr.begin() + c.rep_h[r].abase + c.rep_h[r].ag.ncell, r);
    c.acell_rep.reserve(abase);
    stream_copy(c, c.acell_rep.p, cr.data(), sizeof(int) * abase, cudaMemcpyHostToDevice);
  } else {
    setup_ref_bins(c);
  }

  const int nsi = c.nsite_i();
  const size_t ngid = (size_t)c.ne * NU;
  int nmax = std::max(std::max(c.na, c.ne), 1);
  c.cell_key.reserve(nmax);
  c.cell_key2.reserve(nmax);
  c.idx_tmp.reserve(nmax);
  c.slot_atom.reserve(nmax);
  c.atom_slot.reserve(std::max(c.na, 1));
  c.xss.reserve(std::max(c.xs.n, (size_t)1));
  c.acell_start.reserve(c.agrid.ncell + 1);
  c.acell_pos.reserve(std::max(c.na, 1));
  c.acell_pos32.reserve(std::max(c.na, 1));
  c.acell_of.reserve(std::max(c.na, 1));
  c.ecell_start.reserve(c.egrid.ncell + 1);
  c.ecell_near.reserve(c.egrid.ncell + 1);
  c.acell_near.reserve(c.agrid.ncell + 1);
  c.ecell_elems.reserve(std::max(c.ne, 1));
  size_t slots = (size_t)c.cap * std::max(nsi, 1);
  c.raw_full.reserve(slots);
  c.img_full.reserve(slots);
  c.num_full.reserve(std::max(nsi, 1));
  c.site_from.reserve(std::max(nsi, 1));
  c.nbr_full.reserve(slots);
  if (want_half) {
    c.raw_half.reserve(slots);
    c.img_half.reserve(slots);
    c.num_half.reserve(std::max(nsi, 1));
    c.nbr_half.reserve(slots);
  }
  c.items.reserve((size_t)std::max(nsi, 1) * c.item_cap);
  c.nitems.reserve(std::max(nsi, 1));
  c.atom_work.reserve(std::max(c.na, 1));
  c.atom_nwork.reserve(1);
  c.site_flag.reserve(ngid + 1);
  c.site_pref.reserve(ngid + 1);
  c.act_gid.reserve(std::max<size_t>(ngid, 1));
  c.act_off.reserve(c.ne + 1);
  // site table for every lattice site active, keeping the atom positions
  size_t ns_cap = (size_t)nsi + ngid;
  if (ns_cap > c.xs.n) {
    double4 *np_ = nullptr;
    if (cudaMalloc(&np_, ns_cap * sizeof(double4)) != cudaSuccess) {
      cudaGetLastError();
      throw Error(CACB200_ENOMEM, "site table allocation failed");
    }
    if (c.na)
      CACB200_CUDA(cudaMemcpyAsync(np_, c.xs.p, sizeof(double4) * c.na, cudaMemcpyDeviceToDevice, c.stream));
    CACB200_CUDA(cudaStreamSynchronize(c.stream));
    cudaFree(c.xs.p);
    c.xs.p = np_;
    c.xs.n = ns_cap;
  }
  c.ns_cap = ns_cap;
  // CUB temporary storage for the largest sort and the scan
  size_t need = 0, bytes = 0;
  int bits_a = 1, bits_e = 1;
  while ((1 << bits_a) <= c.agrid.ncell && bits_a < 31) bits_a++;
  while ((1 << bits_e) <= c.egrid.ncell && bits_e < 31) bits_e++;
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, c.cell_key.p, c.cell_key2.p, c.idx_tmp.p, c.slot_atom.p,
                                  std::max(c.na, 1), 0, bits_a, c.stream);
  need = std::max(need, bytes);
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, c.cell_key.p, c.cell_key2.p, c.idx_tmp.p, c.ecell_elems.p,
                                  std::max(c.ne, 1), 0, bits_e, c.stream);
  need = std::max(need, bytes);
  cub::DeviceScan::ExclusiveSum(nullptr, bytes, c.site_flag.p, c.site_pref.p, (int)(ngid + 1), c.stream);
  need = std::max(need, bytes);
  c.cub_tmp.reserve(need);
  c.cub_bytes = need;
  c.sort_bits_a = bits_a;
  c.sort_bits_e = bits_e;
  c.plan_half = want_half;
  c.planned = true;
  const long gen_before = c.gen;
  c.gen++;
  if (c.box_replan) {
    // only the box moved (fix deform): the block sizes chosen for this
    // system stay valid
    if (c.tune_gen == gen_before) c.tune_gen = c.gen;
    if (c.tune_gen32 == gen_before) c.tune_gen32 = c.gen;
    c.box_replan = false;
  }
  c.plan_na = c.na;
  c.plan_ne = c.ne;
}

// Queue a rebuild: pbc, element geometry, binning, candidate search, storage
// rules, compaction of the referenced lattice sites and packing of the list
// entries.  Nothing here allocates or waits for the device; problems are
// reported in the flag words (list overflow, distant image, element grown past
// the grid plan) for neigh_check.
void neigh_build_async(Ctx &c, bool want_half) {
  if (!c.planned || c.plan_na != c.na || c.plan_ne != c.ne || (want_half && !c.plan_half))
    throw Error(CACB200_ESTATE, "rebuild without a capacity plan");
  const int nsi = c.nsite_i();
  const size_t ngid = (size_t)c.ne * NU;
  CACB200_CUDA(cudaMemsetAsync(c.overflow.p, 0, 4 * sizeof(int), c.stream));
  CACB200_CUDA(cudaMemsetAsync(c.overflow.p + 8, 0, 2 * sizeof(int), c.stream));
  with_reps(c, [&](auto P) {
    {
      KernelTimer t(c, "pbc_geom");
      if (c.na) k_pbc_atoms<<<nblk(c.na, 256), 256, 0, c.stream>>>(c.xs.p, c.na, P);
      if (c.ne)
        k_elem_geom<<<nblk(c.ne, 128), 128, 0, c.stream>>>(c.nodex.p, c.ne, P, c.ecenter.p, c.eframe.p,
                                                           c.reach_bits.p, c.overflow.p + 3);
    }
    // the positions these lists are built from, for the displacement test of
    // the inner prefix; the prefix is usable until a site moves half the margin
    if (c.na)
      CACB200_CUDA(cudaMemcpyAsync(c.xbuild.p, c.xs.p, sizeof(double4) * c.na, cudaMemcpyDeviceToDevice, c.stream));
    if (c.ne)
      CACB200_CUDA(cudaMemcpyAsync(c.nodex_build.p, c.nodex.p, sizeof(double) * 24 * c.ne,
                                   cudaMemcpyDeviceToDevice, c.stream));
    CACB200_CUDA(cudaMemsetAsync(c.inner_ok.p, inner_limit(c) > 0.0 ? 1 : 0, sizeof(int) * c.nrep, c.stream));
    // every site is where the lists are built from
    if (c.na) CACB200_CUDA(cudaMemsetAsync(c.disp.p, 0, sizeof(float) * c.na, c.stream));
    if (c.ne) CACB200_CUDA(cudaMemsetAsync(c.edisp.p, 0, sizeof(float) * c.ne, c.stream));
    CACB200_CUDA(cudaMemsetAsync(c.dmax.p, 0, sizeof(unsigned) * c.nrep, c.stream));
    {
      KernelTimer t(c, "bin");
      size_t bytes = c.cub_bytes;
      if (c.na) {
        k_atom_keys<<<nblk(c.na, 256), 256, 0, c.stream>>>(c.xs.p, c.na, P, c.cell_key.p, c.idx_tmp.p);
        CACB200_CUDA(cub::DeviceRadixSort::SortPairs(c.cub_tmp.p, bytes, c.cell_key.p, c.cell_key2.p,
                                                     c.idx_tmp.p, c.slot_atom.p, c.na, 0, c.sort_bits_a,
                                                     c.stream));
        k_cell_start<<<nblk(c.agrid.ncell + 1, 256), 256, 0, c.stream>>>(c.cell_key2.p, c.na, c.agrid.ncell,
                                                                        c.acell_start.p);
        if (c.nrep == 1 && c.ne)
          k_ecell_near<<<nblk(c.agrid.ncell, 256), 256, 0, c.stream>>>(c.acell_start.p, c.rep_h[0].ag,
                                                                       c.acell_near.p);
        k_gather_pos<<<nblk(c.na, 256), 256, 0, c.stream>>>(c.xs.p, c.slot_atom.p, c.cell_key2.p, c.na,
                                                            c.acell_pos.p, c.acell_pos32.p, c.atom_slot.p,
                                                            c.acell_of.p);
      } else {
        CACB200_CUDA(cudaMemsetAsync(c.acell_start.p, 0, sizeof(int) * (c.agrid.ncell + 1), c.stream));
      }
      if (c.ne) {
        bytes = c.cub_bytes;
        k_elem_keys<<<nblk(c.ne, 256), 256, 0, c.stream>>>(c.ecenter.p, c.ne, P, c.cell_key.p, c.idx_tmp.p);
        CACB200_CUDA(cub::DeviceRadixSort::SortPairs(c.cub_tmp.p, bytes, c.cell_key.p, c.cell_key2.p,
                                                     c.idx_tmp.p, c.ecell_elems.p, c.ne, 0, c.sort_bits_e,
                                                     c.stream));
        k_cell_start<<<nblk(c.egrid.ncell + 1, 256), 256, 0, c.stream>>>(c.cell_key2.p, c.ne, c.egrid.ncell,
                                                                        c.ecell_start.p);
        if (c.nrep == 1)
          k_ecell_near<<<nblk(c.egrid.ncell, 256), 256, 0, c.stream>>>(c.ecell_start.p, c.rep_h[0].eg,
                                                                       c.ecell_near.p);
      } else {
        CACB200_CUDA(cudaMemsetAsync(c.ecell_start.p, 0, sizeof(int) * (c.egrid.ncell + 1), c.stream));
      }
    }
    BuildArgs A;
    A.xs = c.xs.p;
    A.nodex = c.nodex.p;
    A.ecenter = c.ecenter.p;
    A.eframe = c.eframe.p;
    A.acell_start = c.acell_start.p;
    A.acell_pos = c.acell_pos.p;
    A.acell_pos32 = c.acell_pos32.p;
    A.acell_of = c.acell_of.p;
    A.ecell_start = c.ecell_start.p;
    A.ecell_near = (c.nrep == 1 && c.ne) ? c.ecell_near.p : nullptr;
    A.acell_near = (c.nrep == 1 && c.na && c.ne) ? c.acell_near.p : nullptr;
    A.ecell_elems = c.ecell_elems.p;
    A.atom_of_slot = c.slot_atom.p;
    A.site_flag = c.site_flag.p;
    if (ngid) CACB200_CUDA(cudaMemsetAsync(c.site_flag.p, 0, sizeof(int) * (ngid + 1), c.stream));
    A.na = c.na;
    A.ne = c.ne;
    A.nsi = nsi;
    A.cap = c.cap;
    A.rb = c.rbins;
    A.cutneigh = c.cutneigh;
    A.cutneighsq = c.cutneighsq;
    A.cutforcesq = (c.pp.cut + c.inner_margin) * (c.pp.cut + c.inner_margin);
    A.want_half = want_half ? 1 : 0;
    A.nbr_full = c.nbr_full.p;
    A.num_in = c.num_in.p;
    A.site_from = c.site_from.p;
    A.raw_full = c.raw_full.p;
    A.num_full = c.num_full.p;
    A.img_full = c.img_full.p;
    A.raw_half = want_half ? c.raw_half.p : nullptr;
    A.num_half = want_half ? c.num_half.p : nullptr;
    A.img_half = want_half ? c.img_half.p : nullptr;
    A.overflow = c.overflow.p;
    // The atom-atom lists need no element work: they run on the context
    // stream while the side stream does phase A for every slot and then the
    // Gauss-point lists (disjoint slots); the atoms' element sites follow the
    // atom-atom lists once phase A is done.  Timed one kernel at a time when
    // profiling.
    const bool split = c.na && c.ne && !c.prof.enabled;
    cudaStream_t es = split ? c.side : c.stream;
    if (split) {
      CACB200_CUDA(cudaEventRecord(c.fork_ev, c.stream));
      CACB200_CUDA(cudaStreamWaitEvent(c.side, c.fork_ev, 0));
    }
    if (c.ne) {
      {
        KernelTimer t(c, "build_items");
        CACB200_CUDA(cudaMemsetAsync(c.atom_nwork.p, 0, sizeof(int), es));
        k_elem_items<<<nblk(nsi, 128), 128, 0, es>>>(A, P, c.items.p, c.nitems.p, c.item_cap, c.atom_work.p,
                                                    c.atom_nwork.p);
      }
      if (split) CACB200_CUDA(cudaEventRecord(c.items_ev, c.side));
      {
        KernelTimer t(c, "build_gauss");
        k_build_gauss<<<nblk(32L * NG * c.ne, 128), 128, 0, es>>>(A, P, c.items.p, c.nitems.p, c.item_cap);
      }
      if (split) CACB200_CUDA(cudaEventRecord(c.join_ev, c.side));
    }
    if (c.na) {
      KernelTimer t(c, "build_atoms");
      if constexpr (std::is_same_v<decltype(P), OneRep>) {
        if (c.work_queue) {
          static const int per_sm = [] {
            int b = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_build_atoms_sm, 32, 0);
            return b > 0 ? b : 1;
          }();
          CACB200_CUDA(cudaMemsetAsync(c.sm_counter.p, 0, sizeof(int) * c.num_sms, c.stream));
          k_build_atoms_sm<<<per_sm * c.num_sms, 32, 0, c.stream>>>(A, P, (c.na + 31) / 32, c.sm_counter.p,
                                                                   c.num_sms);
        } else {
          k_build_atoms<<<(c.na + 31) / 32, 32, 0, c.stream>>>(A, P);
        }
      } else {
        k_build_atoms<<<(c.na + 31) / 32, 32, 0, c.stream>>>(A, P);
      }
    }
    if (c.na && c.ne) {
      if (split) CACB200_CUDA(cudaStreamWaitEvent(c.stream, c.items_ev, 0));
      KernelTimer t(c, "build_atom_sites");
      // the warps stride over the work list: one wave of resident blocks
      static const int per_sm = [] {
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_build_atom_sites<decltype(P)>, 128, 0);
        return b > 0 ? b : 1;
      }();
      const int grid = (int)std::min<long>(stride_grid(32L * c.na, 128), (long)per_sm * c.num_sms);
      k_build_atom_sites<<<grid, 128, 0, c.stream>>>(A, P, c.items.p, c.nitems.p, c.item_cap, c.atom_work.p,
                                                     c.atom_nwork.p);
    }
    if (split) CACB200_CUDA(cudaStreamWaitEvent(c.stream, c.join_ev, 0));
  });
  {
    KernelTimer t(c, "compact");
    int *flag = c.site_flag.p;
    int *pref = c.site_pref.p;
    if (ngid) {
      size_t bytes = c.cub_bytes;
      CACB200_CUDA(cub::DeviceScan::ExclusiveSum(c.cub_tmp.p, bytes, flag, pref, (int)(ngid + 1), c.stream));
      k_act_table<<<nblk((long)ngid, 256), 256, 0, c.stream>>>(flag, pref, (int)ngid, c.ne, nsi, c.act_gid.p,
                                                              c.act_off.p, c.dev_nact.p, c.overflow.p + 7);
    }
    if (c.ne)
      k_remap_sites<<<nblk(nsi, 256), 256, 0, c.stream>>>(c.raw_full.p, c.img_full.p, c.num_full.p, c.num_in.p,
                                                         c.site_from.p, nsi, c.cap, pref, c.na, c.ne,
                                                         c.nbr_full.p);
    if (want_half)
      k_remap<<<nblk(nsi, 256), 256, 0, c.stream>>>(c.raw_half.p, c.img_half.p, c.num_half.p, nsi, c.cap, pref,
                                                     c.atom_slot.p, c.na, c.ne, c.nbr_half.p, nullptr);
  }
  c.have_half = want_half;
  c.lists_valid = true;
  c.nact_known = false;
  c.build_count++;
  CACB200_CUDA(cudaGetLastError());
}

// Read the rebuild's flag words (synchronises).  Returns 0 when the lists are
// good, 1 when a capacity must grow (the plan was updated: rebuild again).
int neigh_check(Ctx &c) {
  int ov[16];
  stream_copy(c, ov, c.overflow.p, sizeof(ov), cudaMemcpyDeviceToHost);
  if (ov[2]) throw Error(CACB200_EINVAL, "neighbour image beyond the first periodic image (box too small)");
  if (ov[6]) throw Error(CACB200_EUNSTABLE, "a site position is not finite or absurdly far from the box (unstable run)");
  if (ov[7]) throw Error(CACB200_EOVERFLOW, "more referenced sites than 26-bit list entries can address");
  int again = 0;
  if (ov[0]) {
    c.cap = ((ov[1] + 31) / 32) * 32;
    again = 1;
  }
  if (ov[3]) again = 1;   // an element outgrew the candidate grid
  if (ov[8]) {            // a query met more element boxes than its item slots
    c.item_cap = ((ov[9] + 15) / 16) * 16;
    again = 1;
  }
  if (again) {
    c.lists_valid = false;
    neigh_plan(c, c.plan_half);
  }
  return again;
}

// Synchronous rebuild with retries (API calls, setup, tests).
void neigh_build(Ctx &c, bool want_half) {
  c.check_system();
  if (!c.planned || c.plan_na != c.na || c.plan_ne != c.ne || (want_half && !c.plan_half))
    neigh_plan(c, want_half || c.plan_half);
  for (int attempt = 0; attempt < 4; attempt++) {
    neigh_build_async(c, want_half);
    if (!neigh_check(c)) {
      note_build_box(c);
      return;
    }
  }
  throw Error(CACB200_EOVERFLOW, "neighbour list capacity could not be settled");
}

int device_nact(Ctx &c) {
  if (!c.nact_known) {
    int n = 0;
    if (c.ne) stream_copy(c, &n, c.dev_nact.p, sizeof(int), cudaMemcpyDeviceToHost);
    c.nact = n;
    c.nact_known = true;
  }
  return c.nact;
}

void neigh_download(Ctx &c, bool half, int64_t *offset, int8_t *kind, int32_t *idx, int32_t *site,
                    int8_t *img, int64_t *nentries) {
  if (!c.lists_valid || (half && !c.have_half)) throw Error(CACB200_ESTATE, "list not built");
  const int nsi = c.nsite_i();
  std::vector<int> num_slot(nsi), num(nsi), slot_of(nsi), nin_slot(nsi, 0);
  std::vector<int> ent((size_t)c.cap * nsi);
  std::vector<int> atom_of(std::max(c.na, 1));
  device_nact(c);
  std::vector<int> act(std::max(c.nact, 1));
  CACB200_CUDA(cudaStreamSynchronize(c.stream));
  stream_copy(c, num_slot.data(), half ? c.num_half.p : c.num_full.p, sizeof(int) * nsi,
                          cudaMemcpyDeviceToHost);
  if (!half) stream_copy(c, nin_slot.data(), c.num_in.p, sizeof(int) * nsi, cudaMemcpyDeviceToHost);
  if (c.na) stream_copy(c, atom_of.data(), c.slot_atom.p, sizeof(int) * c.na, cudaMemcpyDeviceToHost);
  for (int k = 0; k < nsi; k++) slot_of[k] = k;
  for (int h = 0; h < c.na; h++) slot_of[atom_of[h]] = h;
  for (int i = 0; i < nsi; i++) num[i] = num_slot[slot_of[i]];
  stream_copy(c, ent.data(), half ? c.nbr_half.p : c.nbr_full.p, sizeof(int) * ent.size(),
                          cudaMemcpyDeviceToHost);
  if (c.nact)
    stream_copy(c, act.data(), c.act_gid.p, sizeof(int) * c.nact, cudaMemcpyDeviceToHost);
  int64_t total = 0;
  for (int i = 0; i < nsi; i++) total += num[i];
  *nentries = total;
  if (!offset) return;
  int64_t pos = 0;
  std::vector<std::tuple<int, int, int, int, int, int>> row;
  for (int i = 0; i < nsi; i++) {
    offset[i] = pos;
    row.clear();
    const int sl = slot_of[i], nin = half ? num[i] : nin_slot[sl];
    for (int k = 0; k < num[i]; k++) {
      // full lists: the front segment, then the back one from row cap - 1 down
      const int r = k < nin ? k : c.cap - 1 - (k - nin);
      int v = ent[(size_t)r * nsi + sl];
      int sidx = v >> IMG_BITS, code = v & ((1 << IMG_BITS) - 1);
      int sx, sy, sz;
      img_decode(code, sx, sy, sz);
      int kd, id, st;
      if (sidx < c.na) {   // atoms are stored by list slot
        kd = 0;
        id = atom_of[sidx];
        st = -1;
      } else if (sidx < c.na + NG * c.ne) {
        kd = 1;
        id = (sidx - c.na) / NG;
        st = gauss_site((sidx - c.na) % NG);
      } else {
        int gid = act[sidx - c.na - NG * c.ne];
        kd = 1;
        id = gid / NU;
        st = gid % NU;
      }
      row.emplace_back(kd, id, st, sx, sy, sz);
    }
    std::sort(row.begin(), row.end());
    for (auto &t : row) {
      kind[pos] = (int8_t)std::get<0>(t);
      idx[pos] = std::get<1>(t);
      site[pos] = std::get<2>(t);
      img[3 * pos] = (int8_t)std::get<3>(t);
      img[3 * pos + 1] = (int8_t)std::get<4>(t);
      img[3 * pos + 2] = (int8_t)std::get<5>(t);
      pos++;
    }
  }
  offset[nsi] = pos;
}

}  // namespace cacb200
