// Pair kernels: LJ 12-6 and two-pass EAM over the full neighbour list.
//
// Each i-site (atom or Gauss point) gathers over its own full list, so every
// force, density and per-site energy is written once by one thread with no
// atomics; the totals equal the reference's half-list sums with reactions
// (pair_lj_cut.cpp:227-417, pair_eam.cpp:618-1031) up to summation order:
//   * an atom's force is the sum over every neighbour; a Gauss point's force
//     likewise (its atom neighbours are the reactions the reference applies
//     from atom lists);
//   * the global energy and virial are sum_i scale_i * sum_j term_ij with
//     scale 1/2 for atoms and nodal_weight/2 for node Gauss points (the
//     reference's iescale + jescale split over the two ends of a pair);
//   * per-site energy and virial are half of each pair term (Pair::ev_tally,
//     pair.cpp:428-482).
// EAM evaluates F'(rho) once per site (atoms and nodes from their own
// density, interpolated lattice sites from shape-weighted nodal density)
// instead of once per pair, and keeps it in the w slot of the site table so
// one 32-byte load brings a neighbour's position and F'.
#include <algorithm>
#include <cmath>
#include <vector>

#include "ctx.cuh"
#include "device.cuh"

namespace cacb200 {

namespace {

inline int nblk(long n, int t) { return (int)((n + t - 1) / t); }

struct PairArgs {
  const double4 *xs;                // pair table (list-slot order; w = F')
  const int *nbr;                   // lists and counts indexed by list slot
  const int *num;
  const int *num_in;                // inner prefix length of each list ...
  PrefixRule prefix;                // ... and the rule for walking the rest
  const int *slot_atom;             // list slot -> atom (slots past the atoms are Gauss points)
  int na, ne, nsi;
  int cap;                          // list rows: the rest of a list fills its last rows
  double L[3];                      // box of a single system
  const Rep *reps;                  // batches: replica descriptors ...
  const int *site_rep;              // ... and the replica of each i-site (null for one system)
  double *f, *gaussf;
  double *eatom, *vatom, *enode, *vnode;
  double *partial;
  int eflag, vflag;
  double escale_node, vscale_node;  // global scales of a node Gauss point
};

__device__ __forceinline__ int site_of_slot(const PairArgs &A, int t) { return t < A.na ? A.slot_atom[t] : t; }

// The FP64 EAM arithmetic in explicitly rounded operations, with no fused
// multiply-add: the operation order of the reference's source (compiled
// there without contraction), and the same rounding in every kernel that
// inlines it (grid and SM-local launches, grouped and remainder walks), where
// the compiler would otherwise contract each copy its own way.
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }

__device__ __forceinline__ void neighbour_pos(const PairArgs &A, double Lx, double Ly, double Lz, int v,
                                              double4 &xj) {
  int j = v >> IMG_BITS, code = v & ((1 << IMG_BITS) - 1);
  xj = ldg256(A.xs + j);
  if (code != IMG_ZERO) {
    int sx, sy, sz;
    img_decode(code, sx, sy, sz);
    xj.x = radd(xj.x, rmul((double)sx, Lx));
    xj.y = radd(xj.y, rmul((double)sy, Ly));
    xj.z = radd(xj.z, rmul((double)sz, Lz));
  }
}

// Walks a site's list four entries at a time: the four entry loads, then the
// four position loads, are issued back to back before any of them is used, so
// each thread keeps eight independent loads in flight instead of a chain of
// dependent pairs.  List entries are read once per pass: they are loaded as
// streaming (evict-first) so that L1 keeps the neighbour positions and spline
// records, which are reused.  MANY: the site belongs to a batch replica with
// its own box.
template <bool MANY, class F>
__device__ __forceinline__ void for_each_neighbour(const PairArgs &A, int i, const int *nb, int n, F &&f) {
  double Lx = A.L[0], Ly = A.L[1], Lz = A.L[2];
  if (MANY) {
    const Rep *r = A.reps + A.site_rep[i];
    Lx = r->b.L[0];
    Ly = r->b.L[1];
    Lz = r->b.L[2];
  }
  int k = 0;
  for (; k + 4 <= n; k += 4) {
    int v0 = __ldcs(nb + (size_t)k * A.nsi), v1 = __ldcs(nb + (size_t)(k + 1) * A.nsi);
    int v2 = __ldcs(nb + (size_t)(k + 2) * A.nsi), v3 = __ldcs(nb + (size_t)(k + 3) * A.nsi);
    double4 p0, p1, p2, p3;
    neighbour_pos(A, Lx, Ly, Lz, v0, p0);
    neighbour_pos(A, Lx, Ly, Lz, v1, p1);
    neighbour_pos(A, Lx, Ly, Lz, v2, p2);
    neighbour_pos(A, Lx, Ly, Lz, v3, p3);
    f(p0);
    f(p1);
    f(p2);
    f(p3);
  }
  for (; k < n; k++) {
    double4 p;
    neighbour_pos(A, Lx, Ly, Lz, __ldcs(nb + (size_t)k * A.nsi), p);
    f(p);
  }
}

// A site's list in two walks: the inner prefix (entries within the cutoff
// plus a margin at the build, the list's first rows), then, unless the
// site's displacement since the build and the largest one cannot close the
// margin (walk_rest, device.cuh), the rest (the list's last rows).  Each entry's arithmetic depends on its place in the walk (the
// compiler may fuse multiply-adds differently in the grouped and the
// remainder loop), so the prefix is always walked on its own: the sums are
// the same whether the rest is walked or not.
// The rule's flag and largest displacement belong to the site's replica (one
// hot replica of a batch does not end the shortcut for the others); one copy
// of the walk serves both segments, which keeps the register count of the
// unrolled body.
template <bool MANY, class F>
__device__ __forceinline__ void walk_list(const PairArgs &A, int i, const int *nb, int n_in, int n, F &&f) {
  const bool rest = n > n_in && walk_rest(A.prefix, i, MANY ? A.site_rep[i] : 0);
#pragma unroll 1
  for (int seg = 0; seg < (rest ? 2 : 1); seg++)
    for_each_neighbour<MANY>(A, i, seg ? nb + (size_t)(A.cap - (n - n_in)) * A.nsi : nb, seg ? n - n_in : n_in,
                             f);
}

// Writes force and per-site energy/virial of i-site i and accumulates the
// global sums (reduced per block in fixed order).
__device__ __forceinline__ void finish_site(const PairArgs &A, int i, bool valid, const double fi[3],
                                            double esum, const double vsum[6], double eextra_site,
                                            double eextra_global) {
  double red[7] = {0, 0, 0, 0, 0, 0, 0};
  if (valid) {
    bool atom = i < A.na;
    int e = 0, g = 0, node = 0;
    double *fo;
    if (atom) {
      fo = A.f + 3 * (size_t)i;
    } else {
      e = (i - A.na) / NG;
      g = (i - A.na) % NG;
      node = gauss_node(g);
      fo = A.gaussf + (size_t)e * 24 + 3 * g;
    }
    fo[0] = fi[0];
    fo[1] = fi[1];
    fo[2] = fi[2];
    double es = atom ? 0.5 : A.escale_node, vs = atom ? 0.5 : A.vscale_node;
    if (A.eflag & CACB200_ENERGY_GLOBAL) red[0] = es * esum + eextra_global;
    if (A.vflag & CACB200_VIRIAL_GLOBAL)
#pragma unroll
      for (int k = 0; k < 6; k++) red[1 + k] = vs * vsum[k];
    if (A.eflag & CACB200_ENERGY_ATOM) {
      double ev = 0.5 * esum + eextra_site;
      if (atom) A.eatom[i] = ev;
      else A.enode[(size_t)e * 8 + node] = ev;
    }
    if (A.vflag & CACB200_VIRIAL_ATOM) {
      double *vo = atom ? A.vatom + 6 * (size_t)i : A.vnode + 48 * (size_t)e + 6 * node;
#pragma unroll
      for (int k = 0; k < 6; k++) vo[k] = 0.5 * vsum[k];
    }
  }
  if (A.eflag || A.vflag) block_reduce_store<7>(red, A.partial);
}

// Force only (no energy or virial requested): one write per site.
__device__ __forceinline__ void finish_force(const PairArgs &A, int i, bool valid, const double fi[3]) {
  if (!valid) return;
  double *fo;
  if (i < A.na) {
    fo = A.f + 3 * (size_t)i;
  } else {
    int e = (i - A.na) / NG, g = (i - A.na) % NG;
    fo = A.gaussf + (size_t)e * 24 + 3 * g;
  }
  fo[0] = fi[0];
  fo[1] = fi[1];
  fo[2] = fi[2];
}

// ------------------------------------------------------------------- LJ

struct LjParams {
  double cutsq, lj1, lj2, lj3, lj4, offset;
};

template <bool EV, bool MANY>
__global__ void __launch_bounds__(128, EV ? 4 : 8) k_lj(PairArgs A, LjParams P) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;   // list slot
  const bool valid = t < A.nsi;
  const int i = valid ? site_of_slot(A, t) : 0;           // site-table index
  double fi[3] = {0, 0, 0}, esum = 0.0, vsum[6] = {0, 0, 0, 0, 0, 0};
  if (valid) {
    double4 xi = A.xs[t];
    const int n_in = A.num_in[t], n = A.num[t];
    const int *nb = A.nbr + t;
    auto pair = [&](const double4 &xj) {
      double dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
      double rsq = dx * dx + dy * dy + dz * dz;
      if (rsq < P.cutsq) {
        double r2inv = 1.0 / rsq;
        double r6inv = r2inv * r2inv * r2inv;
        double forcelj = r6inv * (P.lj1 * r6inv - P.lj2);
        double fpair = forcelj * r2inv;
        fi[0] += dx * fpair;
        fi[1] += dy * fpair;
        fi[2] += dz * fpair;
        if (EV && A.eflag) esum += r6inv * (P.lj3 * r6inv - P.lj4) - P.offset;
        if (EV && A.vflag) {
          vsum[0] += dx * dx * fpair;
          vsum[1] += dy * dy * fpair;
          vsum[2] += dz * dz * fpair;
          vsum[3] += dx * dy * fpair;
          vsum[4] += dx * dz * fpair;
          vsum[5] += dy * dz * fpair;
        }
      }
    };
    walk_list<MANY>(A, i, nb, n_in, n, pair);
  }
  if (EV) finish_site(A, i, valid, fi, esum, vsum, 0.0, 0.0);
  else finish_force(A, i, valid, fi);
}

// ------------------------------------------------------------------ EAM

// r-dependent splines as one 64-byte record per knot m: rz[2m] the rhor value
// coefficients (S3, S4, S5, S6 of PairEAM::interpolate), rz[2m+1] those of
// z2r.  A pair reads the record once; the derivative coefficients are the
// reference's (S0, S1, S2) = (3 S3, 2 S4, S5) / dr (pair_eam.cpp:612-614),
// applied as ((3 S3 p + 2 S4) p + S5) * (1/dr).
struct EamTables {
  const double4 *rz, *frho_val, *frho_der;
  double rdr, rdrho, rhomax, cutforcesq;
  int nr, nrho;
};

// F'(rho) and F(rho) on the frho spline row (PairEAM::compute_fp,
// pair_eam.cpp:1160-1169; the energy read on the same row, i.e. the
// reference with its coefficient pointer returned to the caller)
__device__ __forceinline__ double eam_fp(const EamTables &T, double rho, double *phi) {
  double p = radd(rmul(rho, T.rdrho), 1.0);
  int m = (int)p;
  m = max(1, min(m, T.nrho - 1));
  p = rsub(p, (double)m);
  p = fmin(p, 1.0);
  double4 d = T.frho_der[m];
  double fp = radd(rmul(radd(rmul(d.x, p), d.y), p), d.z);
  if (phi) {
    double4 v = T.frho_val[m];
    double e = radd(rmul(radd(rmul(radd(rmul(v.x, p), v.y), p), v.z), p), v.w);
    if (rho > T.rhomax) e = radd(e, rmul(fp, rsub(rho, T.rhomax)));
    *phi = e;
  }
  return fp;
}

// pass 1: density at atoms and node Gauss points (pair_eam.cpp:707-812), then
// F' at the site itself into xs[i].w (pair_eam.cpp:819-833 for atoms; for a
// node the reference's rhoi = noderho at :901-903).
template <bool MANY>
__device__ __forceinline__ void rho_slot(const PairArgs &A, const EamTables &T, int t, double *rho_out,
                                         double *phi_site) {
  const int i = site_of_slot(A, t);                       // site-table index
  double4 xi = A.xs[t];
  const int n_in = A.num_in[t], n = A.num[t];
  const int *nb = A.nbr + t;
  double rho = 0.0;
  auto pair = [&](const double4 &xj) {
    const double dx = rsub(xi.x, xj.x), dy = rsub(xi.y, xj.y), dz = rsub(xi.z, xj.z);
    const double rsq = radd(radd(rmul(dx, dx), rmul(dy, dy)), rmul(dz, dz));
    if (rsq < T.cutforcesq) {
      double p = radd(rmul(sqrt(rsq), T.rdr), 1.0);
      int m = (int)p;
      m = max(1, min(m, T.nr - 1));
      p = rsub(p, (double)m);
      p = fmin(p, 1.0);
      double4 c = ldg256(T.rz + 2 * m);
      rho = radd(rho, radd(rmul(radd(rmul(radd(rmul(c.x, p), c.y), p), c.z), p), c.w));
    }
  };
  walk_list<MANY>(A, i, nb, n_in, n, pair);
  int slot = i;
  if (i >= A.na) {
    int e = (i - A.na) / NG, g = (i - A.na) % NG;
    slot = A.na + 8 * e + gauss_node(g);
  }
  rho_out[slot] = rho;
  double phi = 0.0;
  double fp = eam_fp(T, rho, A.eflag ? &phi : nullptr);
  ((double *)A.xs)[4 * (size_t)t + 3] = fp;
  if (A.eflag) phi_site[i] = phi;
}

template <int TB, bool MANY>
__global__ void __launch_bounds__(TB, 1024 / TB) k_eam_rho(PairArgs A, EamTables T, double *rho_out,
                                                       double *phi_site) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;   // list slot
  if (t >= A.nsi) return;
  rho_slot<MANY>(A, T, t, rho_out, phi_site);
}

// Single systems: the force-only passes over SM-local runs of list slots
// (sm_run, device.cuh); each slot is computed by the same function as in the
// grid launch, so the results are the grid launch's bit for bit.
template <int TB>
__global__ void __launch_bounds__(TB, 1024 / TB) k_eam_rho_sm(PairArgs A, EamTables T, double *rho_out,
                                                          double *phi_site, int *cnt, int nsm) {
  __shared__ int v;
  if (threadIdx.x == 0) v = sm_id() % nsm;
  const int nrun = (A.nsi + TB - 1) / TB;
  for (;;) {
    const int r = sm_run(cnt, nsm, nrun, v);
    if (r < 0) return;
    const int t = r * TB + threadIdx.x;
    if (t < A.nsi) rho_slot<false>(A, T, t, rho_out, phi_site);
  }
}

// F' at interpolated lattice sites from shape-weighted nodal density
// (pair_eam.cpp:957-969)
__global__ void k_eam_site_fp(double4 *xs, const int *act_gid, const int *nact_dev, int base, int na,
                              const double *rho, EamTables T) {
  const int nact = *nact_dev;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nact; k += gridDim.x * blockDim.x) {
    int gid = act_gid[k];
    int e = gid / NU, u = gid % NU;
    const double *rn = rho + na + 8 * (size_t)e;
    double r = 0.0;
#pragma unroll
    for (int n = 0; n < NPE; n++) r = radd(r, rmul(shape_val(u, n), rn[n]));
    xs[base + k].w = eam_fp(T, r, nullptr);
  }
}

// pass 2: forces (pair_eam.cpp:845-1028)
template <bool EV, bool MANY>
__device__ __forceinline__ void force_slot(const PairArgs &A, const EamTables &T, int t, int i,
                                           const double *phi_site, double fi[3], double &esum, double vsum[6],
                                           double &eemb_site, double &eemb_global) {
  {
    double4 xi = A.xs[t];
    double fpi = xi.w;
    const int n_in = A.num_in[t], n = A.num[t];
    const int *nb = A.nbr + t;
    auto pair = [&](const double4 &xj) {
      const double dx = rsub(xi.x, xj.x), dy = rsub(xi.y, xj.y), dz = rsub(xi.z, xj.z);
      const double rsq = radd(radd(rmul(dx, dx), rmul(dy, dy)), rmul(dz, dz));
      if (rsq < T.cutforcesq) {
        const double r = sqrt(rsq);
        double p = radd(rmul(r, T.rdr), 1.0);
        int m = (int)p;
        m = max(1, min(m, T.nr - 1));
        p = rsub(p, (double)m);
        p = fmin(p, 1.0);
        double4 rv = ldg256(T.rz + 2 * m);
        double4 zv = ldg256(T.rz + 2 * m + 1);
        const double rhop = rmul(radd(rmul(radd(rmul(rmul(3.0, rv.x), p), rmul(2.0, rv.y)), p), rv.z), T.rdr);
        const double z2p = rmul(radd(rmul(radd(rmul(rmul(3.0, zv.x), p), rmul(2.0, zv.y)), p), zv.z), T.rdr);
        const double z2 = radd(rmul(radd(rmul(radd(rmul(zv.x, p), zv.y), p), zv.z), p), zv.w);
        const double recip = 1.0 / r;
        const double phi = rmul(z2, recip);
        const double phip = rsub(rmul(z2p, recip), rmul(phi, recip));
        const double psip = radd(radd(rmul(fpi, rhop), rmul(xj.w, rhop)), phip);
        const double fpair = -rmul(psip, recip);
        fi[0] = radd(fi[0], rmul(dx, fpair));
        fi[1] = radd(fi[1], rmul(dy, fpair));
        fi[2] = radd(fi[2], rmul(dz, fpair));
        if (EV && A.eflag) esum = radd(esum, phi);
        if (EV && A.vflag) {
          vsum[0] = radd(vsum[0], rmul(rmul(dx, dx), fpair));
          vsum[1] = radd(vsum[1], rmul(rmul(dy, dy), fpair));
          vsum[2] = radd(vsum[2], rmul(rmul(dz, dz), fpair));
          vsum[3] = radd(vsum[3], rmul(rmul(dx, dy), fpair));
          vsum[4] = radd(vsum[4], rmul(rmul(dx, dz), fpair));
          vsum[5] = radd(vsum[5], rmul(rmul(dy, dz), fpair));
        }
      }
    };
    walk_list<MANY>(A, i, nb, n_in, n, pair);
    if (EV && A.eflag) {
      double phi = phi_site[i];
      eemb_site = phi;
      eemb_global = (i < A.na) ? phi : phi * A.escale_node * 2.0;
    }
  }
}

template <int TB, bool EV, bool MANY>
__global__ void __launch_bounds__(TB, (EV ? 512 : 768) / TB) k_eam_force(PairArgs A, EamTables T,
                                                                       const double *phi_site) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;   // list slot
  const bool valid = t < A.nsi;
  const int i = valid ? site_of_slot(A, t) : 0;           // site-table index
  double fi[3] = {0, 0, 0}, esum = 0.0, vsum[6] = {0, 0, 0, 0, 0, 0};
  double eemb_site = 0.0, eemb_global = 0.0;
  if (valid) force_slot<EV, MANY>(A, T, t, i, phi_site, fi, esum, vsum, eemb_site, eemb_global);
  if (EV) finish_site(A, i, valid, fi, esum, vsum, eemb_site, eemb_global);
  else finish_force(A, i, valid, fi);
}

template <int TB>
__global__ void __launch_bounds__(TB, 768 / TB) k_eam_force_sm(PairArgs A, EamTables T, const double *phi_site,
                                                           int *cnt, int nsm) {
  __shared__ int v;
  if (threadIdx.x == 0) v = sm_id() % nsm;
  const int nrun = (A.nsi + TB - 1) / TB;
  for (;;) {
    const int r = sm_run(cnt, nsm, nrun, v);
    if (r < 0) return;
    const int t = r * TB + threadIdx.x;
    if (t < A.nsi) {
      const int i = site_of_slot(A, t);
      double fi[3] = {0, 0, 0}, esum = 0.0, vsum[6] = {0, 0, 0, 0, 0, 0};
      double eemb_site = 0.0, eemb_global = 0.0;
      force_slot<false, false>(A, T, t, i, phi_site, fi, esum, vsum, eemb_site, eemb_global);
      finish_force(A, i, true, fi);
    }
  }
}

__global__ void k_reduce_partials(const double *partial, int nblocks, double *out) {
  // one warp per component, fixed order
  int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (k >= 7) return;
  double s = 0.0;
  for (int b = lane; b < nblocks; b += 32) s += partial[b * 7 + k];
  s = warp_sum(s);
  if (lane == 0) out[k] = s;
}

// ---------------------------------------------------------- spline tables

// PairEAM::interpolate (pair_eam.cpp:580-616): 7 coefficients per knot m = 1..n
void spline7(int n, double delta, const std::vector<double> &f1, std::vector<double> &sp) {
  sp.assign((size_t)(n + 1) * 7, 0.0);
  auto S = [&](int m, int c) -> double & { return sp[(size_t)m * 7 + c]; };
  for (int m = 1; m <= n; m++) S(m, 6) = f1[m];
  S(1, 5) = S(2, 6) - S(1, 6);
  S(2, 5) = 0.5 * (S(3, 6) - S(1, 6));
  S(n - 1, 5) = 0.5 * (S(n, 6) - S(n - 2, 6));
  S(n, 5) = S(n, 6) - S(n - 1, 6);
  for (int m = 3; m <= n - 2; m++)
    S(m, 5) = ((S(m - 2, 6) - S(m + 2, 6)) + 8.0 * (S(m + 1, 6) - S(m - 1, 6))) / 12.0;
  for (int m = 1; m <= n - 1; m++) {
    S(m, 4) = 3.0 * (S(m + 1, 6) - S(m, 6)) - 2.0 * S(m, 5) - S(m + 1, 5);
    S(m, 3) = S(m, 5) + S(m + 1, 5) - 2.0 * (S(m + 1, 6) - S(m, 6));
  }
  S(n, 4) = 0.0;
  S(n, 3) = 0.0;
  for (int m = 1; m <= n; m++) {
    S(m, 2) = S(m, 5) / delta;
    S(m, 1) = 2.0 * S(m, 4) / delta;
    S(m, 0) = 3.0 * S(m, 3) / delta;
  }
}

void upload_split(Ctx &c, const std::vector<double> &sp, int n, DBuf<double4> &val, DBuf<double4> &der) {
  std::vector<double4> hv(n + 1), hd(n + 1);
  for (int m = 0; m <= n; m++) {
    const double *r = &sp[(size_t)m * 7];
    hv[m] = make_double4(r[3], r[4], r[5], r[6]);
    hd[m] = make_double4(r[0], r[1], r[2], 0.0);
  }
  val.reserve(n + 1);
  der.reserve(n + 1);
  stream_copy(c, val.p, hv.data(), sizeof(double4) * (n + 1), cudaMemcpyHostToDevice);
  stream_copy(c, der.p, hd.data(), sizeof(double4) * (n + 1), cudaMemcpyHostToDevice);
}

}  // namespace

void eam_tables(Ctx &c, const double *frho, const double *rhor, const double *z2r) {
  PairParams &p = c.pp;
  std::vector<double> a(p.nrho + 1, 0.0), b(p.nr + 1, 0.0), z(p.nr + 1, 0.0), sp;
  for (int m = 1; m <= p.nrho; m++) a[m] = frho[m - 1];
  for (int m = 1; m <= p.nr; m++) {
    b[m] = rhor[m - 1];
    z[m] = z2r[m - 1];
  }
  c.have_mixed_tables = false;
  spline7(p.nrho, p.drho, a, sp);
  upload_split(c, sp, p.nrho, c.frho_val, c.frho_der);
  spline7(p.nr, p.dr, b, sp);
  upload_split(c, sp, p.nr, c.rhor_val, c.rhor_der);
  std::vector<double4> rz((size_t)2 * (p.nr + 1));
  for (int m = 0; m <= p.nr; m++) {
    const double *r = &sp[(size_t)m * 7];
    rz[2 * m] = make_double4(r[3], r[4], r[5], r[6]);
  }
  spline7(p.nr, p.dr, z, sp);
  upload_split(c, sp, p.nr, c.z2r_val, c.z2r_der);
  for (int m = 0; m <= p.nr; m++) {
    const double *r = &sp[(size_t)m * 7];
    rz[2 * m + 1] = make_double4(r[3], r[4], r[5], r[6]);
  }
  c.rz.reserve(rz.size());
  stream_copy(c, c.rz.p, rz.data(), sizeof(double4) * rz.size(), cudaMemcpyHostToDevice);
}

// Block size of the force-only pair passes, chosen per context by timing 64,
// 128 and 256 threads (best of three launches each; 128 unless another is at
// least 3 % faster) on the context's own lists the first time they run
// (every thread owns one list slot, so results do not depend on the choice;
// the passes are idempotent, so the trial launches change nothing).  Not
// during stream capture: there the default stays.
template <bool MANY>
void launch_rho(int tb, int nsi, cudaStream_t st, const PairArgs &A, const EamTables &T, double *rho, double *phi) {
  if (tb == 64) k_eam_rho<64, MANY><<<std::max(nblk(nsi, 64), 1), 64, 0, st>>>(A, T, rho, phi);
  else if (tb == 256) k_eam_rho<256, MANY><<<std::max(nblk(nsi, 256), 1), 256, 0, st>>>(A, T, rho, phi);
  else k_eam_rho<128, MANY><<<std::max(nblk(nsi, 128), 1), 128, 0, st>>>(A, T, rho, phi);
}
template <bool MANY>
void launch_force(int tb, int nsi, cudaStream_t st, const PairArgs &A, const EamTables &T, const double *phi) {
  if (tb == 64) k_eam_force<64, false, MANY><<<std::max(nblk(nsi, 64), 1), 64, 0, st>>>(A, T, phi);
  else if (tb == 256) k_eam_force<256, false, MANY><<<std::max(nblk(nsi, 256), 1), 256, 0, st>>>(A, T, phi);
  else k_eam_force<128, false, MANY><<<std::max(nblk(nsi, 128), 1), 128, 0, st>>>(A, T, phi);
}

template <class F>
float time_launch(cudaStream_t st, F &&launch) {
  cudaEvent_t a, b;
  CACB200_CUDA(cudaEventCreate(&a));
  CACB200_CUDA(cudaEventCreate(&b));
  float best = 1e30f;
  for (int rep = 0; rep < 3; rep++) {
    CACB200_CUDA(cudaEventRecord(a, st));
    launch();
    CACB200_CUDA(cudaEventRecord(b, st));
    CACB200_CUDA(cudaEventSynchronize(b));
    float ms = 0.f;
    CACB200_CUDA(cudaEventElapsedTime(&ms, a, b));
    best = std::min(best, ms);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return best;
}

bool capturing(cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  CACB200_CUDA(cudaStreamIsCapturing(st, &cs));
  return cs != cudaStreamCaptureStatusNone;
}

void pair_compute(Ctx &c, int eflag, int vflag) {
  c.check_system();
  if (!c.lists_valid) throw Error(CACB200_ESTATE, "neighbour lists not built");
  if (c.precision == CACB200_MIXED) {
    pair_compute_mixed(c, eflag, vflag);
    return;
  }
  const int nsi = c.nsite_i();
  const int T = 128;
  const int nb = std::max(nblk(nsi, T), 1);
  PairArgs A;
  A.xs = c.xss.p;
  A.nbr = c.nbr_full.p;
  A.num = c.num_full.p;
  A.num_in = c.num_in.p;
  A.prefix = prefix_rule(c);
  A.slot_atom = c.slot_atom.p;
  A.na = c.na;
  A.ne = c.ne;
  A.nsi = nsi;
  A.cap = c.cap;
  for (int d = 0; d < 3; d++) A.L[d] = c.prd[d];
  A.reps = c.rep_d.p;
  A.site_rep = c.nrep > 1 ? c.site_rep.p : nullptr;
  A.f = c.f.p;
  A.gaussf = c.gaussf.p;
  if (eflag & CACB200_ENERGY_ATOM) {
    c.eatom.reserve(std::max(c.na, 1));
    c.enode.reserve(std::max(c.ne * 8, 1));
  }
  if (vflag & CACB200_VIRIAL_ATOM) {
    c.vatom.reserve(std::max(c.na * 6, 1));
    c.vnode.reserve(std::max(c.ne * 48, 1));
  }
  A.eatom = c.eatom.p;
  A.enode = c.enode.p;
  A.vatom = c.vatom.p;
  A.vnode = c.vnode.p;
  c.partial.reserve((size_t)nb * 7);
  c.ev_out.reserve(7);
  A.partial = c.partial.p;
  A.eflag = eflag;
  A.vflag = vflag;
  double nodal_weight = (double)NU / (double)NPE;   // element_vec_cac.cpp:1732
  A.vscale_node = nodal_weight / 2.0;
  A.escale_node = nodal_weight / 2.0;
  if (c.pp.style == CACB200_PAIR_EAM && c.nodal_energy_weight >= 0.0)
    A.escale_node = c.nodal_energy_weight / 2.0;
  c.escale_node_last = A.escale_node;

  if (c.pp.style == CACB200_PAIR_LJ) {
    LjParams P{c.pp.cut * c.pp.cut, c.pp.lj1, c.pp.lj2, c.pp.lj3, c.pp.lj4, c.pp.offset};
    KernelTimer t(c, "pair_lj");
    if (c.nrep > 1) {
      if (eflag || vflag) k_lj<true, true><<<nb, T, 0, c.stream>>>(A, P);
      else k_lj<false, true><<<nb, T, 0, c.stream>>>(A, P);
    } else {
      if (eflag || vflag) k_lj<true, false><<<nb, T, 0, c.stream>>>(A, P);
      else k_lj<false, false><<<nb, T, 0, c.stream>>>(A, P);
    }
  } else if (c.pp.style == CACB200_PAIR_EAM) {
    EamTables Tb;
    Tb.rz = c.rz.p;
    Tb.frho_val = c.frho_val.p;
    Tb.frho_der = c.frho_der.p;
    Tb.rdr = c.pp.rdr;
    Tb.rdrho = c.pp.rdrho;
    Tb.rhomax = c.pp.rhomax;
    Tb.cutforcesq = c.pp.cut * c.pp.cut;
    Tb.nr = c.pp.nr;
    Tb.nrho = c.pp.nrho;
    c.rho.reserve(std::max(c.na + 8 * c.ne, 1));
    c.phi_site.reserve(std::max(nsi, 1));
    const bool many = c.nrep > 1;
    auto site_fp = [&] {
      if (c.ne)
        k_eam_site_fp<<<stride_grid((long)c.ne * NU, 256), 256, 0, c.stream>>>(
            c.xss.p, c.act_gid.p, c.dev_nact.p, c.na + NG * c.ne, c.na, c.rho.p, Tb);
    };
    auto rho = [&](int tb) {
      if (many) launch_rho<true>(tb, nsi, c.stream, A, Tb, c.rho.p, c.phi_site.p);
      else launch_rho<false>(tb, nsi, c.stream, A, Tb, c.rho.p, c.phi_site.p);
    };
    auto force = [&](int tb) {
      if (many) launch_force<true>(tb, nsi, c.stream, A, Tb, c.phi_site.p);
      else launch_force<false>(tb, nsi, c.stream, A, Tb, c.phi_site.p);
    };
    // single systems: the force-only passes over SM-local runs
    const bool smq = !many && c.work_queue;
    c.sm_counter.reserve(2 * c.num_sms);
    auto sm_grid = [&](auto kernel, int &cache) {
      if (!cache) {
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, 128, 0);
        cache = (b > 0 ? b : 1) * c.num_sms;
      }
      return cache;
    };
    static int grid_rho_sm = 0, grid_force_sm = 0;
    auto rho_s = [&] {
      CACB200_CUDA(cudaMemsetAsync(c.sm_counter.p, 0, sizeof(int) * c.num_sms, c.stream));
      k_eam_rho_sm<128><<<sm_grid(k_eam_rho_sm<128>, grid_rho_sm), 128, 0, c.stream>>>(
          A, Tb, c.rho.p, c.phi_site.p, c.sm_counter.p, c.num_sms);
    };
    auto force_s = [&] {
      CACB200_CUDA(cudaMemsetAsync(c.sm_counter.p + c.num_sms, 0, sizeof(int) * c.num_sms, c.stream));
      k_eam_force_sm<128><<<sm_grid(k_eam_force_sm<128>, grid_force_sm), 128, 0, c.stream>>>(
          A, Tb, c.phi_site.p, c.sm_counter.p + c.num_sms, c.num_sms);
    };
    if (!smq && c.tune_gen != c.gen && !eflag && !vflag && !capturing(c.stream)) {
      // another size replaces 128 only when it is at least 3 % faster
      const int cand[3] = {128, 64, 256};
      float best = 1e30f;
      for (int tb : cand) {
        float ms = time_launch(c.stream, [&] { rho(tb); });
        if (tb == 128 || ms < 0.97f * best) best = ms, c.tb_rho = tb;
      }
      rho(c.tb_rho);
      site_fp();
      best = 1e30f;
      for (int tb : cand) {
        float ms = time_launch(c.stream, [&] { force(tb); });
        if (tb == 128 || ms < 0.97f * best) best = ms, c.tb_force = tb;
      }
      c.tune_gen = c.gen;
    }
    {
      KernelTimer t(c, "eam_rho");
      if (smq) rho_s();
      else rho(c.tb_rho);
    }
    {
      KernelTimer t(c, "eam_site_fp");
      site_fp();
    }
    {
      KernelTimer t(c, "eam_force");
      if (eflag || vflag) {
        if (many) k_eam_force<128, true, true><<<nb, T, 0, c.stream>>>(A, Tb, c.phi_site.p);
        else k_eam_force<128, true, false><<<nb, T, 0, c.stream>>>(A, Tb, c.phi_site.p);
      } else if (smq) {
        force_s();
      } else {
        force(c.tb_force);
      }
    }
  } else {
    throw Error(CACB200_ESTATE, "no pair style set");
  }
  if (eflag || vflag) {
    k_reduce_partials<<<1, 256, 0, c.stream>>>(c.partial.p, nb, c.ev_out.p);
    c.have_peratom_e = (eflag & CACB200_ENERGY_ATOM) != 0;
    c.have_peratom_v = (vflag & CACB200_VIRIAL_ATOM) != 0;
    c.ev_pending = true;
    if (eflag & CACB200_ENERGY_GLOBAL) c.tally_step_e = c.step;
    if (vflag & CACB200_VIRIAL_GLOBAL) c.tally_step_v = c.step;
    if (eflag & CACB200_ENERGY_ATOM) c.tally_step_ae = c.step;
    if (vflag & CACB200_VIRIAL_ATOM) c.tally_step_av = c.step;
  }
  CACB200_CUDA(cudaGetLastError());
}

}  // namespace cacb200
