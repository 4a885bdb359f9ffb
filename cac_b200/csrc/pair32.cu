// Mixed-precision pair kernels: FP32 distances and force arithmetic on
// fixed-point positions, FP64 everywhere else.
//
// Every site of the site table gets, each step, a 32-bit fixed-point copy of
// its FP64 position relative to the box corner, q = rint((x - lo) 2^26) taken
// modulo 2^32.  A pair's separation is then
//     x_i - (x_j + s L) = (q_i - q_j - s Lq) 2^-26   (mod 2^32 quanta),
// an exact integer difference in wrap-around 32-bit arithmetic, which is the
// true difference whenever that is shorter than 2^31 quanta = 32 A (pairs are
// within the neighbour cutoff), rounded once to FP32: no FP32 sum ever
// carries a box-sized coordinate, and the quantum (1.5e-8 A) does not depend
// on the box size.  A site's record is 16 bytes, (qx, qy, qz, F'), so one
// 128-bit load brings everything a pair needs from its neighbour.
//
// What stays FP64 (as the mixed form specifies): positions and velocities and
// their integration, element interpolation, nodal assembly over Gauss points,
// and the global energy/virial reductions (per-block partials in FP64).
// Per-site sums of pair terms are FP32; EAM spline coefficients are FP32
// copies of the FP64 splines.
#include <algorithm>
#include <cmath>
#include <vector>

#include "ctx.cuh"
#include "device.cuh"

namespace cacb200 {

namespace {

inline int nblk(long n, int t) { return (int)((n + t - 1) / t); }

// Fixed-point frame of a single system; batches read each replica's from its
// descriptor.
struct FixGrid {
  double lo[3];
  double scale[3];
  float inv[3];
  int Lq[3];
  const Rep *reps;          // batches (null for one system)
  const int *site_rep;      // [nsite_i]
  const int *elem_rep;      // [ne]
  const int *act_gid;       // active lattice sites -> element * 729 + site
  const int *slot_atom;     // list slot -> atom
  int na, nsi;
};

// Fixed-point record of pair-table entry k at FP64 position (px, py, pz),
// in the frame of its replica; w (F') is written later in the step.
__device__ __forceinline__ void pack_pos(double px, double py, double pz, int k, const FixGrid &G, int4 *pos,
                                         int *bad) {
  double q[3] = {px, py, pz};
  double lo[3] = {G.lo[0], G.lo[1], G.lo[2]};
  double sc[3] = {G.scale[0], G.scale[1], G.scale[2]};
  if (G.reps) {
    int r = k < G.na ? G.site_rep[G.slot_atom[k]]
                     : (k < G.nsi ? G.site_rep[k] : G.elem_rep[G.act_gid[k - G.nsi] / NU]);
    const Rep *R = G.reps + r;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      lo[d] = R->b.lo[d];
      sc[d] = R->qscale[d];
    }
  }
  int o[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    double rel = (q[d] - lo[d]) * sc[d];
    // positions further than 2^62 quanta (~7e10 A) from the box, or not
    // finite, only come from a run that has blown up
    if (!(rel > -4.6e18 && rel < 4.6e18)) {
      atomicExch(bad, 1);
      rel = 0.0;
    }
    o[d] = (int)(unsigned)(unsigned long long)__double2ll_rn(rel);   // modulo 2^32
  }
  pos[k] = make_int4(o[0], o[1], o[2], 0);
}

// The mixed form's pair table in one pass: the slot-ordered atoms, the Gauss
// points and the interpolated active lattice sites (the positions of
// k_pair_table, integrate.cu, in the same FP64 operations) written straight
// as fixed-point records, with no FP64 copy in between.
__global__ void k_pair_table32(const double4 *xs, const int *slot_atom, const double *nodex, int na, int ne,
                               const int *act_gid, const int *nact_dev, FixGrid G, int4 *pos, int *bad) {
  const int ngp = NG * ne;
  const int n = na + ngp + *nact_dev;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    if (t < na) {
      const double4 p = xs[slot_atom[t]];
      pack_pos(p.x, p.y, p.z, t, G, pos, bad);
      continue;
    }
    const int s = t - na;
    if (s < ngp) {
      const int e = s / NG, g = s % NG;
      const double *nx = nodex + (size_t)e * 24 + 3 * gauss_node(g);
      pack_pos(nx[0], nx[1], nx[2], t, G, pos, bad);
      continue;
    }
    const int gid = act_gid[s - ngp];
    const int e = gid / NU, u = gid % NU;
    const double *nx = nodex + (size_t)e * 24;
    double x = 0.0, y = 0.0, z = 0.0;
#pragma unroll
    for (int m = 0; m < NPE; m++) {
      const double N = shape_val(u, m);
      x += N * nx[3 * m];
      y += N * nx[3 * m + 1];
      z += N * nx[3 * m + 2];
    }
    pack_pos(x, y, z, t, G, pos, bad);
  }
}

struct Args32 {
  const int4 *pos;
  const int *nbr;          // lists and counts indexed by list slot
  const int *num;
  const int *num_in;                // inner prefix length of each list ...
  PrefixRule prefix;                // ... and the rule for walking the rest
  const int *slot_atom;    // list slot -> atom (slots past the atoms are Gauss points)
  int na, ne, nsi;
  int cap;                 // list rows: the rest of a list fills its last rows
  FixGrid G;
  double *f, *gaussf;
  double *eatom, *vatom, *enode, *vnode;
  double *partial;
  int eflag, vflag;
  double escale_node, vscale_node;
};

__device__ __forceinline__ float fix_delta(int qi, int qj, int s, int Lq, float inv) {
  const unsigned sl = (unsigned)s * (unsigned)Lq;   // s in {-1, 0, 1}, modulo 2^32
  unsigned d = (unsigned)qi - (unsigned)qj - sl;
  return (float)(int)d * inv;
}

// fixed-point frame (box lengths and quanta) of i-site i's replica
struct SiteFix {
  int Lq[3];
  float inv[3];
};
__device__ __forceinline__ SiteFix site_fix(const Args32 &A, int i) {
  SiteFix F;
  if (A.G.reps) {
    const Rep *R = A.G.reps + A.G.site_rep[i];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      F.Lq[d] = R->Lq[d];
      F.inv[d] = R->qinv[d];
    }
  } else {
#pragma unroll
    for (int d = 0; d < 3; d++) {
      F.Lq[d] = A.G.Lq[d];
      F.inv[d] = A.G.inv[d];
    }
  }
  return F;
}

__device__ __forceinline__ int site_of_slot(const Args32 &A, int t) { return t < A.na ? A.slot_atom[t] : t; }

// separation of site i (record oi) from neighbour entry v; wj = F'(j)
__device__ __forceinline__ void sep32(const Args32 &A, const SiteFix &F, const int4 &oi, int v, float &dx,
                                      float &dy, float &dz, float &wj) {
  int j = v >> IMG_BITS, code = v & ((1 << IMG_BITS) - 1);
  int4 oj = __ldg(A.pos + j);
  int s[3] = {0, 0, 0};
  if (code != IMG_ZERO) img_decode(code, s[0], s[1], s[2]);
  dx = fix_delta(oi.x, oj.x, s[0], F.Lq[0], F.inv[0]);
  dy = fix_delta(oi.y, oj.y, s[1], F.Lq[1], F.inv[1]);
  dz = fix_delta(oi.z, oj.z, s[2], F.Lq[2], F.inv[2]);
  wj = __int_as_float(oj.w);
}

template <class F>
__device__ __forceinline__ void walk32(const Args32 &A, const SiteFix &fx, const int4 &oi, const int *nb, int n,
                                       F &&f) {
  int k = 0;
  for (; k + 4 <= n; k += 4) {
    int v0 = __ldcs(nb + (size_t)k * A.nsi), v1 = __ldcs(nb + (size_t)(k + 1) * A.nsi);
    int v2 = __ldcs(nb + (size_t)(k + 2) * A.nsi), v3 = __ldcs(nb + (size_t)(k + 3) * A.nsi);
    float d[4][4];
    sep32(A, fx, oi, v0, d[0][0], d[0][1], d[0][2], d[0][3]);
    sep32(A, fx, oi, v1, d[1][0], d[1][1], d[1][2], d[1][3]);
    sep32(A, fx, oi, v2, d[2][0], d[2][1], d[2][2], d[2][3]);
    sep32(A, fx, oi, v3, d[3][0], d[3][1], d[3][2], d[3][3]);
#pragma unroll
    for (int u = 0; u < 4; u++) f(d[u][0], d[u][1], d[u][2], d[u][3]);
  }
  for (; k < n; k++) {
    float dx, dy, dz, wj;
    sep32(A, fx, oi, __ldcs(nb + (size_t)k * A.nsi), dx, dy, dz, wj);
    f(dx, dy, dz, wj);
  }
}

// A site's list: the inner prefix on its own, then the rest unless the
// prefix still holds every pair of the site inside the cutoff (walk_rest,
// device.cuh; an entry's arithmetic depends on its place in a walk, so the
// prefix is always walked alone).
template <class F>
__device__ __forceinline__ void for_each32(const Args32 &A, int t, int i, const int4 &oi, F &&f) {
  const SiteFix fx = site_fix(A, i);
  const int n_in = A.num_in[t], n = A.num[t];
  const int *nb = A.nbr + t;
  const bool rest = n > n_in && walk_rest(A.prefix, i, A.G.reps ? A.G.site_rep[i] : 0);
#pragma unroll 1
  for (int seg = 0; seg < (rest ? 2 : 1); seg++)
    walk32(A, fx, oi, seg ? nb + (size_t)(A.cap - (n - n_in)) * A.nsi : nb, seg ? n - n_in : n_in, f);
}

__device__ __forceinline__ void finish32(const Args32 &A, int i, bool valid, const float fi[3], bool ev,
                                         float esum, const float vsum[6], double eextra_site,
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
    if (ev) {
      double es = atom ? 0.5 : A.escale_node, vs = atom ? 0.5 : A.vscale_node;
      if (A.eflag & CACB200_ENERGY_GLOBAL) red[0] = es * (double)esum + eextra_global;
      if (A.vflag & CACB200_VIRIAL_GLOBAL)
#pragma unroll
        for (int k = 0; k < 6; k++) red[1 + k] = vs * (double)vsum[k];
      if (A.eflag & CACB200_ENERGY_ATOM) {
        double v = 0.5 * (double)esum + eextra_site;
        if (atom) A.eatom[i] = v;
        else A.enode[(size_t)e * 8 + node] = v;
      }
      if (A.vflag & CACB200_VIRIAL_ATOM) {
        double *vo = atom ? A.vatom + 6 * (size_t)i : A.vnode + 48 * (size_t)e + 6 * node;
#pragma unroll
        for (int k = 0; k < 6; k++) vo[k] = 0.5 * (double)vsum[k];
      }
    }
  }
  if (ev) block_reduce_store<7>(red, A.partial);
}

__device__ __forceinline__ void site_frame(const Args32 &A, int i, int4 &oi) { oi = __ldg(A.pos + i); }

// ---------------------------------------------------------------------- LJ

struct Lj32 {
  float cutsq, lj1, lj2, lj3, lj4, offset;
};

template <bool EV>
__global__ void __launch_bounds__(128, EV ? 4 : 8) k_lj32(Args32 A, Lj32 P) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;   // list slot
  const bool valid = t < A.nsi;
  const int i = valid ? site_of_slot(A, t) : 0;           // site-table index
  float fi[3] = {0, 0, 0}, esum = 0.f, vsum[6] = {0, 0, 0, 0, 0, 0};
  if (valid) {
    int4 oi;
    site_frame(A, t, oi);
    for_each32(A, t, i, oi, [&](float dx, float dy, float dz, float) {
      float rsq = dx * dx + dy * dy + dz * dz;
      if (rsq < P.cutsq) {
        float r2inv = 1.0f / rsq;
        float r6inv = r2inv * r2inv * r2inv;
        float fpair = r6inv * (P.lj1 * r6inv - P.lj2) * r2inv;
        fi[0] += dx * fpair;
        fi[1] += dy * fpair;
        fi[2] += dz * fpair;
        if (EV) {
          esum += r6inv * (P.lj3 * r6inv - P.lj4) - P.offset;
          vsum[0] += dx * dx * fpair;
          vsum[1] += dy * dy * fpair;
          vsum[2] += dz * dz * fpair;
          vsum[3] += dx * dy * fpair;
          vsum[4] += dx * dz * fpair;
          vsum[5] += dy * dz * fpair;
        }
      }
    });
  }
  finish32(A, i, valid, fi, EV, esum, vsum, 0.0, 0.0);
}

// --------------------------------------------------------------------- EAM

// rz: per r-knot m the rhor value coefficients at [2m] and the z2r ones at
// [2m+1], one 32-byte record; derivatives as in the FP64 kernels.
struct Eam32 {
  const float4 *rz, *frho_val, *frho_der;
  float rdr, rdrho, rhomax, cutforcesq;
  int nr, nrho;
};

__device__ __forceinline__ float fp32_of(const Eam32 &T, float rho, float *phi) {
  float p = rho * T.rdrho + 1.0f;
  int m = (int)p;
  m = max(1, min(m, T.nrho - 1));
  p -= (float)m;
  p = fminf(p, 1.0f);
  float4 d = T.frho_der[m];
  float fp = (d.x * p + d.y) * p + d.z;
  if (phi) {
    float4 v = T.frho_val[m];
    float e = ((v.x * p + v.y) * p + v.z) * p + v.w;
    if (rho > T.rhomax) e += fp * (rho - T.rhomax);
    *phi = e;
  }
  return fp;
}

// A pair's density term (one functor for every walk, so the arithmetic is
// the same code wherever the neighbour comes from).
struct RhoPair {
  const Eam32 &T;
  float &rho;
  __device__ __forceinline__ void operator()(float dx, float dy, float dz, float) const {
    float rsq = dx * dx + dy * dy + dz * dz;
    if (rsq < T.cutforcesq) {
      float p = sqrtf(rsq) * T.rdr + 1.0f;
      int m = (int)p;
      m = max(1, min(m, T.nr - 1));
      p -= (float)m;
      p = fminf(p, 1.0f);
      float4 c = __ldg(T.rz + 2 * m);
      rho += ((c.x * p + c.y) * p + c.z) * p + c.w;
    }
  }
};

// One list slot of the density pass: rho at the site, then F' into its
// record (and F into phi_site for energies).
__device__ __forceinline__ void rho32_slot(const Args32 &A, const Eam32 &T, int t, double *rho_out,
                                           double *phi_site, int4 *pos_w) {
  const int i = site_of_slot(A, t);                       // site-table index
  int4 oi;
  site_frame(A, t, oi);
  float rho = 0.f;
  for_each32(A, t, i, oi, RhoPair{T, rho});
  int slot = i;
  if (i >= A.na) {
    int e = (i - A.na) / NG, g = (i - A.na) % NG;
    slot = A.na + 8 * e + gauss_node(g);
  }
  rho_out[slot] = rho;
  float phi = 0.f;
  float fp = fp32_of(T, rho, A.eflag ? &phi : nullptr);
  pos_w[t].w = __float_as_int(fp);
  if (A.eflag) phi_site[i] = phi;
}

template <int TB>
__global__ void __launch_bounds__(TB, 1024 / TB) k_eam_rho32(Args32 A, Eam32 T, double *rho_out, double *phi_site,
                                                      int4 *pos_w) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;   // list slot
  if (t >= A.nsi) return;
  rho32_slot(A, T, t, rho_out, phi_site, pos_w);
}

// Persistent work-queue launches for batches: blocks stay resident and take
// work items one after another from a counter (cleared before the launch);
// an item is a run of consecutive list slots of one replica (x: first slot,
// y: count), the largest replicas' items first.  Each slot is computed by
// the same function as in the grid launch, so results do not change.
__device__ __forceinline__ int next_item(int *counter) {
  __shared__ int it;
  __syncthreads();
  if (threadIdx.x == 0) it = atomicAdd(counter, 1);
  __syncthreads();
  return it;
}

template <int TB>
__global__ void __launch_bounds__(TB, 1024 / TB) k_eam_rho32_queue(Args32 A, Eam32 T, double *rho_out,
                                                            double *phi_site, int4 *pos_w, const int2 *items,
                                                            int nitems, int *counter) {
  for (;;) {
    const int k = next_item(counter);
    if (k >= nitems) return;
    const int2 w = items[k];
    for (int t = w.x + threadIdx.x; t < w.x + w.y; t += TB) rho32_slot(A, T, t, rho_out, phi_site, pos_w);
  }
}

__global__ void k_eam_site_fp32(int4 *pos, const int *act_gid, const int *nact_dev, int base, int na,
                                const double *rho, Eam32 T) {
  const int nact = *nact_dev;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nact; k += gridDim.x * blockDim.x) {
    int gid = act_gid[k];
    int e = gid / NU, u = gid % NU;
    const double *rn = rho + na + 8 * (size_t)e;
    double r = 0.0;
#pragma unroll
    for (int n = 0; n < NPE; n++) r += shape_val(u, n) * rn[n];
    pos[base + k].w = __float_as_int(fp32_of(T, (float)r, nullptr));
  }
}

// A pair's force term (and energy and virial with EV).
template <bool EV>
struct ForcePair {
  const Eam32 &T;
  float fpi;
  float *fi;
  float &esum;
  float *vsum;
  __device__ __forceinline__ void operator()(float dx, float dy, float dz, float fpj) const {
    float rsq = dx * dx + dy * dy + dz * dz;
    if (rsq < T.cutforcesq) {
      float recip = rsqrtf(rsq);
      float r = rsq * recip;
      float p = r * T.rdr + 1.0f;
      int m = (int)p;
      m = max(1, min(m, T.nr - 1));
      p -= (float)m;
      p = fminf(p, 1.0f);
      float4 rv, zv;
      ldg256(T.rz + 2 * m, rv, zv);
      float rhop = ((3.0f * rv.x * p + 2.0f * rv.y) * p + rv.z) * T.rdr;
      float z2p = ((3.0f * zv.x * p + 2.0f * zv.y) * p + zv.z) * T.rdr;
      float z2 = ((zv.x * p + zv.y) * p + zv.z) * p + zv.w;
      float phi = z2 * recip;
      float phip = z2p * recip - phi * recip;
      float psip = (fpi + fpj) * rhop + phip;
      float fpair = -psip * recip;
      fi[0] += dx * fpair;
      fi[1] += dy * fpair;
      fi[2] += dz * fpair;
      if (EV) {
        esum += phi;
        vsum[0] += dx * dx * fpair;
        vsum[1] += dy * dy * fpair;
        vsum[2] += dz * dz * fpair;
        vsum[3] += dx * dy * fpair;
        vsum[4] += dx * dz * fpair;
        vsum[5] += dy * dz * fpair;
      }
    }
  }
};

// One list slot of the force pass: the pair sums of a valid slot (force;
// energy and virial with EV) and its embedding energy.
template <bool EV>
__device__ __forceinline__ void force32_slot(const Args32 &A, const Eam32 &T, int t, int i,
                                             const double *phi_site, float fi[3], float &esum, float vsum[6],
                                             double &eemb_site, double &eemb_global) {
  int4 oi;
  site_frame(A, t, oi);
  const float fpi = __int_as_float(oi.w);
  for_each32(A, t, i, oi, ForcePair<EV>{T, fpi, fi, esum, vsum});
  if (EV && A.eflag) {
    double phi = phi_site[i];
    eemb_site = phi;
    eemb_global = (i < A.na) ? phi : phi * A.escale_node * 2.0;
  }
}

template <int TB, bool EV>
__global__ void __launch_bounds__(TB, (EV ? 512 : 1024) / TB) k_eam_force32(Args32 A, Eam32 T,
                                                                          const double *phi_site) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;   // list slot
  const bool valid = t < A.nsi;
  const int i = valid ? site_of_slot(A, t) : 0;           // site-table index
  float fi[3] = {0, 0, 0}, esum = 0.f, vsum[6] = {0, 0, 0, 0, 0, 0};
  double eemb_site = 0.0, eemb_global = 0.0;
  if (valid) force32_slot<EV>(A, T, t, i, phi_site, fi, esum, vsum, eemb_site, eemb_global);
  finish32(A, i, valid, fi, EV, esum, vsum, eemb_site, eemb_global);
}

template <int TB>
__global__ void __launch_bounds__(TB, 1024 / TB) k_eam_force32_queue(Args32 A, Eam32 T, const double *phi_site,
                                                              const int2 *items, int nitems, int *counter) {
  for (;;) {
    const int k = next_item(counter);
    if (k >= nitems) return;
    const int2 w = items[k];
    for (int t = w.x + threadIdx.x; t < w.x + w.y; t += TB) {
      const int i = site_of_slot(A, t);
      float fi[3] = {0, 0, 0}, esum = 0.f, vsum[6] = {0, 0, 0, 0, 0, 0};
      double eemb_site = 0.0, eemb_global = 0.0;
      force32_slot<false>(A, T, t, i, phi_site, fi, esum, vsum, eemb_site, eemb_global);
      finish32(A, i, true, fi, false, esum, vsum, eemb_site, eemb_global);
    }
  }
}

__global__ void k_reduce_partials32(const double *partial, int nblocks, double *out) {
  int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (k >= 7) return;
  double s = 0.0;
  for (int b = lane; b < nblocks; b += 32) s += partial[b * 7 + k];
  s = warp_sum(s);
  if (lane == 0) out[k] = s;
}

FixGrid make_fix_grid(const Ctx &c) {
  FixGrid G;
  const Rep &r0 = c.rep_h[0];
  for (int d = 0; d < 3; d++) {
    G.lo[d] = r0.b.lo[d];
    G.scale[d] = r0.qscale[d];
    G.inv[d] = r0.qinv[d];
    G.Lq[d] = r0.Lq[d];
  }
  G.reps = c.nrep > 1 ? c.rep_d.p : nullptr;
  G.site_rep = c.site_rep.p;
  G.elem_rep = c.elem_rep.p;
  G.act_gid = c.act_gid.p;
  G.slot_atom = c.slot_atom.p;
  G.na = c.na;
  G.nsi = c.nsite_i();
  return G;
}

}  // namespace

void pair_table_mixed(Ctx &c) {
  const long ns = (long)c.nsite_i() + (long)c.ne * NU;   // capacity: every lattice site active
  c.pos32.reserve(std::max(ns, 1L));
  c.overflow.reserve(16);
  FixGrid G = make_fix_grid(c);
  // 64 blocks per SM: the item loop's loads are in flight across more
  // threads than stride_grid's 16 blocks give (0.193 -> 0.181 ms on config 3)
  k_pair_table32<<<std::min(nblk(ns, 256), 148 * 64), 256, 0, c.stream>>>(c.xs.p, c.slot_atom.p, c.nodex.p, c.na, c.ne,
                                                             c.act_gid.p, c.dev_nact.p, G, c.pos32.p,
                                                             c.overflow.p + 6);
}

void mixed_tables(Ctx &c) {
  auto conv = [&](DBuf<double4> &src, DBuf<float4> &dst, int n) {
    std::vector<double4> h(n + 1);
    stream_copy(c, h.data(), src.p, sizeof(double4) * (n + 1), cudaMemcpyDeviceToHost);
    std::vector<float4> g(n + 1);
    for (int m = 0; m <= n; m++) g[m] = make_float4((float)h[m].x, (float)h[m].y, (float)h[m].z, (float)h[m].w);
    dst.reserve(n + 1);
    stream_copy(c, dst.p, g.data(), sizeof(float4) * (n + 1), cudaMemcpyHostToDevice);
  };
  conv(c.rz, c.rz32, 2 * c.pp.nr + 1);
  conv(c.frho_val, c.frho_val32, c.pp.nrho);
  conv(c.frho_der, c.frho_der32, c.pp.nrho);
}

namespace {

// size class of a replica by its i-sites
int size_class(long sites) { return sites < 8192 ? 0 : sites < 32768 ? 1 : 2; }

// Work items of a batch: replicas by i-sites, largest first; each replica's
// atom slots, then its Gauss-point slots, in runs of its class's tile.
// only_class >= 0 keeps the items of that class alone (tuning).
std::vector<int2> make_items(const Ctx &c, const int tile[3], int only_class) {
  std::vector<int> order(c.nrep);
  for (int r = 0; r < c.nrep; r++) order[r] = r;
  auto sites = [&](int r) { return (long)c.rep_na[r] + 8L * c.rep_ne[r]; };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return sites(a) > sites(b); });
  std::vector<int2> items;
  for (int r : order) {
    const int cl = size_class(sites(r));
    if (only_class >= 0 && cl != only_class) continue;
    const int T = tile[cl];
    const int a0 = c.rep_aoff[r], na = c.rep_na[r];
    for (int o = 0; o < na; o += T) items.push_back(make_int2(a0 + o, std::min(T, na - o)));
    const int g0 = c.na + 8 * c.rep_eoff[r], ng = 8 * c.rep_ne[r];
    for (int o = 0; o < ng; o += T) items.push_back(make_int2(g0 + o, std::min(T, ng - o)));
  }
  return items;
}

int queue_grid(const Ctx &c) {
  static const int per_sm = [] {
    int b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_eam_force32_queue<128>, 128, 0);
    return b > 0 ? b : 1;
  }();
  return per_sm * c.num_sms;
}

void upload_items(Ctx &c, const std::vector<int2> &items) {
  c.work_items.reserve(std::max<size_t>(items.size(), 1));
  if (!items.empty())
    stream_copy(c, c.work_items.p, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice);
  c.nwork_items = (int)items.size();
}

}  // namespace

void pair_compute_mixed(Ctx &c, int eflag, int vflag) {
  const int nsi = c.nsite_i();
  const long ns = (long)nsi + (long)c.ne * NU;   // capacity: every lattice site active
  const int T = 128;
  const int nb = std::max(nblk(nsi, T), 1);
  FixGrid G = make_fix_grid(c);
  (void)ns;   // the fixed-point records were written by pair_table_mixed
  Args32 A;
  A.pos = c.pos32.p;
  A.nbr = c.nbr_full.p;
  A.num = c.num_full.p;
  A.num_in = c.num_in.p;
  A.prefix = prefix_rule(c);
  A.slot_atom = c.slot_atom.p;
  A.na = c.na;
  A.ne = c.ne;
  A.nsi = nsi;
  A.cap = c.cap;
  A.G = G;
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
  double nodal_weight = (double)NU / (double)NPE;
  A.vscale_node = nodal_weight / 2.0;
  A.escale_node = nodal_weight / 2.0;
  if (c.pp.style == CACB200_PAIR_EAM && c.nodal_energy_weight >= 0.0) A.escale_node = c.nodal_energy_weight / 2.0;
  c.escale_node_last = A.escale_node;
  bool ev = eflag || vflag;
  if (c.pp.style == CACB200_PAIR_LJ) {
    Lj32 P{(float)(c.pp.cut * c.pp.cut), (float)c.pp.lj1, (float)c.pp.lj2, (float)c.pp.lj3, (float)c.pp.lj4,
           (float)c.pp.offset};
    KernelTimer t(c, "pair_lj32");
    if (ev) k_lj32<true><<<nb, T, 0, c.stream>>>(A, P);
    else k_lj32<false><<<nb, T, 0, c.stream>>>(A, P);
  } else {
    if (!c.have_mixed_tables) {
      mixed_tables(c);
      c.have_mixed_tables = true;
    }
    Eam32 Tb;
    Tb.rz = c.rz32.p;
    Tb.frho_val = c.frho_val32.p;
    Tb.frho_der = c.frho_der32.p;
    Tb.rdr = (float)c.pp.rdr;
    Tb.rdrho = (float)c.pp.rdrho;
    Tb.rhomax = (float)c.pp.rhomax;
    Tb.cutforcesq = (float)(c.pp.cut * c.pp.cut);
    Tb.nr = c.pp.nr;
    Tb.nrho = c.pp.nrho;
    c.rho.reserve(std::max(c.na + 8 * c.ne, 1));
    c.phi_site.reserve(std::max(nsi, 1));
    auto rho = [&](int tb) {
      if (tb == 64) k_eam_rho32<64><<<std::max(nblk(nsi, 64), 1), 64, 0, c.stream>>>(A, Tb, c.rho.p, c.phi_site.p, c.pos32.p);
      else if (tb == 256) k_eam_rho32<256><<<std::max(nblk(nsi, 256), 1), 256, 0, c.stream>>>(A, Tb, c.rho.p, c.phi_site.p, c.pos32.p);
      else k_eam_rho32<128><<<nb, 128, 0, c.stream>>>(A, Tb, c.rho.p, c.phi_site.p, c.pos32.p);
    };
    auto site_fp = [&] {
      if (c.ne)
        k_eam_site_fp32<<<stride_grid((long)c.ne * NU, 256), 256, 0, c.stream>>>(
            c.pos32.p, c.act_gid.p, c.dev_nact.p, c.na + NG * c.ne, c.na, c.rho.p, Tb);
    };
    auto force = [&](int tb) {
      if (tb == 64) k_eam_force32<64, false><<<std::max(nblk(nsi, 64), 1), 64, 0, c.stream>>>(A, Tb, c.phi_site.p);
      else if (tb == 256) k_eam_force32<256, false><<<std::max(nblk(nsi, 256), 1), 256, 0, c.stream>>>(A, Tb, c.phi_site.p);
      else k_eam_force32<128, false><<<nb, 128, 0, c.stream>>>(A, Tb, c.phi_site.p);
    };
    // batches: the persistent work-queue launches, their tiles tuned per
    // replica size class when the plan changes (idempotent trial launches)
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CACB200_CUDA(cudaStreamIsCapturing(c.stream, &cs));
    bool queue = c.nrep > 1 && c.work_queue;
    c.work_counter.reserve(2);
    auto rho_q = [&] {
      CACB200_CUDA(cudaMemsetAsync(c.work_counter.p, 0, sizeof(int), c.stream));
      k_eam_rho32_queue<128><<<queue_grid(c), 128, 0, c.stream>>>(A, Tb, c.rho.p, c.phi_site.p, c.pos32.p,
                                                                 c.work_items.p, c.nwork_items, c.work_counter.p);
    };
    auto force_q = [&] {
      CACB200_CUDA(cudaMemsetAsync(c.work_counter.p + 1, 0, sizeof(int), c.stream));
      k_eam_force32_queue<128><<<queue_grid(c), 128, 0, c.stream>>>(A, Tb, c.phi_site.p, c.work_items.p,
                                                                   c.nwork_items, c.work_counter.p + 1);
    };
    if (queue && c.work_gen != c.gen && cs == cudaStreamCaptureStatusNone) {
      const int cand[3] = {512, 128, 2048};   // another tile replaces 512 only when >= 3 % faster
      int tile[3] = {512, 512, 512};
      {
        // phase: densities and F' first, so the trial force passes read the step's F'
        upload_items(c, make_items(c, tile, -1));
        rho_q();
        site_fp();
        cudaEvent_t e0, e1;
        CACB200_CUDA(cudaEventCreate(&e0));
        CACB200_CUDA(cudaEventCreate(&e1));
        for (int cl = 0; cl < 3; cl++) {
          float best = 1e30f;
          for (int T : cand) {
            int trial[3] = {T, T, T};
            upload_items(c, make_items(c, trial, cl));
            if (c.nwork_items == 0) break;
            float ms = 1e30f;
            for (int rep = 0; rep < 3; rep++) {
              CACB200_CUDA(cudaEventRecord(e0, c.stream));
              force_q();
              CACB200_CUDA(cudaEventRecord(e1, c.stream));
              CACB200_CUDA(cudaEventSynchronize(e1));
              float m = 0.f;
              CACB200_CUDA(cudaEventElapsedTime(&m, e0, e1));
              ms = std::min(ms, m);
            }
            if (T == 512 || ms < 0.97f * best) best = ms, tile[cl] = T;
          }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
      }
      for (int cl = 0; cl < 3; cl++) c.work_tile[cl] = tile[cl];
      upload_items(c, make_items(c, tile, -1));
      c.work_gen = c.gen;
    }
    // items are made outside stream capture; until then the grid launches
    if (queue && c.work_gen != c.gen) queue = false;
    // block sizes of the force-only passes chosen by timing on first use (as
    // in the FP64 form; results do not depend on them)
    if (!queue && c.tune_gen32 != c.gen && !ev && cs == cudaStreamCaptureStatusNone) {
      const int cand[3] = {128, 64, 256};   // another size replaces 128 only when >= 3 % faster
      cudaEvent_t e0, e1;
      CACB200_CUDA(cudaEventCreate(&e0));
      CACB200_CUDA(cudaEventCreate(&e1));
      auto timed = [&](auto &&launch) {
        float best = 1e30f;
        for (int rep = 0; rep < 3; rep++) {
          CACB200_CUDA(cudaEventRecord(e0, c.stream));
          launch();
          CACB200_CUDA(cudaEventRecord(e1, c.stream));
          CACB200_CUDA(cudaEventSynchronize(e1));
          float ms = 0.f;
          CACB200_CUDA(cudaEventElapsedTime(&ms, e0, e1));
          best = std::min(best, ms);
        }
        return best;
      };
      float best = 1e30f;
      for (int tb : cand) {
        float ms = timed([&] { rho(tb); });
        if (tb == 128 || ms < 0.97f * best) best = ms, c.tb_rho32 = tb;
      }
      rho(c.tb_rho32);
      site_fp();
      best = 1e30f;
      for (int tb : cand) {
        float ms = timed([&] { force(tb); });
        if (tb == 128 || ms < 0.97f * best) best = ms, c.tb_force32 = tb;
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      c.tune_gen32 = c.gen;
    }
    {
      KernelTimer t(c, "eam_rho32");
      if (queue) rho_q();
      else rho(c.tb_rho32);
    }
    if (c.ne) {
      KernelTimer t(c, "eam_site_fp32");
      site_fp();
    }
    {
      KernelTimer t(c, "eam_force32");
      if (ev) k_eam_force32<128, true><<<nb, T, 0, c.stream>>>(A, Tb, c.phi_site.p);
      else if (queue) force_q();
      else force(c.tb_force32);
    }
  }
  if (ev) {
    k_reduce_partials32<<<1, 256, 0, c.stream>>>(c.partial.p, nb, c.ev_out.p);
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
