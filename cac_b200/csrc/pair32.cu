// Mixed-precision pair kernels: FP32 distances and force arithmetic on
// positions stored relative to their cell, FP64 everywhere else.
//
// Every site of the site table gets, each step, an anchor cell of an 8 A grid
// fixed to the box (a = floor((x - lo) / 8), from its FP64 position, which may
// lie outside the box for element sites) and its FP32 offset inside that cell
// (x - lo - 8 a, at most 8 A, so one FP32 ulp is 4.8e-7 A).  A pair's
// separation is then
//     x_i - (x_j + s L) = (off_i - off_j) + (a_i - a_j - s n) * 8 - s r
// per dimension, with n = ceil(L / 8) cells and r = L - 8 n: the cell term is
// a small integer times 8 (exact in FP32), r is rounded once, and no FP32 sum
// ever carries a box-sized coordinate.  Anchors are packed into one 32-bit
// word with per-dimension bit fields sized from the box.
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

constexpr double CELL = 8.0;   // anchor cell edge (A); exact in FP32
constexpr int BIAS = 8;        // anchors may lie up to 8 cells outside the box

struct AnchorGrid {
  double lo[3];
  int n[3];        // cells per box length
  float r[3];      // L - 8 n (rounded once)
  int shift[3];    // bit offsets of the fields
  int bits[3];
};

__device__ __forceinline__ void unpack_anchor(const AnchorGrid &G, unsigned w, int a[3]) {
#pragma unroll
  for (int d = 0; d < 3; d++) a[d] = (int)((w >> G.shift[d]) & ((1u << G.bits[d]) - 1u)) - BIAS;
}

// FP32 copy of every site's position relative to its anchor cell; w keeps F'
// for EAM (written later in the step).
__global__ void k_pack32(const double4 *xs, int n, AnchorGrid G, float4 *pos, unsigned *anc, int *bad) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double4 p = xs[k];
  double q[3] = {p.x, p.y, p.z};
  unsigned w = 0;
  float o[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    double rel = q[d] - G.lo[d];
    int a = (int)floor(rel / CELL);
    int f = a + BIAS;
    if (f < 0 || f >= (1 << G.bits[d])) {
      atomicExch(bad, 1);
      f = 0;
      a = -BIAS;
    }
    o[d] = (float)(rel - CELL * a);
    w |= (unsigned)f << G.shift[d];
  }
  float4 v = pos[k];
  pos[k] = make_float4(o[0], o[1], o[2], v.w);
  anc[k] = w;
}

struct Args32 {
  const float4 *pos;
  const unsigned *anc;
  const int *nbr;
  const int *num;
  int na, ne, nsi;
  AnchorGrid G;
  double *f, *gaussf;
  double *eatom, *vatom, *enode, *vnode;
  double *partial;
  int eflag, vflag;
  double escale_node, vscale_node;
};

// separation of site i (offset oi, anchor ai) from neighbour entry v
__device__ __forceinline__ void sep32(const Args32 &A, const float4 &oi, const int ai[3], int v,
                                      float &dx, float &dy, float &dz, float &wj) {
  int j = v >> IMG_BITS, code = v & ((1 << IMG_BITS) - 1);
  float4 oj = A.pos[j];
  int aj[3];
  unpack_anchor(A.G, A.anc[j], aj);
  int s[3] = {0, 0, 0};
  if (code != IMG_ZERO) img_decode(code, s[0], s[1], s[2]);
  dx = (oi.x - oj.x) + (float)(ai[0] - aj[0] - s[0] * A.G.n[0]) * (float)CELL - (float)s[0] * A.G.r[0];
  dy = (oi.y - oj.y) + (float)(ai[1] - aj[1] - s[1] * A.G.n[1]) * (float)CELL - (float)s[1] * A.G.r[1];
  dz = (oi.z - oj.z) + (float)(ai[2] - aj[2] - s[2] * A.G.n[2]) * (float)CELL - (float)s[2] * A.G.r[2];
  wj = oj.w;
}

template <class F>
__device__ __forceinline__ void for_each32(const Args32 &A, int i, const float4 &oi, const int ai[3], F &&f) {
  int n = A.num[i];
  const int *nb = A.nbr + i;
  int k = 0;
  for (; k + 4 <= n; k += 4) {
    int v0 = nb[(size_t)k * A.nsi], v1 = nb[(size_t)(k + 1) * A.nsi];
    int v2 = nb[(size_t)(k + 2) * A.nsi], v3 = nb[(size_t)(k + 3) * A.nsi];
    float d[4][4];
    sep32(A, oi, ai, v0, d[0][0], d[0][1], d[0][2], d[0][3]);
    sep32(A, oi, ai, v1, d[1][0], d[1][1], d[1][2], d[1][3]);
    sep32(A, oi, ai, v2, d[2][0], d[2][1], d[2][2], d[2][3]);
    sep32(A, oi, ai, v3, d[3][0], d[3][1], d[3][2], d[3][3]);
#pragma unroll
    for (int u = 0; u < 4; u++) f(d[u][0], d[u][1], d[u][2], d[u][3]);
  }
  for (; k < n; k++) {
    float dx, dy, dz, wj;
    sep32(A, oi, ai, nb[(size_t)k * A.nsi], dx, dy, dz, wj);
    f(dx, dy, dz, wj);
  }
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

__device__ __forceinline__ void site_frame(const Args32 &A, int i, float4 &oi, int ai[3]) {
  oi = A.pos[i];
  unpack_anchor(A.G, A.anc[i], ai);
}

// ---------------------------------------------------------------------- LJ

struct Lj32 {
  float cutsq, lj1, lj2, lj3, lj4, offset;
};

template <bool EV>
__global__ void __launch_bounds__(128, EV ? 4 : 8) k_lj32(Args32 A, Lj32 P) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool valid = i < A.nsi;
  float fi[3] = {0, 0, 0}, esum = 0.f, vsum[6] = {0, 0, 0, 0, 0, 0};
  if (valid) {
    float4 oi;
    int ai[3];
    site_frame(A, i, oi, ai);
    for_each32(A, i, oi, ai, [&](float dx, float dy, float dz, float) {
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

struct Eam32 {
  const float4 *rhor_val, *rhor_der, *z2r_val, *z2r_der, *frho_val, *frho_der;
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

__global__ void __launch_bounds__(128, 8) k_eam_rho32(Args32 A, Eam32 T, double *rho_out, double *phi_site,
                                                      float4 *pos_w) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.nsi) return;
  float4 oi;
  int ai[3];
  site_frame(A, i, oi, ai);
  float rho = 0.f;
  for_each32(A, i, oi, ai, [&](float dx, float dy, float dz, float) {
    float rsq = dx * dx + dy * dy + dz * dz;
    if (rsq < T.cutforcesq) {
      float p = sqrtf(rsq) * T.rdr + 1.0f;
      int m = (int)p;
      m = max(1, min(m, T.nr - 1));
      p -= (float)m;
      p = fminf(p, 1.0f);
      float4 c = T.rhor_val[m];
      rho += ((c.x * p + c.y) * p + c.z) * p + c.w;
    }
  });
  int slot = i;
  if (i >= A.na) {
    int e = (i - A.na) / NG, g = (i - A.na) % NG;
    slot = A.na + 8 * e + gauss_node(g);
  }
  rho_out[slot] = rho;
  float phi = 0.f;
  float fp = fp32_of(T, rho, A.eflag ? &phi : nullptr);
  pos_w[i].w = fp;
  if (A.eflag) phi_site[i] = phi;
}

__global__ void k_eam_site_fp32(float4 *pos, const int *act_gid, int nact, int base, int na,
                                const double *rho, Eam32 T) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nact) return;
  int gid = act_gid[k];
  int e = gid / NU, u = gid % NU;
  const double *rn = rho + na + 8 * (size_t)e;
  double r = 0.0;
#pragma unroll
  for (int n = 0; n < NPE; n++) r += shape_val(u, n) * rn[n];
  pos[base + k].w = fp32_of(T, (float)r, nullptr);
}

template <bool EV>
__global__ void __launch_bounds__(128, EV ? 4 : 8) k_eam_force32(Args32 A, Eam32 T, const double *phi_site) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool valid = i < A.nsi;
  float fi[3] = {0, 0, 0}, esum = 0.f, vsum[6] = {0, 0, 0, 0, 0, 0};
  double eemb_site = 0.0, eemb_global = 0.0;
  if (valid) {
    float4 oi;
    int ai[3];
    site_frame(A, i, oi, ai);
    const float fpi = oi.w;
    for_each32(A, i, oi, ai, [&](float dx, float dy, float dz, float fpj) {
      float rsq = dx * dx + dy * dy + dz * dz;
      if (rsq < T.cutforcesq) {
        float recip = rsqrtf(rsq);
        float r = rsq * recip;
        float p = r * T.rdr + 1.0f;
        int m = (int)p;
        m = max(1, min(m, T.nr - 1));
        p -= (float)m;
        p = fminf(p, 1.0f);
        float4 rd = T.rhor_der[m];
        float rhop = (rd.x * p + rd.y) * p + rd.z;
        float4 zd = T.z2r_der[m];
        float4 zv = T.z2r_val[m];
        float z2p = (zd.x * p + zd.y) * p + zd.z;
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
    });
    if (EV && A.eflag) {
      double phi = phi_site[i];
      eemb_site = phi;
      eemb_global = (i < A.na) ? phi : phi * A.escale_node * 2.0;
    }
  }
  finish32(A, i, valid, fi, EV, esum, vsum, eemb_site, eemb_global);
}

__global__ void k_reduce_partials32(const double *partial, int nblocks, double *out) {
  int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (k >= 7) return;
  double s = 0.0;
  for (int b = lane; b < nblocks; b += 32) s += partial[b * 7 + k];
  s = warp_sum(s);
  if (lane == 0) out[k] = s;
}

AnchorGrid make_anchor_grid(const Ctx &c) {
  AnchorGrid G;
  int off = 0;
  for (int d = 0; d < 3; d++) {
    G.lo[d] = c.boxlo[d];
    G.n[d] = (int)std::ceil(c.prd[d] / CELL);
    G.r[d] = (float)(c.prd[d] - CELL * G.n[d]);
    int need = G.n[d] + 2 * BIAS, bits = 1;
    while ((1 << bits) < need) bits++;
    G.bits[d] = bits;
    G.shift[d] = off;
    off += bits;
  }
  if (off > 32) throw Error(CACB200_EINVAL, "box too large for the mixed-precision anchor word");
  return G;
}

}  // namespace

void mixed_tables(Ctx &c) {
  auto conv = [&](DBuf<double4> &src, DBuf<float4> &dst, int n) {
    std::vector<double4> h(n + 1);
    stream_copy(c, h.data(), src.p, sizeof(double4) * (n + 1), cudaMemcpyDeviceToHost);
    std::vector<float4> g(n + 1);
    for (int m = 0; m <= n; m++) g[m] = make_float4((float)h[m].x, (float)h[m].y, (float)h[m].z, (float)h[m].w);
    dst.reserve(n + 1);
    stream_copy(c, dst.p, g.data(), sizeof(float4) * (n + 1), cudaMemcpyHostToDevice);
  };
  conv(c.rhor_val, c.rhor_val32, c.pp.nr);
  conv(c.rhor_der, c.rhor_der32, c.pp.nr);
  conv(c.z2r_val, c.z2r_val32, c.pp.nr);
  conv(c.z2r_der, c.z2r_der32, c.pp.nr);
  conv(c.frho_val, c.frho_val32, c.pp.nrho);
  conv(c.frho_der, c.frho_der32, c.pp.nrho);
}

void pair_compute_mixed(Ctx &c, int eflag, int vflag) {
  const int nsi = c.nsite_i();
  const int ns = c.nsite_s();
  const int T = 128;
  const int nb = std::max(nblk(nsi, T), 1);
  AnchorGrid G = make_anchor_grid(c);
  c.pos32.reserve(std::max(ns, 1));
  c.anc32.reserve(std::max(ns, 1));
  c.overflow.reserve(8);
  {
    KernelTimer t(c, "pack32");
    k_pack32<<<nblk(ns, 256), 256, 0, c.stream>>>(c.xs.p, ns, G, c.pos32.p, c.anc32.p, c.overflow.p + 6);
  }
  Args32 A;
  A.pos = c.pos32.p;
  A.anc = c.anc32.p;
  A.nbr = c.nbr_full.p;
  A.num = c.num_full.p;
  A.na = c.na;
  A.ne = c.ne;
  A.nsi = nsi;
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
    Tb.rhor_val = c.rhor_val32.p;
    Tb.rhor_der = c.rhor_der32.p;
    Tb.z2r_val = c.z2r_val32.p;
    Tb.z2r_der = c.z2r_der32.p;
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
    {
      KernelTimer t(c, "eam_rho32");
      k_eam_rho32<<<nb, T, 0, c.stream>>>(A, Tb, c.rho.p, c.phi_site.p, c.pos32.p);
    }
    if (c.nact) {
      KernelTimer t(c, "eam_site_fp32");
      k_eam_site_fp32<<<nblk(c.nact, 256), 256, 0, c.stream>>>(c.pos32.p, c.act_gid.p, c.nact, c.na + NG * c.ne,
                                                               c.na, c.rho.p, Tb);
    }
    {
      KernelTimer t(c, "eam_force32");
      if (ev) k_eam_force32<true><<<nb, T, 0, c.stream>>>(A, Tb, c.phi_site.p);
      else k_eam_force32<false><<<nb, T, 0, c.stream>>>(A, Tb, c.phi_site.p);
    }
  }
  if (ev) {
    k_reduce_partials32<<<1, 256, 0, c.stream>>>(c.partial.p, nb, c.ev_out.p);
    c.have_peratom_e = (eflag & CACB200_ENERGY_ATOM) != 0;
    c.have_peratom_v = (vflag & CACB200_VIRIAL_ATOM) != 0;
    c.ev_pending = true;
  }
  CACB200_CUDA(cudaGetLastError());
}

}  // namespace cacb200
