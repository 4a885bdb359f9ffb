// Element interpolation, nodal-force assembly and velocity-Verlet updates.
#include "ctx.cuh"
#include "device.cuh"

namespace cacb200 {

namespace {

inline int nblk(long n, int t) { return (int)((n + t - 1) / t); }

// The pair table for this step: atoms in list-slot order (gathered from the
// site table), then the positions of the Gauss points (their nodes) and of
// every active lattice site from the current nodes, x_u = sum_n N_n(u) x_n,
// the interpolation the reference repeats per pair (pair_lj_cut.cpp:364-368,
// pair_eam.cpp:959-964).  The number of active sites is read on the device
// (written by the last rebuild), so a fixed grid strides over the table.
__global__ void k_pair_table(const double4 *xs, double4 *xss, const int *slot_atom, const double *nodex, int na,
                             int ne, const int *act_gid, const int *nact_dev) {
  const int ngp = NG * ne;
  const int n = na + ngp + *nact_dev;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    if (t < na) {
      double4 p = xs[slot_atom[t]];
      p.w = 0.0;
      xss[t] = p;
      continue;
    }
    const int s = t - na;
    if (s < ngp) {
      int e = s / NG, g = s % NG;
      const double *nx = nodex + (size_t)e * 24 + 3 * gauss_node(g);
      xss[t] = make_double4(nx[0], nx[1], nx[2], 0.0);
      continue;
    }
    int gid = act_gid[s - ngp];
    int e = gid / NU, u = gid % NU;
    const double *nx = nodex + (size_t)e * 24;
    double x = 0.0, y = 0.0, z = 0.0;
#pragma unroll
    for (int m = 0; m < NPE; m++) {
      double N = shape_val(u, m);
      x += N * nx[3 * m];
      y += N * nx[3 * m + 1];
      z += N * nx[3 * m + 2];
    }
    xss[t] = make_double4(x, y, z, 0.0);
  }
}

// Element::compute_nodef, CONSISTENT (element.cpp:2178-2210): force columns
// fc[n] = sum_g wsa[g][n] gaussf[g] with wsa = shape * weight / nucell, then
// nodef[a] += sum_b Minv[a][b] fc[b] with the Hex inverse mass matrix
// (element.cpp:1784-1850, the tensor product of [[4,-2],[-2,4]]).  With the
// Gauss points on the nodes, wsa[g][n] = 1/8 when g sits on n, else 0; the
// loops keep the reference's order of terms.  One thread per (element,
// node): the element's 8 threads read its 24 Gauss-point components
// together and each writes its node's force.
__global__ void k_assemble(const double *gaussf, double *nodef, int ne) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const int e = (int)(t >> 3), a = (int)(t & 7);
  if (e >= ne) return;
  const double weight = (double)NU / (1.0 * 8) * 1.0;   // UNIFORM node weight
  const double *gf = gaussf + (size_t)e * 24;
  double fc[8][3];
#pragma unroll
  for (int n = 0; n < 8; n++) fc[n][0] = fc[n][1] = fc[n][2] = 0.0;
#pragma unroll
  for (int g = 0; g < NG; g++) {
    int gn = gauss_node(g);
#pragma unroll
    for (int n = 0; n < NPE; n++) {
      double w = (n == gn ? 1.0 : 0.0) * weight / NU;
#pragma unroll
      for (int d = 0; d < 3; d++) fc[n][d] += w * gf[3 * g + d];
    }
  }
  double *nf = nodef + (size_t)e * 24;
  double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int b = 0; b < NPE; b++) {
    double m = (node_xi(a) == node_xi(b) ? 4.0 : -2.0) * (node_eta(a) == node_eta(b) ? 4.0 : -2.0) *
               (node_zeta(a) == node_zeta(b) ? 4.0 : -2.0);
#pragma unroll
    for (int d = 0; d < 3; d++) acc[d] += m * fc[b][d];
  }
  nf[3 * a] = acc[0];
  nf[3 * a + 1] = acc[1];
  nf[3 * a + 2] = acc[2];
}

// FixNVE::initial_integrate (fix_nve.cpp:62-145): half kick and drift for
// atoms (positions live in the site table; threads [0, na)) and nodes (one
// thread per node from napad, a multiple of 32, so that every warp holds
// whole elements).  With xb, the drift also records each site's distance
// from where the lists were built, rounded up, for the prefix rule
// (PrefixRule, ctx.cuh): disp per atom, edisp per element (its largest node
// displacement), and the largest of all per replica into dmax (cleared
// before the launch; non-negative floats as bits, whose integer order is
// theirs).
__global__ void k_nve_initial(double4 *xs, double *v, const double *f, int na, int napad, double *nodex,
                              double *nodev, const double *nodef, int nnode, double dtfm, double dtv, int prekick,
                              const double4 *xb, const double *nxb, float *disp, float *edisp, unsigned *dmax,
                              const int *site_rep, const int *elem_rep) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  float d = 0.0f;
  int rep = 0;
  if (t < na) {
    double4 p = xs[t];
    double *vi = v + 3 * (size_t)t;
    const double *fi = f + 3 * (size_t)t;
    // separate roundings, as the reference's x86-64 build evaluates them;
    // prekick: the previous step's second half-kick first (k_nve_final's
    // operations on the same forces)
    double vx = vi[0], vy = vi[1], vz = vi[2];
    if (prekick) {
      vx = __dadd_rn(vx, __dmul_rn(dtfm, fi[0]));
      vy = __dadd_rn(vy, __dmul_rn(dtfm, fi[1]));
      vz = __dadd_rn(vz, __dmul_rn(dtfm, fi[2]));
    }
    vx = __dadd_rn(vx, __dmul_rn(dtfm, fi[0]));
    vy = __dadd_rn(vy, __dmul_rn(dtfm, fi[1]));
    vz = __dadd_rn(vz, __dmul_rn(dtfm, fi[2]));
    vi[0] = vx;
    vi[1] = vy;
    vi[2] = vz;
    p.x = __dadd_rn(p.x, __dmul_rn(dtv, vx));
    p.y = __dadd_rn(p.y, __dmul_rn(dtv, vy));
    p.z = __dadd_rn(p.z, __dmul_rn(dtv, vz));
    xs[t] = p;
    if (xb) {
      const double4 b = xb[t];
      const double dx = p.x - b.x, dy = p.y - b.y, dz = p.z - b.z;
      d = __double2float_ru(__dsqrt_ru(__dadd_ru(__dadd_ru(__dmul_ru(dx, dx), __dmul_ru(dy, dy)), __dmul_ru(dz, dz))));
      disp[t] = d;
      if (site_rep) rep = site_rep[t];
    }
  } else if (t >= napad) {
    const int k = t - napad;   // node 8 e + n of element e
    if (k < nnode) {
      double dd = 0.0;
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const size_t m = 3 * (size_t)k + c;
        double vn = nodev[m];
        if (prekick) vn = __dadd_rn(vn, __dmul_rn(dtfm, nodef[m]));
        vn = __dadd_rn(vn, __dmul_rn(dtfm, nodef[m]));
        nodev[m] = vn;
        const double xn = __dadd_rn(nodex[m], __dmul_rn(dtv, vn));
        nodex[m] = xn;
        if (nxb) {
          const double e = xn - nxb[m];
          dd = __dadd_ru(dd, __dmul_ru(e, e));
        }
      }
      if (nxb) {
        d = __double2float_ru(__dsqrt_ru(dd));
        if (elem_rep) rep = elem_rep[k / 8];
      }
    }
    if (nxb) {
      // the element's largest node displacement over its 8 lanes
      float m = d;
      m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 4));
      m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 2));
      m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 1));
      if ((k & 7) == 0 && k < nnode) edisp[k / 8] = m;
    }
  }
  if (!dmax) return;
  const unsigned bits = __float_as_uint(d);
  if (!site_rep) {
    // one system: the block's largest, one atomic per block
    __shared__ unsigned wmax[32];
    const unsigned m = __reduce_max_sync(0xffffffffu, bits);
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned mm = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) mm = max(mm, wmax[w]);
      if (mm) atomicMax(dmax, mm);
    }
  } else {
    // a batch: one atomic per warp when its sites share a replica
    const int r0 = __shfl_sync(0xffffffffu, rep, 0);
    if (__all_sync(0xffffffffu, rep == r0)) {
      const unsigned m = __reduce_max_sync(0xffffffffu, bits);
      if ((threadIdx.x & 31) == 0 && m) atomicMax(dmax + r0, m);
    } else if (bits) {
      atomicMax(dmax + rep, bits);
    }
  }
}

// FixNVE::final_integrate (fix_nve.cpp:148-219)
__global__ void k_nve_final(double *v, const double *f, int n3, double *nodev, const double *nodef,
                            int nn3, double dtfm) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n3) {
    v[t] = __dadd_rn(v[t], __dmul_rn(dtfm, f[t]));
    return;
  }
  int k = t - n3;
  if (k >= nn3) return;
  nodev[k] = __dadd_rn(nodev[k], __dmul_rn(dtfm, nodef[k]));
}

}  // namespace

void interpolate_sites(Ctx &c) {
  if (c.na + c.ne == 0 || !c.lists_valid) return;
  KernelTimer t(c, "interpolate");
  if (c.precision == CACB200_MIXED) {
    pair_table_mixed(c);   // fixed-point records directly (pair32.cu)
    return;
  }
  // 64 blocks per SM, as the mixed form's pair table
  k_pair_table<<<std::min(nblk((long)c.na + (long)NG * c.ne + (long)c.ne * NU, 256), 148 * 64), 256, 0, c.stream>>>(
      c.xs.p, c.xss.p, c.slot_atom.p, c.nodex.p, c.na, c.ne, c.act_gid.p, c.dev_nact.p);
}

void assemble_nodef(Ctx &c) {
  if (c.ne == 0) return;
  KernelTimer t(c, "assemble");
  k_assemble<<<nblk(8L * c.ne, 128), 128, 0, c.stream>>>(c.gaussf.p, c.nodef.p, c.ne);
}

void nve_initial(Ctx &c, double dt, bool prekick) {
  c.forces_current = false;   // the drift moves every site
  double dtf = 0.5 * dt * (1.0 / 1.0364269e-4);   // metal units, update.cpp:161-164
  double dtfm = dtf / c.mass;
  if (c.na + c.ne == 0) return;
  KernelTimer t(c, "nve_initial");
  const bool check = c.lists_valid && c.inner_ok.p && c.xbuild.p && c.disp.p && inner_limit(c) > 0.0;
  if (check) CACB200_CUDA(cudaMemsetAsync(c.dmax.p, 0, sizeof(unsigned) * c.nrep, c.stream));
  const int napad = (c.na + 31) & ~31;
  const long n = (long)napad + 8L * c.ne;
  const bool many = c.nrep > 1;
  k_nve_initial<<<nblk(n, 256), 256, 0, c.stream>>>(
      c.xs.p, c.v.p, c.f.p, c.na, napad, c.nodex.p, c.nodev.p, c.nodef.p, 8 * c.ne, dtfm, dt, prekick ? 1 : 0,
      check ? c.xbuild.p : nullptr, check ? c.nodex_build.p : nullptr, c.disp.p, c.edisp.p,
      check ? c.dmax.p : nullptr, many ? c.site_rep.p : nullptr, many ? c.elem_rep.p : nullptr);
}

// Neighbor::check_distance (neighbor.cpp:1617-1683): does any atom or node
// lie farther than the trigger distance from where the lists were built?
// (the reference's operation order, without fused multiply-adds)
__global__ void k_moved(const double4 *xs, const double4 *xb, int na, const double *nodex, const double *nxb,
                        int nnode, double deltasq, int *flag) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  double dx, dy, dz;
  if (t < na) {
    const double4 p = xs[t], b = xb[t];
    dx = p.x - b.x;
    dy = p.y - b.y;
    dz = p.z - b.z;
  } else if (t < na + nnode) {
    const double *p = nodex + 3 * (size_t)(t - na), *b = nxb + 3 * (size_t)(t - na);
    dx = p[0] - b[0];
    dy = p[1] - b[1];
    dz = p[2] - b[2];
  } else {
    return;
  }
  const double rsq = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
  if (rsq > deltasq) *flag = 1;
}

// The check of neigh_modify check yes.  Trigger: half the skin
// (triggersq, neighbor.cpp:240); while the box changes, half of the skin
// less the movement of the box's lo and hi corners since the build
// (orthogonal boxes; for a batch the smallest over its replicas).  Reads one
// flag back (synchronises).
bool moved_past_trigger(Ctx &c) {
  double deltasq = 0.25 * c.skin * c.skin;
  if (c.dfm.on && c.build_box.size() == 6 * c.rep_h.size()) {
    bool first = true;
    for (size_t r = 0; r < c.rep_h.size(); r++) {
      const BoxD &B = c.rep_h[r].b;
      const double *h = c.build_box.data() + 6 * r;
      const double lx = B.lo[0] - h[0], ly = B.lo[1] - h[1], lz = B.lo[2] - h[2];
      const double delta1 = sqrt(lx * lx + ly * ly + lz * lz);
      const double ux = B.hi[0] - h[3], uy = B.hi[1] - h[4], uz = B.hi[2] - h[5];
      const double delta2 = sqrt(ux * ux + uy * uy + uz * uz);
      const double delta = 0.5 * (c.skin - (delta1 + delta2));
      if (first || delta * delta < deltasq) deltasq = delta * delta;
      first = false;
    }
  }
  c.moved.reserve(1);
  CACB200_CUDA(cudaMemsetAsync(c.moved.p, 0, sizeof(int), c.stream));
  const int n = c.na + 8 * c.ne;
  if (n)
    k_moved<<<nblk(n, 256), 256, 0, c.stream>>>(c.xs.p, c.xbuild.p, c.na, c.nodex.p, c.nodex_build.p, 8 * c.ne,
                                                deltasq, c.moved.p);
  int h = 0;
  stream_copy(c, &h, c.moved.p, sizeof(int), cudaMemcpyDeviceToHost);
  return h != 0;
}

void nve_final(Ctx &c, double dt) {
  double dtf = 0.5 * dt * (1.0 / 1.0364269e-4);
  double dtfm = dtf / c.mass;
  int n = 3 * c.na + 24 * c.ne;
  if (n == 0) return;
  KernelTimer t(c, "nve_final");
  k_nve_final<<<nblk(n, 256), 256, 0, c.stream>>>(c.v.p, c.f.p, 3 * c.na, c.nodev.p, c.nodef.p,
                                                  24 * c.ne, dtfm);
}

}  // namespace cacb200
