// Thermodynamic read-outs reduced on the device: temperature, kinetic,
// potential and total energy, scalar pressure, pressure tensor and volume of
// each replica, so an output step copies CACB200_THERMO_N doubles per replica
// to the host instead of the state and the per-site arrays.
//
// Definitions followed (metal units, thermo_modify norm no):
//   ComputeTemp::dof_compute / compute_scalar / compute_vector
//     (compute_temp.cpp:74-158, 160-243): dof = 3 (atoms + virtual atoms),
//     virtual atoms = nucell * apc per element (group.cpp:1160-1175);
//     atoms add m v^2, an element with CONSISTENT nodal forces adds
//     m nucell sum_kl M[k][l] (v_k . v_l) with the Hex consistent mass
//     matrix M (element.cpp:1959-2060);
//   ComputePressure::compute_scalar / compute_vector
//     (compute_pressure.cpp:140-220): (dof k T + tr W) / 3 / V * nktv2p and
//     (ke_ij + W_ij) / V * nktv2p;
//   Thermo::compute_ke / compute_etotal (thermo.cpp:1913-1936): ke = T dof k / 2;
//   constants of update.cpp:160-172 (metal: pressure in bar; metalgpa: GPa).
// PotEng is the pair energy of the last evaluation (compute_pe.cpp:46-66).
#include <cmath>
#include <vector>

#include "ctx.cuh"
#include "device.cuh"

namespace cacb200 {
namespace {

constexpr double BOLTZ = 8.617343e-5;
constexpr double MVV2E = 1.0364269e-4;
constexpr double NKTV2P_BAR = 1.6021765e6;
constexpr double NKTV2P_GPA = 1.6021765e2;

// per-block sums: [0] sum m v^2 / m, [1..6] KE tensor / m (xx yy zz xy xz yz),
// [7] per-site energy, [8..13] per-site virial (batches)
constexpr int TNV = 14;
constexpr int TB = 256;
constexpr int MAX_BLOCKS = 512;   // blocks per replica: fixes the summation order

struct ThermoArgs {
  const double *v, *nodev;
  const double *eatom, *enode, *vatom, *vnode;
  const int4 *meta;        // per replica: atom offset, atoms, element offset, elements
  double *partial;         // [nrep][B][TNV]
  int B;
  int persite_e, persite_v;
  double node_e, node_v;   // weight of a node's per-site energy / virial in the totals
};

// Hex consistent mass matrix entry (element.cpp:1993-2056): 1/27 halved for
// each natural coordinate in which nodes k and l differ.
__device__ __forceinline__ double hex_mass(int k, int l) {
  int d = (node_xi(k) != node_xi(l)) + (node_eta(k) != node_eta(l)) + (node_zeta(k) != node_zeta(l));
  return d == 0 ? 1.0 / 27.0 : d == 1 ? 1.0 / 54.0 : d == 2 ? 1.0 / 108.0 : 1.0 / 216.0;
}

// Block (b, r) strides over replica r's atoms then elements.
__global__ void __launch_bounds__(TB) k_thermo_partial(ThermoArgs A) {
  const int r = blockIdx.y;
  const int4 m = A.meta[r];
  double acc[TNV];
#pragma unroll
  for (int k = 0; k < TNV; k++) acc[k] = 0.0;
  const long n = (long)m.y + m.w;
  for (long j = (long)blockIdx.x * TB + threadIdx.x; j < n; j += (long)A.B * TB) {
    if (j < m.y) {
      const size_t i = (size_t)m.x + j;
      const double vx = A.v[3 * i], vy = A.v[3 * i + 1], vz = A.v[3 * i + 2];
      acc[0] += vx * vx + vy * vy + vz * vz;
      acc[1] += vx * vx;
      acc[2] += vy * vy;
      acc[3] += vz * vz;
      acc[4] += vx * vy;
      acc[5] += vx * vz;
      acc[6] += vy * vz;
      if (A.persite_e) acc[7] += A.eatom[i];
      if (A.persite_v)
#pragma unroll
        for (int k = 0; k < 6; k++) acc[8 + k] += A.vatom[6 * i + k];
    } else {
      const size_t e = (size_t)m.z + (j - m.y);
      const double *nv = A.nodev + e * 24;
      double vv[NPE][3];
#pragma unroll
      for (int k = 0; k < NPE; k++) {
        vv[k][0] = nv[3 * k];
        vv[k][1] = nv[3 * k + 1];
        vv[k][2] = nv[3 * k + 2];
      }
      double s = 0.0, t[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
      for (int k = 0; k < NPE; k++)
#pragma unroll
        for (int l = 0; l < NPE; l++) {
          const double mkl = hex_mass(k, l);
          s += mkl * (vv[k][0] * vv[l][0] + vv[k][1] * vv[l][1] + vv[k][2] * vv[l][2]);
          t[0] += mkl * vv[k][0] * vv[l][0];
          t[1] += mkl * vv[k][1] * vv[l][1];
          t[2] += mkl * vv[k][2] * vv[l][2];
          t[3] += mkl * vv[k][0] * vv[l][1];
          t[4] += mkl * vv[k][0] * vv[l][2];
          t[5] += mkl * vv[k][1] * vv[l][2];
        }
      acc[0] += s * NU;
#pragma unroll
      for (int k = 0; k < 6; k++) acc[1 + k] += t[k] * NU;
      if (A.persite_e) {
        double es = 0.0;
#pragma unroll
        for (int k = 0; k < NPE; k++) es += A.enode[e * NPE + k];
        acc[7] += A.node_e * es;
      }
      if (A.persite_v) {
        double vs[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int k = 0; k < NPE; k++)
#pragma unroll
          for (int q = 0; q < 6; q++) vs[q] += A.vnode[e * 48 + 6 * k + q];
#pragma unroll
        for (int q = 0; q < 6; q++) acc[8 + q] += A.node_v * vs[q];
      }
    }
  }
  block_reduce_store<TNV>(acc, A.partial + (size_t)r * A.B * TNV);
}

struct FinalArgs {
  const double *partial;
  const double *ev;        // global energy, virial[6] of the last evaluation (single system)
  const int4 *meta;
  const double *vol;       // [nrep] box volumes
  double *out;             // [nrep][CACB200_THERMO_N]
  int B;
  double mass, nktv2p;
  int energy_src, virial_src;   // 0 none (NaN), 1 global tally, 2 per-site sums
};

// One block per replica: warp k sums column k over the B partial rows in a
// fixed order, then thread 0 forms the read-outs.
__global__ void k_thermo_final(FinalArgs F) {
  __shared__ double tot[TNV];
  const int r = blockIdx.x;
  const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (k < TNV) {
    double s = 0.0;
    const double *p = F.partial + (size_t)r * F.B * TNV;
    for (int b = lane; b < F.B; b += 32) s += p[(size_t)b * TNV + k];
    s = warp_sum(s);
    if (lane == 0) tot[k] = s;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  const int4 m = F.meta[r];
  const double nan = __longlong_as_double(0x7ff8000000000000LL);
  const double dof = 3.0 * ((double)m.y + (double)NU * (double)m.w);
  const double tfactor = dof > 0.0 ? MVV2E / (dof * BOLTZ) : 0.0;
  const double temp = tot[0] * F.mass * tfactor;
  const double ke = temp * (0.5 * dof * BOLTZ);
  double pe = nan, w[6] = {nan, nan, nan, nan, nan, nan};
  if (F.energy_src == 1) pe = F.ev[0];
  if (F.energy_src == 2) pe = tot[7];
  for (int q = 0; q < 6; q++) {
    if (F.virial_src == 1) w[q] = F.ev[1 + q];
    if (F.virial_src == 2) w[q] = tot[8 + q];
  }
  const double vol = F.vol[r];
  const double inv_volume = 1.0 / vol;
  double *o = F.out + (size_t)r * CACB200_THERMO_N;
  o[CACB200_THERMO_TEMP] = temp;
  o[CACB200_THERMO_KE] = ke;
  o[CACB200_THERMO_PE] = pe;
  o[CACB200_THERMO_ETOTAL] = pe + ke;
  o[CACB200_THERMO_PRESS] = (dof * BOLTZ * temp + w[0] + w[1] + w[2]) / 3.0 * inv_volume * F.nktv2p;
  for (int q = 0; q < 6; q++)
    o[CACB200_THERMO_PXX + q] = (tot[1 + q] * F.mass * MVV2E + w[q]) * inv_volume * F.nktv2p;
  o[CACB200_THERMO_VOL] = vol;
}

}  // namespace

void thermo(Ctx &c, int units, double *out) {
  c.check_system();
  if (units != CACB200_UNITS_METAL && units != CACB200_UNITS_METALGPA)
    throw Error(CACB200_EINVAL, "unknown unit style");
  if (!out) throw Error(CACB200_EINVAL, "null output array");
  if (c.nrep > 65535) throw Error(CACB200_EINVAL, "at most 65535 replicas per read-out");
  if (c.thermo_gen != c.gen) {
    std::vector<int4> meta(c.nrep);
    std::vector<double> vol(c.nrep);
    for (int r = 0; r < c.nrep; r++) {
      meta[r] = make_int4(c.rep_aoff[r], c.rep_na[r], c.rep_eoff[r], c.rep_ne[r]);
      const BoxD &b = c.rep_h[r].b;
      vol[r] = b.L[0] * b.L[1] * b.L[2];
    }
    c.thermo_meta.reserve(c.nrep);
    c.thermo_vol.reserve(c.nrep);
    stream_copy(c, c.thermo_meta.p, meta.data(), sizeof(int4) * meta.size(), cudaMemcpyHostToDevice);
    stream_copy(c, c.thermo_vol.p, vol.data(), sizeof(double) * vol.size(), cudaMemcpyHostToDevice);
    c.thermo_gen = c.gen;
  }
  long nmax = 1;
  for (int r = 0; r < c.nrep; r++) nmax = std::max(nmax, (long)c.rep_na[r] + c.rep_ne[r]);
  const int B = (int)std::min<long>((nmax + TB - 1) / TB, MAX_BLOCKS);
  c.thermo_part.reserve((size_t)c.nrep * B * TNV);
  c.thermo_out.reserve((size_t)c.nrep * CACB200_THERMO_N);

  const bool single = c.nrep == 1;
  const bool site_e = !single && c.tally_step_ae == c.step;
  const bool site_v = !single && c.tally_step_av == c.step;
  ThermoArgs A{};
  A.v = c.v.p;
  A.nodev = c.nodev.p;
  A.eatom = c.eatom.p;
  A.enode = c.enode.p;
  A.vatom = c.vatom.p;
  A.vnode = c.vnode.p;
  A.meta = c.thermo_meta.p;
  A.partial = c.thermo_part.p;
  A.B = B;
  A.persite_e = site_e;
  A.persite_v = site_v;
  A.node_e = 2.0 * c.escale_node_last;
  A.node_v = (double)NU / (double)NPE;
  k_thermo_partial<<<dim3(B, c.nrep), TB, 0, c.stream>>>(A);

  FinalArgs F{};
  F.partial = c.thermo_part.p;
  F.ev = c.ev_out.p;
  F.meta = c.thermo_meta.p;
  F.vol = c.thermo_vol.p;
  F.out = c.thermo_out.p;
  F.B = B;
  F.mass = c.mass;
  F.nktv2p = units == CACB200_UNITS_METALGPA ? NKTV2P_GPA : NKTV2P_BAR;
  F.energy_src = single ? (c.tally_step_e == c.step ? 1 : 0) : (site_e ? 2 : 0);
  F.virial_src = single ? (c.tally_step_v == c.step ? 1 : 0) : (site_v ? 2 : 0);
  k_thermo_final<<<c.nrep, 32 * TNV, 0, c.stream>>>(F);
  CACB200_CUDA(cudaGetLastError());
  stream_copy(c, out, c.thermo_out.p, sizeof(double) * c.nrep * CACB200_THERMO_N, cudaMemcpyDeviceToHost);
}

}  // namespace cacb200
