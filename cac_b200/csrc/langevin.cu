// fix langevin on the device, drawing the reference's own random stream.
//
// FixLangevin::post_force (fix_langevin.cpp:455-675) adds to every atom and
// every element node a drag gamma1 v and a random force gamma2 (u - 0.5),
// u uniform from one RanMars generator (random_mars.cpp:23-90) drawn in a
// fixed order: atoms x y z, then each element's nodes x y z.  RanMars is
// F. James's RANMAR: Y_n = Y_{n-97} - Y_{n-33} (mod 1) combined with an
// arithmetic sequence C_m = C_0 - m CD (mod CM); every value is a multiple of
// 2^-24, so the whole generator is exact integer arithmetic mod 2^24.
//
// The device generates a call's N = 3 atoms + 24 elements draws in chunks of
// CHUNK draws, one warp each.  A chunk starts from the 97-value window at its
// offset, obtained from the call's starting window by jumping ahead: the
// recurrence has characteristic polynomial P(x) = x^97 + x^64 - 1, and
// x^k mod P gives Y_{a+k} as a fixed combination of Y_a .. Y_{a+96}
// (coefficients precomputed per chunk offset).  Inside a chunk 32 lanes
// produce 32 consecutive values per step (the shorter lag is 33).  Draw q of
// a call lands on the flat force component q of the atoms, then of the nodes,
// so each draw is applied where it is made.  The results equal the
// reference's draw for draw; the drag and random terms use the reference's
// roundings (no contraction into FMA).
//
// A batch gives replica r its own stream with seed + r, as if each replica ran
// in its own process with that seed.
#include <cmath>
#include <vector>

#include "ctx.cuh"
#include "device.cuh"

namespace cacb200 {
namespace {

constexpr unsigned MASK24 = (1u << 24) - 1;
constexpr int WIN = 97;          // window of the long lag
constexpr int EXT = 2 * WIN - 1; // window plus the 96 values after it
constexpr int CHUNK = 512;       // draws per warp
constexpr int WARPS = 4;         // warps (chunks) per block
constexpr long long C0 = 362436, CD = 7654321, CM = 16777213;
constexpr double FTM2V = 1.0 / 1.0364269e-4;   // update.cpp:160-164 (metal)
constexpr double BOLTZ = 8.617343e-5;
constexpr double MVV2E = 1.0364269e-4;

// ------------------------------------------------------------ host: streams

// RanMars::RanMars seeding (random_mars.cpp:29-67) in integers: 97 values of
// 24 bits.  Returns Y_1 .. Y_97 in generation order (Y_k = u[98 - k]).
std::vector<unsigned> seed_window(int seed) {
  int ij = (seed - 1) / 30082;
  int kl = (seed - 1) - 30082 * ij;
  int i = (ij / 177) % 177 + 2, j = ij % 177 + 2, k = (kl / 169) % 178 + 1, l = kl % 169;
  std::vector<unsigned> u(98, 0);
  for (int ii = 1; ii <= 97; ii++) {
    unsigned s = 0;
    for (int jj = 1; jj <= 24; jj++) {
      int m = ((i * j) % 179) * k % 179;
      i = j;
      j = k;
      k = m;
      l = (53 * l + 1) % 169;
      if ((l * m) % 64 >= 32) s |= 1u << (24 - jj);
    }
    u[ii] = s;
  }
  std::vector<unsigned> y(97);
  for (int n = 1; n <= 97; n++) y[n - 1] = u[98 - n];
  return y;
}

// (a * b) mod P over Z/2^24, both of degree < 97.
std::vector<unsigned> polymul(const std::vector<unsigned> &a, const std::vector<unsigned> &b) {
  std::vector<unsigned long long> t(2 * WIN - 1, 0);
  for (int i = 0; i < WIN; i++) {
    if (!a[i]) continue;
    for (int j = 0; j < WIN; j++) t[i + j] += (unsigned long long)a[i] * b[j];
  }
  std::vector<unsigned> r(2 * WIN - 1);
  for (int i = 0; i < 2 * WIN - 1; i++) r[i] = (unsigned)(t[i] & MASK24);
  // x^d = x^(d-97) - x^(d-33) for d >= 97, highest degree first
  for (int d = 2 * WIN - 2; d >= WIN; d--) {
    unsigned c = r[d];
    r[d - WIN] = (r[d - WIN] + c) & MASK24;
    r[d - 33] = (r[d - 33] - c) & MASK24;
  }
  r.resize(WIN);
  return r;
}

// Coefficients of x^(j CHUNK) mod P for j = 0 .. n-1, [j][97].
std::vector<unsigned> jump_table(int n) {
  std::vector<unsigned> one(WIN, 0), step(WIN, 0), cur(WIN, 0);
  one[0] = 1;
  // x^CHUNK by repeated multiplication by x
  step[0] = 1;
  for (int s = 0; s < CHUNK; s++) {
    unsigned top = step[WIN - 1];
    for (int i = WIN - 1; i > 0; i--) step[i] = step[i - 1];
    step[0] = 0;
    // top * x^97 = top * (1 - x^64)
    step[0] = (step[0] + top) & MASK24;
    step[64] = (step[64] - top) & MASK24;
  }
  std::vector<unsigned> out((size_t)n * WIN);
  cur = one;
  for (int j = 0; j < n; j++) {
    std::copy(cur.begin(), cur.end(), out.begin() + (size_t)j * WIN);
    if (j + 1 < n) cur = polymul(cur, step);
  }
  return out;
}

// x^n mod P by squaring.
std::vector<unsigned> xpow(unsigned long long n) {
  std::vector<unsigned> r(WIN, 0), b(WIN, 0);
  r[0] = 1;
  b[1] = 1;
  while (n) {
    if (n & 1) r = polymul(r, b);
    n >>= 1;
    if (n) b = polymul(b, b);
  }
  return r;
}

// The 193 values Y_{B-96} .. Y_{B+96} of a stream after `draws` uniform()
// calls (the constructor's warm-up included), B = 97 + draws the last value
// used: Y_{1+draws+s} = sum_i c_i Y_{1+s+i} with c = x^draws mod P, from the
// seeded values extended to Y_193.
std::vector<unsigned> stream_window(int seed, unsigned long long draws) {
  std::vector<unsigned> y = seed_window(seed);   // Y_1 .. Y_97
  y.resize(EXT);
  for (int n = WIN; n < EXT; n++) y[n] = (y[n - WIN] - y[n - 33]) & MASK24;
  const std::vector<unsigned> c = xpow(draws);
  std::vector<unsigned> w(EXT);
  for (int s = 0; s < WIN; s++) {
    unsigned long long acc = 0;
    for (int i = 0; i < WIN; i++) acc += (unsigned long long)c[i] * y[s + i];
    w[s] = (unsigned)(acc & MASK24);
  }
  for (int n = WIN; n < EXT; n++) w[n] = (w[n - WIN] - w[n - 33]) & MASK24;
  return w;
}

// ---------------------------------------------------------- device kernels

struct LgvArgs {
  double *f, *nodef;
  const double *v, *nodev;
  const unsigned *base;          // [nrep][EXT]: Y_{B-96} .. Y_{B+96}, B the last value drawn
  unsigned *next;                // [nrep][WIN]: the last 97 values of this call
  const unsigned long long *m;   // [nrep] draws made before this call
  const long long *ctl;          // step of this call, first and last step of the run
  const int2 *chunks;            // (replica, chunk index within the replica)
  const int4 *meta;              // per replica: atom offset, atoms, element offset, elements
  const unsigned *poly;          // [j][WIN] jump coefficients
  double *partial;               // [chunk][3] random-force sums (zero yes)
  int nchunks;
  double gfactor1, gfactor2, sqrt_nodal_weight, t_start, t_stop;
};

__device__ __forceinline__ double target_sqrt(const LgvArgs &A) {
  // FixLangevin::compute_target (fix_langevin.cpp:683-694), CONSTANT style
  double delta = (double)(A.ctl[0] - A.ctl[1]);
  if (delta != 0.0) delta = __ddiv_rn(delta, (double)(A.ctl[2] - A.ctl[1]));
  double t_target = __dadd_rn(A.t_start, __dmul_rn(delta, __dsub_rn(A.t_stop, A.t_start)));
  return sqrt(t_target);
}

__global__ void __launch_bounds__(32 * WARPS) k_langevin(LgvArgs A) {
  __shared__ unsigned sb[WARPS][EXT];
  __shared__ unsigned sp[WARPS][WIN];
  __shared__ unsigned seq[WARPS][WIN + CHUNK];   // seq[rho] = Y_{B-96+jC+rho}
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ci = blockIdx.x * WARPS + w;
  if (ci >= A.nchunks) return;   // the whole warp leaves; only warp barriers follow
  const int2 ch = A.chunks[ci];
  const int r = ch.x, j = ch.y;
  const int4 mt = A.meta[r];
  const long long na3 = 3LL * mt.y;
  const long long N = na3 + 24LL * mt.w;
  for (int i = lane; i < EXT; i += 32) sb[w][i] = A.base[(size_t)r * EXT + i];
  for (int i = lane; i < WIN; i += 32) sp[w][i] = A.poly[(size_t)j * WIN + i];
  __syncwarp();
  // window at the chunk's offset
  for (int s = lane; s < WIN; s += 32) {
    unsigned long long acc = 0;
    for (int i = 0; i < WIN; i++) acc += (unsigned long long)sp[w][i] * sb[w][s + i];
    seq[w][s] = (unsigned)(acc & MASK24);
  }
  const long long qbase = (long long)j * CHUNK;
  const int len = (int)min((long long)CHUNK, N - qbase);
  // the chunk's values, 32 per step (the short lag is 33), all in shared
  // memory before any force is touched
  for (int t0 = 0; t0 < len; t0 += 32) {
    __syncwarp();
    const int t = t0 + lane;
    const unsigned y = (seq[w][t] - seq[w][t + 64]) & MASK24;
    seq[w][WIN + t] = y;
  }
  __syncwarp();

  const double tsqrt = target_sqrt(A);
  const double g1 = A.gfactor1;
  const double g2a = __dmul_rn(A.gfactor2, tsqrt);
  const double g2n = __ddiv_rn(__dmul_rn(A.gfactor2, tsqrt), A.sqrt_nodal_weight);
  // C of this lane's first draw, then 32 draws further on per step
  const unsigned long long first = A.m[r] + 1 + qbase + lane;
  long long cm = (C0 - (long long)((first % CM) * CD % CM) + CM) % CM;
  const long long cstep = (32LL * CD) % CM;
  double fs[3] = {0.0, 0.0, 0.0};
  double *fa = A.f + 3LL * mt.x;
  const double *va = A.v + 3LL * mt.x;
  double *fn = A.nodef + 24LL * mt.z;
  const double *vn = A.nodev + 24LL * mt.z;
  unsigned *nx = A.next + (size_t)r * WIN;
  // draw q = qbase + t on force component q of the atoms, then of the nodes;
  // no barrier in this loop, so the loads of successive steps overlap
#pragma unroll 4
  for (int t = lane; t < len; t += 32) {
    const unsigned y = seq[w][WIN + t];
    const long long q = qbase + t;
    const unsigned u = (y - (unsigned)cm) & MASK24;
    const double uni = (double)u * (1.0 / 16777216.0);
    double fran;
    if (q < na3) {
      fran = __dmul_rn(g2a, uni - 0.5);
      fa[q] = __dadd_rn(fa[q], __dadd_rn(__dmul_rn(g1, va[q]), fran));
    } else {
      const long long k = q - na3;
      fran = __dmul_rn(g2n, uni - 0.5);
      fn[k] = __dadd_rn(fn[k], __dadd_rn(__dmul_rn(g1, vn[k]), fran));
    }
    const int d = (int)(q % 3);
    fs[0] += d == 0 ? fran : 0.0;
    fs[1] += d == 1 ? fran : 0.0;
    fs[2] += d == 2 ? fran : 0.0;
    if (q >= N - WIN && N >= WIN) nx[q - (N - WIN)] = y;
    cm -= cstep;
    if (cm < 0) cm += CM;
  }
  if (A.partial) {
#pragma unroll
    for (int d = 0; d < 3; d++) {
      double s = warp_sum(fs[d]);
      if (lane == 0) A.partial[(size_t)ci * 3 + d] = s;
    }
  }
}

// One warp per replica: advance the stream past this call (new window and
// the 96 values after it), count the draws, and form the zero-force means.
// Replica 0's warp also advances the step.
__global__ void k_langevin_advance(unsigned *base, const unsigned *next, unsigned long long *m, long long *ctl,
                                   const int4 *meta, const int2 *rchunk, const double *partial, double *mean,
                                   int nrep) {
  const int r = blockIdx.x;
  const int lane = threadIdx.x;
  if (r >= nrep) return;
  __shared__ unsigned sb[EXT];
  const int4 mt = meta[r];
  const long long N = 3LL * mt.y + 24LL * mt.w;
  if (N > 0) {
    // new window Y_{B+N-96} .. Y_{B+N}: written by the chunks, or for a call
    // of fewer than 97 draws already in the old window and its extension
    for (int i = lane; i < WIN; i += 32)
      sb[i] = N >= WIN ? next[(size_t)r * WIN + i] : base[(size_t)r * EXT + N + i];
    __syncwarp();
    for (int i0 = WIN; i0 < EXT; i0 += 32) {
      int i = i0 + lane;
      unsigned y = 0;
      if (i < EXT) y = (sb[i - WIN] - sb[i - 33]) & MASK24;
      __syncwarp();
      if (i < EXT) sb[i] = y;
      __syncwarp();
    }
    for (int i = lane; i < EXT; i += 32) base[(size_t)r * EXT + i] = sb[i];
    if (lane == 0) m[r] += (unsigned long long)N;
  }
  if (mean && lane < 3) {
    // FixLangevin zero yes: sum over the group / (atoms + elements)
    const int2 rc = rchunk[r];
    double s = 0.0;
    for (int c = 0; c < rc.y; c++) s += partial[(size_t)(rc.x + c) * 3 + lane];
    const double count = (double)(mt.y + mt.w);
    mean[(size_t)r * 3 + lane] = count > 0 ? s / count : 0.0;
  }
  if (r == 0 && lane == 0) ctl[0] += 1;
}

// zero yes: subtract each replica's mean random force from its atoms and nodes
__global__ void k_langevin_zero(double *f, double *nodef, const double *mean, const int *site_rep,
                                const int *elem_rep, int na, int ne) {
  const long long n = 3LL * na + 24LL * ne;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    if (q < 3LL * na) {
      const int r = site_rep ? site_rep[q / 3] : 0;
      f[q] = __dsub_rn(f[q], mean[3 * r + (int)(q % 3)]);
    } else {
      const long long k = q - 3LL * na;
      const int r = elem_rep ? elem_rep[k / 24] : 0;
      nodef[k] = __dsub_rn(nodef[k], mean[3 * r + (int)(k % 3)]);
    }
  }
}

__global__ void k_langevin_begin(long long *ctl, long long step, long long begin, long long end) {
  ctl[0] = step;
  ctl[1] = begin;
  ctl[2] = end;
}

}  // namespace

// fix ID all langevin t_start t_stop t_period seed [zero yes]: validate, seed
// every replica's stream (the constructor's warm-up draw included) and lay
// out the chunks.  A new system or a new set of parameters starts the
// streams afresh, as a new fix would.
void langevin_set(Ctx &c, double t_start, double t_stop, double t_period, int seed, int zero) {
  c.check_system();
  if (!(t_period > 0.0)) throw Error(CACB200_EINVAL, "Fix langevin period must be > 0.0");
  if (seed <= 0 || (long)seed + c.nrep - 1 > 900000000L)
    throw Error(CACB200_EINVAL, "Invalid seed for Marsaglia random # generator");
  if (!(t_start >= 0.0) || !(t_stop >= 0.0)) throw Error(CACB200_EINVAL, "Fix langevin temperatures must be >= 0");
  if (zero)
    for (int r = 0; r < c.nrep; r++)
      if (c.rep_na[r] + c.rep_ne[r] == 0) throw Error(CACB200_EINVAL, "Cannot zero Langevin force of 0 atoms");
  std::vector<unsigned> base((size_t)c.nrep * EXT);
  std::vector<unsigned long long> m(c.nrep, 1);
  std::vector<int2> chunks, rchunk(c.nrep);
  std::vector<int4> meta(c.nrep);
  int maxj = 1;
  for (int r = 0; r < c.nrep; r++) {
    // after the constructor's warm-up draw: window Y_2 .. Y_98, then Y_99 .. Y_194
    const std::vector<unsigned> w = stream_window(seed + r, 1);
    std::copy(w.begin(), w.end(), base.begin() + (size_t)r * EXT);
    const long long N = 3LL * c.rep_na[r] + 24LL * c.rep_ne[r];
    const int nj = (int)((N + CHUNK - 1) / CHUNK);
    rchunk[r] = make_int2((int)chunks.size(), nj);
    for (int j = 0; j < nj; j++) chunks.push_back(make_int2(r, j));
    maxj = std::max(maxj, nj);
    meta[r] = make_int4(c.rep_aoff[r], c.rep_na[r], c.rep_eoff[r], c.rep_ne[r]);
  }
  if (c.lgv_poly_n < maxj) {
    std::vector<unsigned> poly = jump_table(maxj);
    c.lgv_poly.reserve(poly.size());
    stream_copy(c, c.lgv_poly.p, poly.data(), sizeof(unsigned) * poly.size(), cudaMemcpyHostToDevice);
    c.lgv_poly_n = maxj;
  }
  c.lgv_base.reserve(base.size());
  c.lgv_next.reserve((size_t)c.nrep * WIN);
  c.lgv_m.reserve(c.nrep);
  c.lgv_ctl.reserve(3);
  c.lgv_chunks.reserve(std::max<size_t>(chunks.size(), 1));
  c.lgv_rchunk.reserve(c.nrep);
  c.lgv_meta.reserve(c.nrep);
  c.lgv_part.reserve(std::max<size_t>(3 * chunks.size(), 1));
  c.lgv_mean.reserve(3 * (size_t)c.nrep);
  stream_copy(c, c.lgv_base.p, base.data(), sizeof(unsigned) * base.size(), cudaMemcpyHostToDevice);
  stream_copy(c, c.lgv_m.p, m.data(), sizeof(unsigned long long) * m.size(), cudaMemcpyHostToDevice);
  if (!chunks.empty())
    stream_copy(c, c.lgv_chunks.p, chunks.data(), sizeof(int2) * chunks.size(), cudaMemcpyHostToDevice);
  stream_copy(c, c.lgv_rchunk.p, rchunk.data(), sizeof(int2) * rchunk.size(), cudaMemcpyHostToDevice);
  stream_copy(c, c.lgv_meta.p, meta.data(), sizeof(int4) * meta.size(), cudaMemcpyHostToDevice);
  c.lgv.on = true;
  c.lgv.t_start = t_start;
  c.lgv.t_stop = t_stop;
  c.lgv.t_period = t_period;
  c.lgv.seed = seed;
  c.lgv.zero = zero != 0;
  c.lgv_nchunks = (int)chunks.size();
  c.gen++;
}

// Every replica's stream positioned after `draws` uniform() calls of its
// RanMars (the constructor's warm-up is draw 1), e.g. to continue a stream
// the reference's own loop has been drawing from.
void langevin_stream(Ctx &c, long long draws) {
  if (!c.lgv.on) throw Error(CACB200_ESTATE, "no fix langevin set");
  if (draws < 1) throw Error(CACB200_EINVAL, "a RanMars stream has made at least its warm-up draw");
  std::vector<unsigned> base((size_t)c.nrep * EXT);
  for (int r = 0; r < c.nrep; r++) {
    const std::vector<unsigned> w = stream_window(c.lgv.seed + r, (unsigned long long)draws);
    std::copy(w.begin(), w.end(), base.begin() + (size_t)r * EXT);
  }
  std::vector<unsigned long long> m(c.nrep, (unsigned long long)draws);
  stream_copy(c, c.lgv_base.p, base.data(), sizeof(unsigned) * base.size(), cudaMemcpyHostToDevice);
  stream_copy(c, c.lgv_m.p, m.data(), sizeof(unsigned long long) * m.size(), cudaMemcpyHostToDevice);
}

void langevin_unset(Ctx &c) {
  if (c.lgv.on) c.gen++;
  c.lgv.on = false;
}

// Start of a run of nsteps from the current step (Update::beginstep/endstep).
void langevin_begin(Ctx &c, long nsteps) {
  if (!c.lgv.on) return;
  k_langevin_begin<<<1, 1, 0, c.stream>>>(c.lgv_ctl.p, c.step, c.step, c.step + nsteps);
  CACB200_CUDA(cudaGetLastError());
}

// FixLangevin::post_force for the step the device counter holds.
void langevin_post_force(Ctx &c, double dt) {
  if (!c.lgv.on) return;
  c.forces_current = false;   // f and nodef now hold the draws as well
  LgvArgs A{};
  A.f = c.f.p;
  A.nodef = c.nodef.p;
  A.v = c.v.p;
  A.nodev = c.nodev.p;
  A.base = c.lgv_base.p;
  A.next = c.lgv_next.p;
  A.m = c.lgv_m.p;
  A.ctl = c.lgv_ctl.p;
  A.chunks = c.lgv_chunks.p;
  A.meta = c.lgv_meta.p;
  A.poly = c.lgv_poly.p;
  A.partial = c.lgv.zero ? c.lgv_part.p : nullptr;
  A.nchunks = c.lgv_nchunks;
  // FixLangevin::init (fix_langevin.cpp:266-273), one atom type, ratio 1
  A.gfactor1 = -c.mass / c.lgv.t_period / FTM2V;
  A.gfactor2 = std::sqrt(c.mass) * std::sqrt(24.0 * BOLTZ / c.lgv.t_period / dt / MVV2E) / FTM2V;
  A.sqrt_nodal_weight = std::sqrt((double)NU / (double)NPE);
  A.t_start = c.lgv.t_start;
  A.t_stop = c.lgv.t_stop;
  {
    KernelTimer t(c, "langevin");
    if (c.lgv_nchunks > 0)
      k_langevin<<<(c.lgv_nchunks + WARPS - 1) / WARPS, 32 * WARPS, 0, c.stream>>>(A);
    k_langevin_advance<<<c.nrep, 32, 0, c.stream>>>(c.lgv_base.p, c.lgv_next.p, c.lgv_m.p, c.lgv_ctl.p,
                                                     c.lgv_meta.p, c.lgv_rchunk.p, c.lgv_part.p,
                                                     c.lgv.zero ? c.lgv_mean.p : nullptr, c.nrep);
    if (c.lgv.zero)
      k_langevin_zero<<<stride_grid(3L * c.na + 24L * c.ne, 256), 256, 0, c.stream>>>(
          c.f.p, c.nodef.p, c.lgv_mean.p, c.nrep > 1 ? c.site_rep.p : nullptr, c.nrep > 1 ? c.elem_rep.p : nullptr,
          c.na, c.ne);
  }
  CACB200_CUDA(cudaGetLastError());
}

}  // namespace cacb200
