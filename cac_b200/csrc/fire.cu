// FIRE energy minimisation over atoms and element nodes, controlled on the
// device.
//
// The reference has no FIRE minimiser: Min carries only its parameters
// (min.h:61-72, defaults min.cpp:33-47) and the stop codes (min.h:46-47).
// This is FIRE 2.0 (Guenole et al., Comput. Mater. Sci. 175, 109584 (2020),
// Algorithm 2: semi-implicit Euler, velocity mixing, delayed time-step
// growth, half step back on uphill motion) over the combined degree-of-freedom
// vector of the reference's minimisers (atoms, then nodes,
// min_linesearch.cpp:118-160), with node mass = atom mass as in fix nve, the
// displacement cap dmax of Min, and the stopping tests of Min (energy change
// relative to |E|, force-norm squared under ftol^2).
//
// Every decision (time step, mixing, reset, convergence) is taken by a
// one-block kernel from device reductions, so iterations queue without host
// round trips; the host looks at the status only every few iterations.
#include <cmath>

#include "ctx.cuh"
#include "device.cuh"

namespace cacb200 {

namespace {

inline int nblk(long n, int t) { return (int)((n + t - 1) / t); }

constexpr double FTM2V = 1.0 / 1.0364269e-4;   // metal units, update.cpp:161-164
constexpr double EPS_ENERGY = 1.0e-8;

// per-block partials: [0] v.f  [1] v.v  [2] f.f  [3] max|v_d|  [4] max|f_d|  [5] max_i |f_i|^2
constexpr int NP = 6;

__global__ void k_fire_dots(const double *v, const double *f, int na, const double *nodev,
                            const double *nodef, int nn, double *partial) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  double vf = 0, vv = 0, ff = 0, vmax = 0, fmx = 0, fi2 = 0;
  const double *vp = nullptr, *fp = nullptr;
  if (t < na) {
    vp = v + 3 * (size_t)t;
    fp = f + 3 * (size_t)t;
  } else if (t - na < nn) {
    vp = nodev + 3 * (size_t)(t - na);
    fp = nodef + 3 * (size_t)(t - na);
  }
  if (vp) {
#pragma unroll
    for (int d = 0; d < 3; d++) {
      vf += vp[d] * fp[d];
      vv += vp[d] * vp[d];
      ff += fp[d] * fp[d];
      vmax = fmax(vmax, fabs(vp[d]));
      fmx = fmax(fmx, fabs(fp[d]));
    }
    fi2 = fp[0] * fp[0] + fp[1] * fp[1] + fp[2] * fp[2];
  }
  // sums by the deterministic block reduction; maxima by warp shuffles
  double s[3] = {vf, vv, ff};
  block_reduce_store<3>(s, partial + 0);  // writes partial[blockIdx*3 + k]
  for (int o = 16; o > 0; o >>= 1) {
    vmax = fmax(vmax, __shfl_down_sync(0xffffffffu, vmax, o));
    fmx = fmax(fmx, __shfl_down_sync(0xffffffffu, fmx, o));
    fi2 = fmax(fi2, __shfl_down_sync(0xffffffffu, fi2, o));
  }
  __shared__ double sm[3][32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sm[0][warp] = vmax;
    sm[1][warp] = fmx;
    sm[2][warp] = fi2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int nw = (blockDim.x + 31) >> 5;
    double a = 0, b = 0, c = 0;
    for (int w = 0; w < nw; w++) {
      a = fmax(a, sm[0][w]);
      b = fmax(b, sm[1][w]);
      c = fmax(c, sm[2][w]);
    }
    double *q = partial + 3 * (size_t)gridDim.x + 3 * (size_t)blockIdx.x;
    q[0] = a;
    q[1] = b;
    q[2] = c;
  }
}

// Iteration control (one block).  Order per iteration, as in the published
// algorithm and the reference's Min driver: test convergence of the previous
// force evaluation, then adapt dt and alpha from P = v.f, then publish the
// coefficients of the update kernel.
__global__ void k_fire_control(const double *partial, int nb, const double *ev_out, FireState *S,
                               FireParams P) {
  __shared__ double red[6][256];
  int t = threadIdx.x;
  double a[6] = {0, 0, 0, 0, 0, 0};
  for (int b = t; b < nb; b += blockDim.x) {
    a[0] += partial[3 * b + 0];
    a[1] += partial[3 * b + 1];
    a[2] += partial[3 * b + 2];
    const double *q = partial + 3 * (size_t)nb + 3 * (size_t)b;
    a[3] = fmax(a[3], q[0]);
    a[4] = fmax(a[4], q[1]);
    a[5] = fmax(a[5], q[2]);
  }
  for (int k = 0; k < 6; k++) red[k][t] = a[k];
  __syncthreads();
  if (t != 0) return;
  // fixed-order final reduction
  double vdotf = 0, vdotv = 0, fdotf = 0, vmax = 0, fmaxd = 0, fmax2 = 0;
  for (int k = 0; k < (int)blockDim.x; k++) {
    vdotf += red[0][k];
    vdotv += red[1][k];
    fdotf += red[2][k];
    vmax = fmax(vmax, red[3][k]);
    fmaxd = fmax(fmaxd, red[4][k]);
    fmax2 = fmax(fmax2, red[5][k]);
  }
  FireState &s = *S;
  s.apply = 0;
  if (s.status >= 0) return;
  // convergence of the state reached by the previous iteration
  s.fnorm = (P.normstyle == 1) ? fmax2 : (P.normstyle == 2 ? fmaxd * fmaxd : fdotf);
  if (s.iter > 0) {
    s.eprev = s.ecur;
    s.ecur = ev_out[0];
    if (P.etol > 0.0 && s.step - s.last_negative > P.delaystep &&
        fabs(s.ecur - s.eprev) < P.etol * 0.5 * (fabs(s.ecur) + fabs(s.eprev) + EPS_ENERGY)) {
      s.status = 2;  // ETOL
      return;
    }
    if (P.ftol > 0.0 && s.fnorm < P.ftol * P.ftol) {
      s.status = 3;  // FTOL
      return;
    }
  } else {
    s.ecur = ev_out[0];
  }
  if (s.iter >= P.maxiter) {
    s.status = 0;  // MAXITER
    return;
  }
  s.iter += 1;
  s.step += 1;
  s.vdotf = vdotf;
  s.reset = 0;
  if (vdotf > 0.0) {
    s.vdotf_neg = 0;
    if (s.step - s.last_negative > P.delaystep) {
      s.dt = fmin(s.dt * P.dtgrow, P.dtmax);
      s.alpha *= P.alphashrink;
    }
  } else {
    s.last_negative = s.step;
    bool delayed = !(P.delaystep_start && s.step - s.start < P.delaystep);
    if (delayed) {
      s.alpha = P.alpha0;
      if (s.dt * P.dtshrink >= P.dtmin) s.dt *= P.dtshrink;
    }
    s.vdotf_neg += 1;
    if (P.max_vdotf_negatif > 0 && s.vdotf_neg > P.max_vdotf_negatif) {
      s.status = 11;  // MAXVDOTF
      return;
    }
    s.reset = 1;
  }
  // displacement cap: no coordinate moves further than dmax in one step
  double vest = s.reset ? s.dt * FTM2V / P.mass * fmaxd : vmax;
  double dtv = s.dt;
  if (dtv * vest > P.dmax && vest > 0.0) dtv = P.dmax / vest;
  s.halfback = (s.reset && P.halfstepback) ? 0.5 * s.dtv : 0.0;
  s.dtv = dtv;
  s.mix = (vdotf > 0.0) ? 1 : 0;
  s.s1 = 1.0 - s.alpha;
  s.s2 = (fdotf <= 1e-20) ? 0.0 : s.alpha * sqrt(vdotv / fdotf);
  s.apply = 1;
}

// Semi-implicit Euler step with FIRE mixing (Algorithm 2 of the paper):
// optional half step back and velocity reset, v += dt F/m, mixing, x += dt v.
// The FIRE move; like the velocity-Verlet drift it tests each site's
// displacement since the list build (the inner-prefix flag of its replica).
__global__ void k_fire_update(double4 *xs, double *v, const double *f, int na, double *nodex,
                              double *nodev, const double *nodef, int nn3, const FireState *S,
                              double mass, const double4 *xb, const double *nxb, int *inner_ok, double lim2,
                              double limc, const int *site_rep, const int *elem_rep) {
  if (!S->apply) return;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  const double dtv = S->dtv, dtfm = dtv * FTM2V / mass, hb = S->halfback;
  const double s1 = S->s1, s2 = S->s2;
  const int reset = S->reset, mix = S->mix;
  if (t < na) {
    double4 p = xs[t];
    double *vi = v + 3 * (size_t)t;
    const double *fi = f + 3 * (size_t)t;
    double *q = &p.x;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      double vd = vi[d];
      if (reset) {
        q[d] -= hb * vd;
        vd = 0.0;
      }
      vd += dtfm * fi[d];
      if (mix) vd = s1 * vd + s2 * fi[d];
      q[d] += dtv * vd;
      vi[d] = vd;
    }
    xs[t] = p;
    if (xb) {
      const double4 b = xb[t];
      const double dx = p.x - b.x, dy = p.y - b.y, dz = p.z - b.z;
      if (dx * dx + dy * dy + dz * dz > lim2) inner_ok[site_rep ? site_rep[t] : 0] = 0;
    }
    return;
  }
  int k = t - na;
  if (k >= nn3) return;
  double vd = nodev[k];
  double x = nodex[k];
  if (reset) {
    x -= hb * vd;
    vd = 0.0;
  }
  vd += dtfm * nodef[k];
  if (mix) vd = s1 * vd + s2 * nodef[k];
  const double xn = x + dtv * vd;
  nodex[k] = xn;
  nodev[k] = vd;
  if (nxb && fabs(xn - nxb[k]) > limc) inner_ok[elem_rep ? elem_rep[k / 24] : 0] = 0;
}

__global__ void k_zero(double *a, size_t n) {
  size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t < n) a[t] = 0.0;
}

}  // namespace

void fire_init(Ctx &c, double dt) {
  c.fire_state.reserve(1);
  FireState s;
  s.dt = dt;
  s.alpha = c.fire.alpha0;
  s.dtv = dt;
  s.halfback = 0.0;
  s.s1 = s.s2 = 0.0;
  s.vdotf = 0.0;
  s.ecur = s.eprev = 0.0;
  s.fnorm = 0.0;
  s.step = 0;
  s.last_negative = 0;
  s.start = 0;
  s.vdotf_neg = 0;
  s.reset = 0;
  s.mix = 0;
  s.apply = 0;
  s.status = -1;
  s.iter = 0;
  stream_copy(c, c.fire_state.p, &s, sizeof(FireState), cudaMemcpyHostToDevice);
  c.fire.dtmax = c.fire.tmax * dt;
  c.fire.dtmin = c.fire.tmin * dt;
  // minimisation starts from rest (Min::setup zeroes velocities for FIRE)
  if (c.na) k_zero<<<nblk(3 * c.na, 256), 256, 0, c.stream>>>(c.v.p, 3 * (size_t)c.na);
  if (c.ne) k_zero<<<nblk(24 * c.ne, 256), 256, 0, c.stream>>>(c.nodev.p, 24 * (size_t)c.ne);
}

// One queued FIRE step: reductions and control from the current forces, then
// the velocity/position update (the force evaluation follows, after the
// caller's list-rebuild decision, as in Min::energy_force).
void fire_step(Ctx &c) {
  int nsite = c.na + 8 * c.ne;
  int nb = std::max(nblk(nsite, 256), 1);
  c.fire_partial.reserve((size_t)6 * nb);
  c.fire.mass = c.mass;
  {
    KernelTimer t(c, "fire_dots");
    k_fire_dots<<<nb, 256, 0, c.stream>>>(c.v.p, c.f.p, c.na, c.nodev.p, c.nodef.p, 8 * c.ne,
                                          c.fire_partial.p);
  }
  {
    KernelTimer t(c, "fire_control");
    k_fire_control<<<1, 256, 0, c.stream>>>(c.fire_partial.p, nb, c.ev_out.p, c.fire_state.p, c.fire);
  }
  int n = c.na + 24 * c.ne;
  if (n) {
    KernelTimer t(c, "fire_update");
    const bool check = c.lists_valid && c.inner_ok.p && c.xbuild.p && inner_limit(c) > 0.0;
    const double lim = inner_limit(c);
    k_fire_update<<<nblk(n, 256), 256, 0, c.stream>>>(
        c.xs.p, c.v.p, c.f.p, c.na, c.nodex.p, c.nodev.p, c.nodef.p, 24 * c.ne, c.fire_state.p, c.mass,
        check ? c.xbuild.p : nullptr, check ? c.nodex_build.p : nullptr, c.inner_ok.p, lim * lim,
        lim / 1.7320508075688772, c.nrep > 1 ? c.site_rep.p : nullptr, c.nrep > 1 ? c.elem_rep.p : nullptr);
  }
}

FireState fire_read(Ctx &c) {
  FireState s;
  stream_copy(c, &s, c.fire_state.p, sizeof(FireState), cudaMemcpyDeviceToHost);
  return s;
}

}  // namespace cacb200
