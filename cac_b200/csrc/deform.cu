// fix deform for orthogonal periodic boxes.
//
// FixDeform (fix_deform.cpp) changes the box at the end of every N-th step:
// per dimension a target [lo, hi] from the run's start box and the style
// (final, delta, scale, vel, erate, trate, wiggle, volume; apply_strain and
// apply_volume, fix_deform.cpp:1020-1127), then with remap x the atoms and
// nodes are mapped to fractional coordinates of the old box and back with the
// new one (update_domain, fix_deform.cpp:1129-1240; Domain::x2lamda /
// lamda2x / nodex2lamda / lamda2nodex, domain.cpp:2268-2410).  The box
// arithmetic is a handful of host scalars per replica, restated in the
// reference's order of operations; the remap of every atom and node is one
// device kernel with the same roundings (no contraction into FMA).
//
// The new box reaches the force path through the context's box (single
// system) and replica descriptors (batch); candidate grids and reference bins
// follow at the next list rebuild, which replans them.  Steps with a deforming
// box are queued eagerly (graphs hold the box as a launch argument).
#include <cmath>
#include <cstring>
#include <vector>

#include "ctx.cuh"
#include "device.cuh"

namespace cacb200 {
namespace {

constexpr double MY_2PI = 6.28318530717958647692;   // math_const.h

struct Remap {
  double lo0[3], hinv0[3], lo1[3], h1[3];
};

__device__ __forceinline__ void remap_point(const Remap &R, double &x, double &y, double &z) {
  // x2lamda with the old box, lamda2x with the new one (orthogonal: the tilt
  // terms are zero and drop out exactly)
  double l0 = __dmul_rn(R.hinv0[0], __dsub_rn(x, R.lo0[0]));
  double l1 = __dmul_rn(R.hinv0[1], __dsub_rn(y, R.lo0[1]));
  double l2 = __dmul_rn(R.hinv0[2], __dsub_rn(z, R.lo0[2]));
  x = __dadd_rn(__dmul_rn(R.h1[0], l0), R.lo1[0]);
  y = __dadd_rn(__dmul_rn(R.h1[1], l1), R.lo1[1]);
  z = __dadd_rn(__dmul_rn(R.h1[2], l2), R.lo1[2]);
}

// Atoms (site table, atom order) then nodes; per-replica maps for a batch.
__global__ void k_deform_remap(double4 *xs, int na, double *nodex, int ne, Remap one, const Remap *many,
                               const int *site_rep, const int *elem_rep) {
  const long long n = (long long)na + 8LL * ne;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    if (t < na) {
      const Remap &R = many ? many[site_rep[t]] : one;
      double4 p = xs[t];
      remap_point(R, p.x, p.y, p.z);
      xs[t] = p;
    } else {
      const long long k = t - na;   // node k % 8 of element k / 8
      const Remap &R = many ? many[elem_rep[k / 8]] : one;
      double *p = nodex + 3 * k;
      double x = p[0], y = p[1], z = p[2];
      remap_point(R, x, y, z);
      p[0] = x;
      p[1] = y;
      p[2] = z;
    }
  }
}

}  // namespace

// fix ID all deform N x|y|z style args ... remap x|none units box.
// Validates the styles and links volume dimensions to the others
// (FixDeform::FixDeform, fix_deform.cpp:40-372).
void deform_set(Ctx &c, int nevery, const int *style, const double *a, const double *b, int remap_x) {
  c.check_system();
  if (nevery <= 0) throw Error(CACB200_EINVAL, "Illegal fix deform command");
  if (!style || !a || !b) throw Error(CACB200_EINVAL, "null deform arguments");
  DeformParams P;
  P.nevery = nevery;
  P.remap_x = remap_x != 0;
  bool any = false;
  for (int i = 0; i < 3; i++) {
    if (style[i] < CACB200_DEFORM_NONE || style[i] > CACB200_DEFORM_VOLUME)
      throw Error(CACB200_EINVAL, "Illegal fix deform command");
    DeformDim &d = P.dim[i];
    d.style = style[i];
    d.a = a[i];
    d.b = b[i];
    if (d.style == CACB200_DEFORM_WIGGLE && !(d.b > 0.0)) throw Error(CACB200_EINVAL, "Illegal fix deform command");
    any = any || d.style != CACB200_DEFORM_NONE;
  }
  if (!any) throw Error(CACB200_EINVAL, "Illegal fix deform command");
  for (int i = 0; i < 3; i++) {
    DeformDim &d = P.dim[i];
    if (d.style != CACB200_DEFORM_VOLUME) continue;
    const int o1 = (i + 1) % 3, o2 = (i + 2) % 3;
    const int s1 = P.dim[o1].style, s2 = P.dim[o2].style;
    auto invalid = [] { throw Error(CACB200_EINVAL, "Fix deform volume setting is invalid"); };
    if (s1 == CACB200_DEFORM_NONE) {
      if (s2 == CACB200_DEFORM_NONE || s2 == CACB200_DEFORM_VOLUME) invalid();
      d.substyle = DeformDim::ONE_FROM_ONE, d.fixed = o1, d.dynamic1 = o2;
    } else if (s2 == CACB200_DEFORM_NONE) {
      if (s1 == CACB200_DEFORM_NONE || s1 == CACB200_DEFORM_VOLUME) invalid();
      d.substyle = DeformDim::ONE_FROM_ONE, d.fixed = o2, d.dynamic1 = o1;
    } else if (s1 == CACB200_DEFORM_VOLUME) {
      if (s2 == CACB200_DEFORM_NONE || s2 == CACB200_DEFORM_VOLUME) invalid();
      d.substyle = DeformDim::TWO_FROM_ONE, d.fixed = o1, d.dynamic1 = o2;
    } else if (s2 == CACB200_DEFORM_VOLUME) {
      if (s1 == CACB200_DEFORM_NONE || s1 == CACB200_DEFORM_VOLUME) invalid();
      d.substyle = DeformDim::TWO_FROM_ONE, d.fixed = o2, d.dynamic1 = o1;
    } else {
      d.substyle = DeformDim::ONE_FROM_TWO, d.dynamic1 = o1, d.dynamic2 = o2;
    }
  }
  P.on = true;
  c.dfm = P;
  c.dfm_rep.assign(c.nrep, DeformRep{});
  c.gen++;
}

void deform_unset(Ctx &c) {
  if (c.dfm.on) c.gen++;
  c.dfm.on = false;
}

// FixDeform::init for a run of nsteps from the current step
// (fix_deform.cpp:417-487): start box = the current box, stop box per style.
void deform_begin(Ctx &c, long nsteps, double dt) {
  if (!c.dfm.on) return;
  c.dfm.begin = c.step;
  c.dfm.end = c.step + nsteps;
  const double delt = (double)(c.dfm.end - c.dfm.begin) * dt;
  for (int r = 0; r < c.nrep; r++) {
    const BoxD &B = c.rep_h[r].b;
    DeformRep &R = c.dfm_rep[r];
    const double vol = B.L[0] * B.L[1] * B.L[2];
    for (int i = 0; i < 3; i++) {
      const DeformDim &d = c.dfm.dim[i];
      double &lo_start = R.lo_start[i], &hi_start = R.hi_start[i], &lo_stop = R.lo_stop[i], &hi_stop = R.hi_stop[i];
      lo_start = B.lo[i];
      hi_start = B.hi[i];
      R.vol_start[i] = vol;
      lo_stop = lo_start;
      hi_stop = hi_start;
      switch (d.style) {
        case CACB200_DEFORM_FINAL:
          lo_stop = d.a;
          hi_stop = d.b;
          break;
        case CACB200_DEFORM_DELTA:
          lo_stop = lo_start + d.a;
          hi_stop = hi_start + d.b;
          break;
        case CACB200_DEFORM_SCALE:
          lo_stop = 0.5 * (lo_start + hi_start) - 0.5 * d.a * (hi_start - lo_start);
          hi_stop = 0.5 * (lo_start + hi_start) + 0.5 * d.a * (hi_start - lo_start);
          break;
        case CACB200_DEFORM_VEL:
          lo_stop = lo_start - 0.5 * delt * d.a;
          hi_stop = hi_start + 0.5 * delt * d.a;
          break;
        case CACB200_DEFORM_ERATE:
          lo_stop = lo_start - 0.5 * delt * d.a * (hi_start - lo_start);
          hi_stop = hi_start + 0.5 * delt * d.a * (hi_start - lo_start);
          if (hi_stop <= lo_stop) throw Error(CACB200_EINVAL, "Final box dimension due to fix deform is < 0.0");
          break;
        case CACB200_DEFORM_TRATE:
          lo_stop = 0.5 * (lo_start + hi_start) - 0.5 * ((hi_start - lo_start) * std::exp(d.a * delt));
          hi_stop = 0.5 * (lo_start + hi_start) + 0.5 * ((hi_start - lo_start) * std::exp(d.a * delt));
          break;
        case CACB200_DEFORM_WIGGLE:
          lo_stop = lo_start - 0.5 * d.a * std::sin(MY_2PI * delt / d.b);
          hi_stop = hi_start + 0.5 * d.a * std::sin(MY_2PI * delt / d.b);
          break;
        default:
          break;
      }
    }
  }
}

void box_changed(Ctx &c);

// FixDeform::end_of_step on the steps it applies to (Modify::end_of_step,
// modify.cpp:910-915): new targets, remap, new box.
void deform_end_of_step(Ctx &c, double dt) {
  if (!c.dfm.on || c.step % c.dfm.nevery != 0) return;
  double delta = (double)(c.step - c.dfm.begin);
  if (delta != 0.0) delta /= (double)(c.dfm.end - c.dfm.begin);
  const double delt = (double)(c.step - c.dfm.begin) * dt;
  std::vector<Remap> maps(c.nrep);
  for (int r = 0; r < c.nrep; r++) {
    BoxD &B = c.rep_h[r].b;
    DeformRep &R = c.dfm_rep[r];
    double lo_t[3], hi_t[3];
    // apply_strain (fix_deform.cpp:1020-1097)
    for (int i = 0; i < 3; i++) {
      const DeformDim &d = c.dfm.dim[i];
      switch (d.style) {
        case CACB200_DEFORM_NONE:
          lo_t[i] = B.lo[i];
          hi_t[i] = B.hi[i];
          break;
        case CACB200_DEFORM_TRATE: {
          double shift = 0.5 * ((R.hi_start[i] - R.lo_start[i]) * std::exp(d.a * delt));
          lo_t[i] = 0.5 * (R.lo_start[i] + R.hi_start[i]) - shift;
          hi_t[i] = 0.5 * (R.lo_start[i] + R.hi_start[i]) + shift;
          break;
        }
        case CACB200_DEFORM_WIGGLE: {
          double shift = 0.5 * d.a * std::sin(MY_2PI * delt / d.b);
          lo_t[i] = R.lo_start[i] - shift;
          hi_t[i] = R.hi_start[i] + shift;
          break;
        }
        case CACB200_DEFORM_VOLUME:
          break;
        default:
          lo_t[i] = R.lo_start[i] + delta * (R.lo_stop[i] - R.lo_start[i]);
          hi_t[i] = R.hi_start[i] + delta * (R.hi_stop[i] - R.hi_start[i]);
          break;
      }
    }
    // apply_volume (fix_deform.cpp:1101-1127), dimensions in order
    for (int i = 0; i < 3; i++) {
      const DeformDim &d = c.dfm.dim[i];
      if (d.style != CACB200_DEFORM_VOLUME) continue;
      const double v0 = R.vol_start[i];
      double shift = 0.0;
      if (d.substyle == DeformDim::ONE_FROM_ONE) {
        shift = 0.5 * (v0 / (hi_t[d.dynamic1] - lo_t[d.dynamic1]) / (R.hi_start[d.fixed] - R.lo_start[d.fixed]));
      } else if (d.substyle == DeformDim::ONE_FROM_TWO) {
        shift = 0.5 * (v0 / (hi_t[d.dynamic1] - lo_t[d.dynamic1]) / (hi_t[d.dynamic2] - lo_t[d.dynamic2]));
      } else {
        shift = 0.5 * std::sqrt(v0 * (R.hi_start[i] - R.lo_start[i]) / (hi_t[d.dynamic1] - lo_t[d.dynamic1]) /
                                (R.hi_start[d.fixed] - R.lo_start[d.fixed]));
      }
      lo_t[i] = 0.5 * (R.lo_start[i] + R.hi_start[i]) - shift;
      hi_t[i] = 0.5 * (R.lo_start[i] + R.hi_start[i]) + shift;
    }
    // update_domain (fix_deform.cpp:1129-1240): old box for x2lamda, then
    // the new box (Domain::set_global_box, domain.cpp:227-238)
    Remap &M = maps[r];
    for (int i = 0; i < 3; i++) {
      M.lo0[i] = B.lo[i];
      M.hinv0[i] = 1.0 / B.L[i];
      if (c.dfm.dim[i].style != CACB200_DEFORM_NONE) {
        B.lo[i] = lo_t[i];
        B.hi[i] = hi_t[i];
      }
      B.L[i] = B.hi[i] - B.lo[i];
      if (!(B.L[i] > 0.0)) throw Error(CACB200_EINVAL, "fix deform made a box dimension non-positive");
      M.lo1[i] = B.lo[i];
      M.h1[i] = B.L[i];
    }
  }
  if (c.dfm.remap_x && (c.na || c.ne)) {
    const Remap *many = nullptr;
    if (c.nrep > 1) {
      static_assert(sizeof(Remap) == 12 * sizeof(double), "Remap is 12 doubles");
      c.dfm_maps.reserve(12 * (size_t)c.nrep);
      CACB200_CUDA(cudaMemcpyAsync(c.dfm_maps.p, maps.data(), sizeof(Remap) * c.nrep, cudaMemcpyHostToDevice,
                                   c.stream));
      many = reinterpret_cast<const Remap *>(c.dfm_maps.p);
    }
    k_deform_remap<<<stride_grid((long)c.na + 8L * c.ne, 256), 256, 0, c.stream>>>(
        c.xs.p, c.na, c.nodex.p, c.ne, maps[0], many, c.nrep > 1 ? c.site_rep.p : nullptr,
        c.nrep > 1 ? c.elem_rep.p : nullptr);
    CACB200_CUDA(cudaGetLastError());
  }
  // energies tallied this step stay (the reference's thermo output after
  // end_of_step reports them with the new volume)
  box_changed(c);
}

// The replica boxes in rep_h changed: the fixed-point box lengths, the
// context box, the device descriptors; grids and reference bins are replanned
// at the next rebuild, read-outs see the new volume, and a run starts from
// forces of the new box.
void box_changed(Ctx &c) {
  for (Rep &P : c.rep_h)
    for (int i = 0; i < 3; i++) P.Lq[i] = (int)(uint32_t)(uint64_t)std::llrint(P.b.L[i] * P.qscale[i]);
  for (int i = 0; i < 3; i++) {
    c.boxlo[i] = c.rep_h[0].b.lo[i];
    c.boxhi[i] = c.rep_h[0].b.hi[i];
    c.prd[i] = c.rep_h[0].b.L[i];
  }
  if (c.rep_d.p && c.rep_d.n >= (size_t)c.nrep)
    CACB200_CUDA(cudaMemcpyAsync(c.rep_d.p, c.rep_h.data(), sizeof(Rep) * c.nrep, cudaMemcpyHostToDevice, c.stream));
  c.planned = false;
  c.box_replan = true;
  c.thermo_gen = -1;
  c.forces_current = false;
  inner_off(c);   // distances changed by more than the sites' own motion
}

// A new box for a single system without moving its sites (the box a host
// loop has just changed, e.g. the reference's own fix deform; the positions
// follow with the next set_state).
void set_box(Ctx &c, const double *lo, const double *hi) {
  c.check_system();
  if (c.nrep != 1) throw Error(CACB200_ESTATE, "a batch has one box per replica");
  if (!lo || !hi) throw Error(CACB200_EINVAL, "box required");
  BoxD &B = c.rep_h[0].b;
  for (int i = 0; i < 3; i++)
    if (!(hi[i] > lo[i])) throw Error(CACB200_EINVAL, "empty box");
  bool same = true;
  for (int i = 0; i < 3; i++) same = same && B.lo[i] == lo[i] && B.hi[i] == hi[i];
  if (same) return;
  for (int i = 0; i < 3; i++) {
    B.lo[i] = lo[i];
    B.hi[i] = hi[i];
    B.L[i] = hi[i] - lo[i];
  }
  box_changed(c);
}

}  // namespace cacb200
