// Context lifetime, host<->device transfer and the extern "C" entry points.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ctx.cuh"
#include "device.cuh"

struct cacb200_ctx {
  cacb200::Ctx *impl;
};

namespace cacb200 {

namespace {

struct PendingTimer {
  std::string name;
  cudaEvent_t a, b;
};

void flush_profile(Ctx &c, std::vector<PendingTimer> &pend) {
  if (pend.empty()) return;
  cudaStreamSynchronize(c.stream);
  for (auto &p : pend) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, p.a, p.b);
    size_t k = 0;
    for (; k < c.prof.names.size(); k++)
      if (c.prof.names[k] == p.name) break;
    if (k == c.prof.names.size()) {
      c.prof.names.push_back(p.name);
      c.prof.ms.push_back(0.0);
      c.prof.launches.push_back(0);
    }
    c.prof.ms[k] += ms;
    c.prof.launches[k] += 1;
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  pend.clear();
}

std::vector<PendingTimer> &pending_for(Ctx &c) {
  static thread_local std::vector<std::pair<Ctx *, std::vector<PendingTimer>>> table;
  for (auto &t : table)
    if (t.first == &c) return t.second;
  table.emplace_back(&c, std::vector<PendingTimer>());
  return table.back().second;
}

}  // namespace

Ctx::Ctx(int dev) : device(dev) {
  CACB200_CUDA(cudaSetDevice(dev));
  CACB200_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  CACB200_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
  CACB200_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
  CACB200_CUDA(cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming));
  CACB200_CUDA(cudaEventCreateWithFlags(&join_ev, cudaEventDisableTiming));
  CACB200_CUDA(cudaEventCreateWithFlags(&items_ev, cudaEventDisableTiming));
  CACB200_CUDA(cudaStreamCreateWithFlags(&copy, cudaStreamNonBlocking));
  CACB200_CUDA(cudaEventCreateWithFlags(&pos_ev, cudaEventDisableTiming));
}

Ctx::~Ctx() {
  if (g_build) cudaGraphExecDestroy(g_build);
  if (g_steps) cudaGraphExecDestroy(g_steps);
  if (side) {
    cudaStreamSynchronize(side);
    cudaStreamDestroy(side);
  }
  if (fork_ev) cudaEventDestroy(fork_ev);
  if (join_ev) cudaEventDestroy(join_ev);
  if (items_ev) cudaEventDestroy(items_ev);
  if (copy) {
    cudaStreamSynchronize(copy);
    cudaStreamDestroy(copy);
  }
  if (pos_ev) cudaEventDestroy(pos_ev);
  if (stream) {
    cudaStreamSynchronize(stream);
    auto &pend = pending_for(*this);
    flush_profile(*this, pend);
    cudaStreamDestroy(stream);
  }
}

KernelTimer::KernelTimer(Ctx &ctx, const char *n) : c(ctx), name(n) {
  if (!c.prof.enabled) return;
  PendingTimer p{name, nullptr, nullptr};
  cudaEventCreate(&p.a);
  cudaEventCreate(&p.b);
  cudaEventRecord(p.a, c.stream);
  pending_for(c).push_back(p);
}

KernelTimer::~KernelTimer() {
  if (!c.prof.enabled) return;
  auto &pend = pending_for(c);
  if (!pend.empty()) cudaEventRecord(pend.back().b, c.stream);
  if (pend.size() > 4096) flush_profile(c, pend);
}

namespace {

// A system of nrep independent replicas stored one after another (a single
// system is nrep = 1).  Each replica has its own periodic box; atoms and
// elements keep the order of the input arrays.
// Energies and virials tallied before the positions changed no longer
// describe the system.
void forget_tallies(Ctx &c) { c.tally_step_e = c.tally_step_v = c.tally_step_ae = c.tally_step_av = -1; }

void upload_system(Ctx &c, int nrep, const int *rna, const int *rne, const double *lo, const double *hi,
                   const double *x, const double *v, const double *nodex, const double *nodev, double mass) {
  if (nrep < 1 || !rna || !rne || !lo || !hi) throw Error(CACB200_EINVAL, "invalid replica description");
  long na_l = 0, ne_l = 0;
  for (int r = 0; r < nrep; r++) {
    if (rna[r] < 0 || rne[r] < 0) throw Error(CACB200_EINVAL, "negative atom or element count");
    na_l += rna[r];
    ne_l += rne[r];
    for (int d = 0; d < 3; d++)
      if (!(hi[3 * r + d] > lo[3 * r + d])) throw Error(CACB200_EINVAL, "empty box");
  }
  // list entries pack a site index in 26 bits: atoms and Gauss points must
  // fit (referenced lattice sites are checked at each rebuild), and element
  // lattice-site ids e * 729 + u must fit in 30 bits during the build
  if (na_l + (long)NG * ne_l >= (1L << 26) || ne_l * NU >= (1L << 30))
    throw Error(CACB200_EINVAL, "system too large for 26-bit site indices");
  const int na = (int)na_l, ne = (int)ne_l;
  if ((na > 0 && (!x || !v)) || (ne > 0 && (!nodex || !nodev)))
    throw Error(CACB200_EINVAL, "invalid system arrays");
  if (!(mass > 0.0)) throw Error(CACB200_EINVAL, "mass must be positive");
  for (int d = 0; d < 3; d++) {
    c.boxlo[d] = lo[d];
    c.boxhi[d] = hi[d];
    c.prd[d] = hi[d] - lo[d];
  }
  c.nrep = nrep;
  c.rep_na.assign(rna, rna + nrep);
  c.rep_ne.assign(rne, rne + nrep);
  c.rep_aoff.assign(nrep, 0);
  c.rep_eoff.assign(nrep, 0);
  c.rep_h.assign(nrep, Rep{});
  for (int r = 0; r < nrep; r++) {
    if (r) {
      c.rep_aoff[r] = c.rep_aoff[r - 1] + rna[r - 1];
      c.rep_eoff[r] = c.rep_eoff[r - 1] + rne[r - 1];
    }
    for (int d = 0; d < 3; d++) {
      c.rep_h[r].b.lo[d] = lo[3 * r + d];
      c.rep_h[r].b.hi[d] = hi[3 * r + d];
      c.rep_h[r].b.L[d] = hi[3 * r + d] - lo[3 * r + d];
    }
  }
  c.na = na;
  c.ne = ne;
  c.mass = mass;
  c.nact = 0;
  c.nact_known = true;
  c.lists_valid = false;
  c.have_half = false;
  c.planned = false;
  c.gen++;
  c.step = c.last_build_step = 0;
  forget_tallies(c);
  c.forces_current = false;
  c.lgv.on = false;   // a thermostat or deformation is set for the system it acts on
  c.dfm.on = false;
  c.box_replan = false;
  // site table at full capacity (kept across uploads while large enough): atoms, Gauss points and every lattice site
  size_t ns = (size_t)na + NG * (size_t)ne + (size_t)ne * NU;
  c.xs.reserve(ns);
  c.dev_nact.reserve(1);
  CACB200_CUDA(cudaMemsetAsync(c.dev_nact.p, 0, sizeof(int), c.stream));
  c.v.reserve(std::max(3 * na, 1));
  c.f.reserve(std::max(3 * na, 1));
  c.nodex.reserve(std::max(24 * ne, 1));
  c.nodev.reserve(std::max(24 * ne, 1));
  c.nodef.reserve(std::max(24 * ne, 1));
  c.gaussf.reserve(std::max(24 * ne, 1));
  CACB200_CUDA(cudaMemsetAsync(c.f.p, 0, sizeof(double) * std::max(3 * na, 1), c.stream));
  CACB200_CUDA(cudaMemsetAsync(c.nodef.p, 0, sizeof(double) * std::max(24 * ne, 1), c.stream));
  CACB200_CUDA(cudaMemsetAsync(c.gaussf.p, 0, sizeof(double) * std::max(24 * ne, 1), c.stream));
  CACB200_CUDA(cudaMemsetAsync(c.xs.p, 0, sizeof(double4) * c.xs.n, c.stream));
  c.have_system = true;
  // replica of every i-site and element (batches)
  if (nrep > 1) {
    std::vector<int> sr(std::max(na + NG * ne, 1)), er(std::max(ne, 1));
    for (int r = 0; r < nrep; r++) {
      for (int i = 0; i < rna[r]; i++) sr[c.rep_aoff[r] + i] = r;
      for (int e = 0; e < rne[r]; e++) {
        int eg = c.rep_eoff[r] + e;
        er[eg] = r;
        for (int g = 0; g < NG; g++) sr[na + NG * eg + g] = r;
      }
    }
    c.site_rep.reserve(sr.size());
    c.elem_rep.reserve(er.size());
    stream_copy(c, c.site_rep.p, sr.data(), sizeof(int) * sr.size(), cudaMemcpyHostToDevice);
    stream_copy(c, c.elem_rep.p, er.data(), sizeof(int) * er.size(), cudaMemcpyHostToDevice);
  }
  // positions/velocities
  std::vector<double4> hx(std::max(na, 1));
  for (int i = 0; i < na; i++) hx[i] = make_double4(x[3 * i], x[3 * i + 1], x[3 * i + 2], 0.0);
  if (na) {
    stream_copy(c, c.xs.p, hx.data(), sizeof(double4) * na, cudaMemcpyHostToDevice);
    stream_copy(c, c.v.p, v, sizeof(double) * 3 * na, cudaMemcpyHostToDevice);
  }
  if (ne) {
    stream_copy(c, c.nodex.p, nodex, sizeof(double) * 24 * ne, cudaMemcpyHostToDevice);
    stream_copy(c, c.nodev.p, nodev, sizeof(double) * 24 * ne, cudaMemcpyHostToDevice);
  }
  CACB200_CUDA(cudaStreamSynchronize(c.stream));
}

// Energy of each replica from the per-site energies of the last evaluation:
// atoms count their own, node Gauss points theirs times the node weight (the
// global sum's split, per replica).  One block per replica, fixed order.
__global__ void k_replica_energy(const double *eatom, const double *enode, const int *aoff, const int *rna,
                                 const int *eoff, const int *rne, double node_scale, double *out) {
  int r = blockIdx.x;
  double s = 0.0;
  for (int i = threadIdx.x; i < rna[r]; i += blockDim.x) s += eatom[aoff[r] + i];
  double t = 0.0;
  for (int k = threadIdx.x; k < 8 * rne[r]; k += blockDim.x) t += enode[8 * (size_t)eoff[r] + k];
  double v[1] = {s + node_scale * t};
  block_reduce_store<1>(v, out);
}

__device__ __forceinline__ bool same_bits(double a, double b) {
  return __double_as_longlong(a) == __double_as_longlong(b);
}

// New positions into the site table; *changed is set when any differs
// from the one it replaces (bit for bit).
__global__ void k_pack_x(const double *x, double4 *xs, int n, int *changed) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double4 p = xs[i];
  const double a = x[3 * i], b = x[3 * i + 1], d = x[3 * i + 2];
  if (!same_bits(p.x, a) || !same_bits(p.y, b) || !same_bits(p.z, d)) atomicOr(changed, 1);
  p.x = a;
  p.y = b;
  p.z = d;
  xs[i] = p;
}

__global__ void k_copy_cmp(const double *src, double *dst, long n, int *changed) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double v = src[i];
  if (!same_bits(dst[i], v)) atomicOr(changed, 1);
  dst[i] = v;
}

__global__ void k_unpack_x(const double4 *xs, double *x, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double4 p = xs[i];
  x[3 * i] = p.x;
  x[3 * i + 1] = p.y;
  x[3 * i + 2] = p.z;
}

// Positions and velocities from host arrays.  Lists are kept, as the
// reference keeps them between rebuilds while forward communication moves the
// ghosts; rebuild when atoms moved further than half the skin.
void set_state(Ctx &c, const double *x, const double *v, const double *nodex, const double *nodev) {
  c.check_system();
  const bool moves = (x && c.na) || (nodex && c.ne);
  if (moves) {
    c.state_changed.reserve(1);
    CACB200_CUDA(cudaMemsetAsync(c.state_changed.p, 0, sizeof(int), c.stream));
  }
  if (x && c.na) {
    c.stage.reserve(3 * (size_t)c.na);
    CACB200_CUDA(cudaMemcpyAsync(c.stage.p, x, sizeof(double) * 3 * c.na, cudaMemcpyHostToDevice, c.stream));
    k_pack_x<<<(c.na + 255) / 256, 256, 0, c.stream>>>(c.stage.p, c.xs.p, c.na, c.state_changed.p);
  }
  if (v && c.na)
    CACB200_CUDA(cudaMemcpyAsync(c.v.p, v, sizeof(double) * 3 * c.na, cudaMemcpyHostToDevice, c.stream));
  if (nodex && c.ne) {
    const long n = 24L * c.ne;
    c.stage_nodes.reserve(n);
    CACB200_CUDA(cudaMemcpyAsync(c.stage_nodes.p, nodex, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream));
    k_copy_cmp<<<(int)((n + 255) / 256), 256, 0, c.stream>>>(c.stage_nodes.p, c.nodex.p, n, c.state_changed.p);
  }
  if (nodev && c.ne)
    CACB200_CUDA(cudaMemcpyAsync(c.nodev.p, nodev, sizeof(double) * 24 * c.ne, cudaMemcpyHostToDevice, c.stream));
  CACB200_CUDA(cudaGetLastError());
  CACB200_CUDA(cudaStreamSynchronize(c.stream));
  if (moves) {
    // positions written back unchanged keep the forces and tallies they had
    int changed = 1;
    stream_copy(c, &changed, c.state_changed.p, sizeof(int), cudaMemcpyDeviceToHost);
    if (changed) {
      forget_tallies(c);
      c.forces_current = false;
      inner_off(c);
    }
  }
}

void get_state(Ctx &c, double *x, double *v, double *nodex, double *nodev) {
  c.check_system();
  if (x && c.na) {
    c.stage.reserve(3 * (size_t)c.na);
    k_unpack_x<<<(c.na + 255) / 256, 256, 0, c.stream>>>(c.xs.p, c.stage.p, c.na);
    CACB200_CUDA(cudaMemcpyAsync(x, c.stage.p, sizeof(double) * 3 * c.na, cudaMemcpyDeviceToHost, c.stream));
  }
  if (v && c.na)
    CACB200_CUDA(cudaMemcpyAsync(v, c.v.p, sizeof(double) * 3 * c.na, cudaMemcpyDeviceToHost, c.stream));
  if (nodex && c.ne)
    CACB200_CUDA(cudaMemcpyAsync(nodex, c.nodex.p, sizeof(double) * 24 * c.ne, cudaMemcpyDeviceToHost, c.stream));
  if (nodev && c.ne)
    CACB200_CUDA(cudaMemcpyAsync(nodev, c.nodev.p, sizeof(double) * 24 * c.ne, cudaMemcpyDeviceToHost, c.stream));
  CACB200_CUDA(cudaStreamSynchronize(c.stream));
}

void snapshot(Ctx &c) {
  c.check_system();
  size_t na = std::max(c.na, 1), ne = std::max(c.ne, 1);
  c.snap_x.reserve(na);
  c.snap_v.reserve(3 * na);
  c.snap_nodex.reserve(24 * ne);
  c.snap_nodev.reserve(24 * ne);
  auto d2d = [&](void *dst, const void *src, size_t bytes) {
    if (bytes) CACB200_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, c.stream));
  };
  d2d(c.snap_x.p, c.xs.p, sizeof(double4) * c.na);
  d2d(c.snap_v.p, c.v.p, sizeof(double) * 3 * c.na);
  d2d(c.snap_nodex.p, c.nodex.p, sizeof(double) * 24 * c.ne);
  d2d(c.snap_nodev.p, c.nodev.p, sizeof(double) * 24 * c.ne);
  c.have_snapshot = true;
}

void restore(Ctx &c) {
  c.check_system();
  if (!c.have_snapshot) throw Error(CACB200_ESTATE, "no snapshot taken");
  auto d2d = [&](void *dst, const void *src, size_t bytes) {
    if (bytes) CACB200_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, c.stream));
  };
  d2d(c.xs.p, c.snap_x.p, sizeof(double4) * c.na);
  d2d(c.v.p, c.snap_v.p, sizeof(double) * 3 * c.na);
  d2d(c.nodex.p, c.snap_nodex.p, sizeof(double) * 24 * c.ne);
  d2d(c.nodev.p, c.snap_nodev.p, sizeof(double) * 24 * c.ne);
  c.lists_valid = false;
  c.forces_current = false;
  inner_off(c);
  forget_tallies(c);
}

void fetch_ev(Ctx &c) {
  if (!c.ev_pending) return;
  double h[7];
  CACB200_CUDA(cudaMemcpyAsync(h, c.ev_out.p, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
  CACB200_CUDA(cudaStreamSynchronize(c.stream));
  c.energy = h[0];
  for (int k = 0; k < 6; k++) c.virial[k] = h[1 + k];
  c.ev_pending = false;
}

void build(Ctx &c, bool want_half) {
  neigh_build(c, want_half);
  interpolate_sites(c);
  c.last_build_step = c.step;
}

// Neighbor::decide (neighbor.cpp:1584-1604): a rebuild is due when at least
// `delay` steps have passed since the last one and their count is a multiple
// of `every`; with check yes it happens only when a site has moved past the
// trigger (otherwise the next one is due `every` steps later).
bool rebuild_due(Ctx &c) {
  const long ago = c.step - c.last_build_step;
  if (c.every <= 0 || ago < c.delay || ago % c.every != 0) return false;
  return !c.dist_check || moved_past_trigger(c);
}

void forces(Ctx &c, int eflag, int vflag) {
  interpolate_sites(c);
  pair_compute(c, eflag, vflag);
  assemble_nodef(c);
  c.forces_current = true;
}

void setup(Ctx &c) {
  c.check_system();
  build(c, false);
  forces(c, CACB200_ENERGY_GLOBAL, CACB200_VIRIAL_GLOBAL);
}

void drop_graphs(Ctx &c) {
  if (c.g_build) cudaGraphExecDestroy(c.g_build);
  if (c.g_steps) cudaGraphExecDestroy(c.g_steps);
  c.g_build = c.g_steps = nullptr;
  c.graph_gen = -1;
}

// Record what `body` queues on the context stream as an executable graph.
template <class F>
cudaGraphExec_t capture(Ctx &c, F &&body) {
  cudaGraph_t g = nullptr;
  CACB200_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeRelaxed));
  try {
    body();
  } catch (...) {
    cudaStreamEndCapture(c.stream, &g);
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    throw;
  }
  CACB200_CUDA(cudaStreamEndCapture(c.stream, &g));
  cudaGraphExec_t x = nullptr;
  cudaError_t e = cudaGraphInstantiate(&x, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) throw Error(CACB200_ECUDA, std::string("graph instantiation: ") + cudaGetErrorString(e));
  return x;
}

// One rebuild cycle of `every` velocity-Verlet steps from two graph launches:
// [half-kick + drift of the rebuild step, list rebuild], a check of the
// rebuild's flag words (the one host wait of the cycle; an overflow is
// repaired by a synchronous rebuild before any force uses the lists), then
// [forces and second half-kick of that step, the every-1 steps that follow].
void nve_cycle(Ctx &c, double dt) {
  const int every = c.every;
  if (c.graph_gen != c.gen || c.graph_dt != dt || c.graph_every != every || !c.g_build || !c.g_steps) {
    drop_graphs(c);
    // one eager evaluation first, so that every buffer and table the force
    // path grows on first use exists before capture (it recomputes the
    // forces of the current positions: the state does not change; forces
    // that hold a thermostat's last draws are kept aside and put back)
    const size_t n3 = 3 * (size_t)c.na, n24 = 24 * (size_t)c.ne;
    if (c.lgv.on) {
      c.lgv_save.reserve(n3 + n24 + 1);
      if (n3) CACB200_CUDA(cudaMemcpyAsync(c.lgv_save.p, c.f.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, c.stream));
      if (n24)
        CACB200_CUDA(cudaMemcpyAsync(c.lgv_save.p + n3, c.nodef.p, sizeof(double) * n24, cudaMemcpyDeviceToDevice,
                                     c.stream));
    }
    forces(c, 0, 0);
    if (c.lgv.on) {
      if (n3) CACB200_CUDA(cudaMemcpyAsync(c.f.p, c.lgv_save.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, c.stream));
      if (n24)
        CACB200_CUDA(cudaMemcpyAsync(c.nodef.p, c.lgv_save.p + n3, sizeof(double) * n24, cudaMemcpyDeviceToDevice,
                                     c.stream));
    }
    c.g_build = capture(c, [&] {
      nve_initial(c, dt);
      neigh_build_async(c, false);
    });
    // between two steps of the cycle nothing reads the velocities, so each
    // step's second half-kick runs inside the next step's drift kernel
    c.g_steps = capture(c, [&] {
      forces(c, 0, 0);
      langevin_post_force(c, dt);
      for (int k = 1; k < every; k++) {
        nve_initial(c, dt, true);
        forces(c, 0, 0);
        langevin_post_force(c, dt);
      }
      nve_final(c, dt);
    });
    c.graph_gen = c.gen;
    c.graph_dt = dt;
    c.graph_every = every;
  }
  CACB200_CUDA(cudaGraphLaunch(c.g_build, c.stream));
  c.graph_launches++;
  c.step++;
  c.lists_valid = true;
  c.nact_known = false;
  if (neigh_check(c)) neigh_build(c, false);   // plan grew: rebuild once more, synchronously
  note_build_box(c);
  c.last_build_step = c.step;
  if (c.graph_gen == c.gen) {
    CACB200_CUDA(cudaGraphLaunch(c.g_steps, c.stream));
    c.graph_launches++;
  } else {
    forces(c, 0, 0);
    langevin_post_force(c, dt);
    nve_final(c, dt);
    for (int k = 1; k < every; k++) {
      nve_initial(c, dt);
      forces(c, 0, 0);
      langevin_post_force(c, dt);
      nve_final(c, dt);
    }
  }
  c.step += every - 1;
}

// Verlet::setup for a run of nsteps (verlet.cpp:64-190): the forces of the
// positions the run starts from (evaluated again only when they are not
// current or when the requested tallies are missing), the thermostat's setup
// draws, the deformation's start and stop boxes.  eflag / vflag: tallies of
// the setup evaluation (the reference tallies them for its step-0 output).
void run_begin(Ctx &c, long nsteps, double dt, int eflag, int vflag) {
  c.check_system();
  if (nsteps < 0) throw Error(CACB200_EINVAL, "negative step count");
  const bool need_tally = ((eflag & CACB200_ENERGY_GLOBAL) && c.tally_step_e != c.step) ||
                          ((vflag & CACB200_VIRIAL_GLOBAL) && c.tally_step_v != c.step) ||
                          ((eflag & CACB200_ENERGY_ATOM) && c.tally_step_ae != c.step) ||
                          ((vflag & CACB200_VIRIAL_ATOM) && c.tally_step_av != c.step);
  if (!c.lists_valid) {
    setup(c);   // lists, then forces with the global tallies
    if ((eflag & CACB200_ENERGY_ATOM) || (vflag & CACB200_VIRIAL_ATOM)) forces(c, eflag, vflag);
  } else if (c.lgv.on || !c.forces_current || need_tally) {
    // forces of the positions the run starts from: they differ from the last
    // evaluation after a box change, new positions or a thermostat's draws
    forces(c, eflag, vflag);
  }
  if (c.lgv.on) {
    // the fixes' setup, which for fix langevin is its first post_force of the run
    langevin_begin(c, nsteps);
    langevin_post_force(c, dt);
  }
  deform_begin(c, nsteps, dt);
  c.run_left = nsteps;
}

// nsteps of the run begun by run_begin (Verlet::run, verlet.cpp:218-360);
// energy / virial tallied on the last of them when eflag / vflag are set.
void run_steps(Ctx &c, int nsteps, double dt, int eflag, int vflag) {
  c.check_system();
  if (nsteps < 0) throw Error(CACB200_EINVAL, "negative step count");
  if (nsteps > c.run_left) throw Error(CACB200_ESTATE, "more steps than the run begun has left");
  // a deforming box changes launch arguments every step, and the check of
  // check yes decides on the host: no graph replay for either (nor for a
  // delay that moves the rebuilds off the multiples of every)
  const bool graphs = c.graphs_enabled && c.every > 0 && !c.prof.enabled && !c.dfm.on && !c.dist_check &&
                      c.delay <= c.every;
  const bool want_ev = eflag || vflag;
  int s = 1;
  while (s <= nsteps) {
    int left = nsteps - s + 1;
    bool at_cycle = c.every > 0 && (c.step + 1 - c.last_build_step) % c.every == 0;
    if (graphs && at_cycle && (left > c.every || (left == c.every && !want_ev))) {
      nve_cycle(c, dt);
      s += c.every;
      continue;
    }
    nve_initial(c, dt);
    c.step++;
    if (rebuild_due(c)) build(c, false);
    bool last = (s == nsteps);
    forces(c, last ? eflag : 0, last ? vflag : 0);
    langevin_post_force(c, dt);
    nve_final(c, dt);
    deform_end_of_step(c, dt);
    s++;
  }
  c.run_left -= nsteps;
  CACB200_CUDA(cudaGetLastError());
}

void run_nve(Ctx &c, int nsteps, double dt, int eflag, int vflag) {
  run_begin(c, nsteps, dt, 0, 0);
  run_steps(c, nsteps, dt, eflag, vflag);
}

// A run from host state to host state: the state is copied in (as by
// set_state), nsteps are run, and the state is copied out.  The positions
// are final once the last step's drift and its list rebuild (which wraps
// them into the box) are done, so their copy to the host runs on a second
// stream while that step's forces are evaluated; the velocities follow its
// second half-kick.  (A deforming box remaps positions at the end of the
// step: then every copy waits for the step.)
void run_nve_host(Ctx &c, int nsteps, double dt, double *x, double *v, double *nodex, double *nodev) {
  c.check_system();
  if (nsteps < 0) throw Error(CACB200_EINVAL, "negative step count");
  set_state(c, x, v, nodex, nodev);
  run_begin(c, nsteps, dt, 0, 0);
  if (nsteps == 0) {
    get_state(c, x, v, nodex, nodev);
    return;
  }
  run_steps(c, nsteps - 1, dt, 0, 0);
  nve_initial(c, dt);
  c.step++;
  if (rebuild_due(c)) build(c, false);
  const bool overlap = !c.dfm.on;
  if (overlap) {
    CACB200_CUDA(cudaEventRecord(c.pos_ev, c.stream));
    CACB200_CUDA(cudaStreamWaitEvent(c.copy, c.pos_ev, 0));
    if (x && c.na) {
      c.stage.reserve(3 * (size_t)c.na);
      k_unpack_x<<<(c.na + 255) / 256, 256, 0, c.copy>>>(c.xs.p, c.stage.p, c.na);
      CACB200_CUDA(cudaMemcpyAsync(x, c.stage.p, sizeof(double) * 3 * c.na, cudaMemcpyDeviceToHost, c.copy));
    }
    if (nodex && c.ne)
      CACB200_CUDA(cudaMemcpyAsync(nodex, c.nodex.p, sizeof(double) * 24 * c.ne, cudaMemcpyDeviceToHost, c.copy));
  }
  forces(c, 0, 0);
  langevin_post_force(c, dt);
  nve_final(c, dt);
  deform_end_of_step(c, dt);
  c.run_left -= 1;
  CACB200_CUDA(cudaGetLastError());
  if (overlap) {
    if (v && c.na)
      CACB200_CUDA(cudaMemcpyAsync(v, c.v.p, sizeof(double) * 3 * c.na, cudaMemcpyDeviceToHost, c.stream));
    if (nodev && c.ne)
      CACB200_CUDA(cudaMemcpyAsync(nodev, c.nodev.p, sizeof(double) * 24 * c.ne, cudaMemcpyDeviceToHost,
                                   c.stream));
    CACB200_CUDA(cudaStreamSynchronize(c.copy));
    CACB200_CUDA(cudaStreamSynchronize(c.stream));
  } else {
    get_state(c, x, v, nodex, nodev);
  }
}

// Minimize::command + Min::setup/run with a FIRE iterate (minimize.cpp:21-70,
// min.cpp:182-463): nodal_energy_weight 1 for the duration (minimize.cpp:37),
// lists rebuilt every `every` iterations, energy evaluated every iteration.
void minimize_fire(Ctx &c, double etol, double ftol, int maxiter, double dt, int normstyle,
                   int *stop_code, int *niter, double *energy, double *fnorm) {
  c.check_system();
  if (maxiter < 0 || !(dt > 0.0) || normstyle < 0 || normstyle > 2)
    throw Error(CACB200_EINVAL, "invalid minimize arguments");
  double saved_w = c.nodal_energy_weight;
  c.nodal_energy_weight = 1.0;
  c.fire.etol = etol;
  c.fire.ftol = ftol;
  c.fire.maxiter = maxiter;
  c.fire.normstyle = normstyle;
  try {
    build(c, false);
    fire_init(c, dt);
    forces(c, CACB200_ENERGY_GLOBAL, 0);
    FireState s{};
    int done = 0;
    const int chunk = 25;
    while (true) {
      for (int k = 0; k < chunk; k++) {
        fire_step(c);
        done++;
        c.step++;
        if (rebuild_due(c)) build(c, false);
        forces(c, CACB200_ENERGY_GLOBAL, 0);
      }
      s = fire_read(c);
      if (s.status >= 0 || done > maxiter + chunk) break;
    }
    if (s.status < 0) s.status = 0;
    *stop_code = s.status;
    *niter = s.iter;
    *energy = s.ecur;
    *fnorm = s.fnorm;
  } catch (...) {
    c.nodal_energy_weight = saved_w;
    throw;
  }
  c.nodal_energy_weight = saved_w;
  fetch_ev(c);
}

}  // namespace
}  // namespace cacb200

using namespace cacb200;

#define API_BEGIN                                                \
  if (!ctx || !ctx->impl) return CACB200_EINVAL;                 \
  Ctx &c = *ctx->impl;                                           \
  try {
#define API_END                                                  \
  }                                                              \
  catch (const Error &e) {                                       \
    c.last_error = e.what();                                     \
    return e.code;                                               \
  }                                                              \
  catch (const std::exception &e) {                              \
    c.last_error = e.what();                                     \
    return CACB200_EINVAL;                                       \
  }                                                              \
  return CACB200_OK;

extern "C" {

int cacb200_ctx_create(int device, cacb200_ctx **out) {
  if (!out) return CACB200_EINVAL;
  *out = nullptr;
  try {
    auto *h = new cacb200_ctx;
    h->impl = new Ctx(device);
    *out = h;
  } catch (const Error &e) {
    std::fprintf(stderr, "cacb200_ctx_create: %s\n", e.what());
    return e.code;
  }
  return CACB200_OK;
}

int cacb200_ctx_destroy(cacb200_ctx *ctx) {
  if (!ctx) return CACB200_EINVAL;
  delete ctx->impl;
  delete ctx;
  return CACB200_OK;
}

const char *cacb200_last_error(const cacb200_ctx *ctx) {
  if (!ctx || !ctx->impl) return "invalid context";
  return ctx->impl->last_error.c_str();
}

void *cacb200_stream(cacb200_ctx *ctx) {
  if (!ctx || !ctx->impl) return nullptr;
  return (void *)ctx->impl->stream;
}

int cacb200_set_precision(cacb200_ctx *ctx, int form) {
  API_BEGIN
  if (form != CACB200_FP64 && form != CACB200_MIXED) throw Error(CACB200_EINVAL, "unknown precision form");
  c.precision = form;
  c.gen++;
  API_END
}

int cacb200_upload_system(cacb200_ctx *ctx, const double boxlo[3], const double boxhi[3], int natoms,
                          const double *x, const double *v, int nelements, const double *nodex,
                          const double *nodev, double mass) {
  API_BEGIN
  if (!boxlo || !boxhi) throw Error(CACB200_EINVAL, "box required");
  upload_system(c, 1, &natoms, &nelements, boxlo, boxhi, x, v, nodex, nodev, mass);
  API_END
}

int cacb200_upload_batch(cacb200_ctx *ctx, int nreplicas, const int *natoms, const int *nelements,
                         const double *boxlo, const double *boxhi, const double *x, const double *v,
                         const double *nodex, const double *nodev, double mass) {
  API_BEGIN
  upload_system(c, nreplicas, natoms, nelements, boxlo, boxhi, x, v, nodex, nodev, mass);
  API_END
}

int cacb200_replica_energy(cacb200_ctx *ctx, double *energy) {
  API_BEGIN
  c.check_system();
  if (!energy) throw Error(CACB200_EINVAL, "null output array");
  if (!c.have_peratom_e) throw Error(CACB200_ESTATE, "no per-site energies: evaluate with CACB200_ENERGY_ATOM");
  std::vector<int> meta(4 * (size_t)c.nrep);
  for (int r = 0; r < c.nrep; r++) {
    meta[r] = c.rep_aoff[r];
    meta[c.nrep + r] = c.rep_na[r];
    meta[2 * c.nrep + r] = c.rep_eoff[r];
    meta[3 * c.nrep + r] = c.rep_ne[r];
  }
  c.rep_meta.reserve(meta.size());
  c.rep_energy.reserve(c.nrep);
  stream_copy(c, c.rep_meta.p, meta.data(), sizeof(int) * meta.size(), cudaMemcpyHostToDevice);
  k_replica_energy<<<c.nrep, 256, 0, c.stream>>>(c.eatom.p, c.enode.p, c.rep_meta.p, c.rep_meta.p + c.nrep,
                                                 c.rep_meta.p + 2 * c.nrep, c.rep_meta.p + 3 * c.nrep,
                                                 2.0 * c.escale_node_last, c.rep_energy.p);
  CACB200_CUDA(cudaGetLastError());
  stream_copy(c, energy, c.rep_energy.p, sizeof(double) * c.nrep, cudaMemcpyDeviceToHost);
  API_END
}

int cacb200_thermo(cacb200_ctx *ctx, int units, double *out) {
  API_BEGIN
  thermo(c, units, out);
  API_END
}

int cacb200_set_langevin(cacb200_ctx *ctx, double t_start, double t_stop, double t_period, int seed, int zero) {
  API_BEGIN
  langevin_set(c, t_start, t_stop, t_period, seed, zero);
  API_END
}

int cacb200_set_langevin_stream(cacb200_ctx *ctx, long long draws) {
  API_BEGIN
  langevin_stream(c, draws);
  API_END
}

int cacb200_unset_langevin(cacb200_ctx *ctx) {
  API_BEGIN
  langevin_unset(c);
  API_END
}

int cacb200_set_deform(cacb200_ctx *ctx, int nevery, const int style[3], const double a[3], const double b[3],
                       int remap_x) {
  API_BEGIN
  deform_set(c, nevery, style, a, b, remap_x);
  API_END
}

int cacb200_set_box(cacb200_ctx *ctx, const double boxlo[3], const double boxhi[3]) {
  API_BEGIN
  set_box(c, boxlo, boxhi);
  API_END
}

int cacb200_unset_deform(cacb200_ctx *ctx) {
  API_BEGIN
  deform_unset(c);
  API_END
}

int cacb200_set_list_prefix(cacb200_ctx *ctx, double margin) {
  API_BEGIN
  c.inner_margin_set = margin;
  c.planned = false;
  c.lists_valid = false;
  API_END
}

int cacb200_set_graphs(cacb200_ctx *ctx, int enable) {
  API_BEGIN
  c.graphs_enabled = enable != 0;
  if (!c.graphs_enabled) drop_graphs(c);
  API_END
}

int cacb200_pair_blocks(cacb200_ctx *ctx, int *rho_threads, int *force_threads) {
  API_BEGIN
  const bool mixed = c.precision == CACB200_MIXED;
  if (rho_threads) *rho_threads = mixed ? c.tb_rho32 : c.tb_rho;
  if (force_threads) *force_threads = mixed ? c.tb_force32 : c.tb_force;
  API_END
}

int cacb200_work_queue(cacb200_ctx *ctx, int enable, int tiles[3]) {
  API_BEGIN
  if (enable >= 0) {
    c.work_queue = enable != 0;
    c.work_gen = -1;
  }
  if (tiles)
    for (int k = 0; k < 3; k++) tiles[k] = c.work_tile[k];
  API_END
}

int cacb200_graph_launches(cacb200_ctx *ctx, long long *count) {
  API_BEGIN
  if (count) *count = c.graph_launches;
  API_END
}

int cacb200_set_state(cacb200_ctx *ctx, const double *x, const double *v, const double *nodex,
                      const double *nodev) {
  API_BEGIN
  set_state(c, x, v, nodex, nodev);
  API_END
}

int cacb200_get_state(cacb200_ctx *ctx, double *x, double *v, double *nodex, double *nodev) {
  API_BEGIN
  get_state(c, x, v, nodex, nodev);
  API_END
}

int cacb200_get_forces(cacb200_ctx *ctx, double *f, double *nodef, double *gaussf) {
  API_BEGIN
  c.check_system();
  CACB200_CUDA(cudaStreamSynchronize(c.stream));
  if (f && c.na) stream_copy(c, f, c.f.p, sizeof(double) * 3 * c.na, cudaMemcpyDeviceToHost);
  if (nodef && c.ne)
    stream_copy(c, nodef, c.nodef.p, sizeof(double) * 24 * c.ne, cudaMemcpyDeviceToHost);
  if (gaussf && c.ne)
    stream_copy(c, gaussf, c.gaussf.p, sizeof(double) * 24 * c.ne, cudaMemcpyDeviceToHost);
  API_END
}

int cacb200_get_energy(cacb200_ctx *ctx, double *energy, double virial[6], double *eatom, double *vatom,
                       double *enode, double *vnode) {
  API_BEGIN
  c.check_system();
  fetch_ev(c);
  if (energy) *energy = c.energy;
  if (virial)
    for (int k = 0; k < 6; k++) virial[k] = c.virial[k];
  if ((eatom || enode) && !c.have_peratom_e) throw Error(CACB200_ESTATE, "per-site energy not computed");
  if ((vatom || vnode) && !c.have_peratom_v) throw Error(CACB200_ESTATE, "per-site virial not computed");
  if (eatom && c.na) stream_copy(c, eatom, c.eatom.p, sizeof(double) * c.na, cudaMemcpyDeviceToHost);
  if (enode && c.ne) stream_copy(c, enode, c.enode.p, sizeof(double) * 8 * c.ne, cudaMemcpyDeviceToHost);
  if (vatom && c.na)
    stream_copy(c, vatom, c.vatom.p, sizeof(double) * 6 * c.na, cudaMemcpyDeviceToHost);
  if (vnode && c.ne)
    stream_copy(c, vnode, c.vnode.p, sizeof(double) * 48 * c.ne, cudaMemcpyDeviceToHost);
  API_END
}

int cacb200_get_box(cacb200_ctx *ctx, double boxlo[3], double boxhi[3], double *mass) {
  API_BEGIN
  c.check_system();
  if (c.nrep != 1) throw Error(CACB200_ESTATE, "a batch has one box per replica");
  for (int d = 0; d < 3; d++) {
    if (boxlo) boxlo[d] = c.boxlo[d];
    if (boxhi) boxhi[d] = c.boxhi[d];
  }
  if (mass) *mass = c.mass;
  API_END
}

int cacb200_device_array(cacb200_ctx *ctx, int which, void **ptr, int64_t *count) {
  API_BEGIN
  c.check_system();
  if (!ptr || !count) throw Error(CACB200_EINVAL, "null output");
  const int64_t na = c.na, ne = c.ne;
  void *p = nullptr;
  int64_t n = 0;
  switch (which) {
    case CACB200_ARRAY_X: p = c.xs.p, n = 4 * na; break;
    case CACB200_ARRAY_V: p = c.v.p, n = 3 * na; break;
    case CACB200_ARRAY_F: p = c.f.p, n = 3 * na; break;
    case CACB200_ARRAY_NODEX: p = c.nodex.p, n = 24 * ne; break;
    case CACB200_ARRAY_NODEV: p = c.nodev.p, n = 24 * ne; break;
    case CACB200_ARRAY_NODEF: p = c.nodef.p, n = 24 * ne; break;
    case CACB200_ARRAY_EATOM:
    case CACB200_ARRAY_ENODE:
      if (!c.have_peratom_e) throw Error(CACB200_ESTATE, "per-site energy not computed");
      if (which == CACB200_ARRAY_EATOM) p = c.eatom.p, n = na;
      else p = c.enode.p, n = 8 * ne;
      break;
    case CACB200_ARRAY_VATOM:
    case CACB200_ARRAY_VNODE:
      if (!c.have_peratom_v) throw Error(CACB200_ESTATE, "per-site virial not computed");
      if (which == CACB200_ARRAY_VATOM) p = c.vatom.p, n = 6 * na;
      else p = c.vnode.p, n = 48 * ne;
      break;
    default:
      throw Error(CACB200_EINVAL, "unknown array");
  }
  *ptr = p;
  *count = n;
  API_END
}

int cacb200_counts(cacb200_ctx *ctx, int *natoms, int *nelements, int *nactive_sites) {
  API_BEGIN
  if (natoms) *natoms = c.na;
  if (nelements) *nelements = c.ne;
  if (nactive_sites) *nactive_sites = c.lists_valid ? device_nact(c) : 0;
  API_END
}

int cacb200_set_lj(cacb200_ctx *ctx, double epsilon, double sigma, double cut) {
  API_BEGIN
  if (!(cut > 0.0) || !(sigma > 0.0)) throw Error(CACB200_EINVAL, "invalid LJ parameters");
  // PairLJCut::init_one (pair_lj_cut.cpp:142-160), no offset (pair_modify shift no)
  c.pp = PairParams();
  c.pp.style = CACB200_PAIR_LJ;
  c.pp.cut = cut;
  c.pp.lj1 = 48.0 * epsilon * std::pow(sigma, 12.0);
  c.pp.lj2 = 24.0 * epsilon * std::pow(sigma, 6.0);
  c.pp.lj3 = 4.0 * epsilon * std::pow(sigma, 12.0);
  c.pp.lj4 = 4.0 * epsilon * std::pow(sigma, 6.0);
  c.pp.offset = 0.0;
  c.lists_valid = false;
  c.planned = false;
  c.gen++;
  API_END
}

int cacb200_set_eam(cacb200_ctx *ctx, int nrho, double drho, int nr, double dr, double cut,
                    const double *frho, const double *rhor, const double *z2r) {
  API_BEGIN
  if (nrho < 5 || nr < 5 || !(drho > 0) || !(dr > 0) || !(cut > 0) || !frho || !rhor || !z2r)
    throw Error(CACB200_EINVAL, "invalid EAM tables");
  c.pp = PairParams();
  c.pp.style = CACB200_PAIR_EAM;
  c.pp.cut = cut;
  c.pp.nrho = nrho;
  c.pp.nr = nr;
  c.pp.drho = drho;
  c.pp.dr = dr;
  c.pp.rdr = 1.0 / dr;
  c.pp.rdrho = 1.0 / drho;
  c.pp.rhomax = (nrho - 1) * drho;
  eam_tables(c, frho, rhor, z2r);
  c.lists_valid = false;
  c.planned = false;
  c.gen++;
  API_END
}

int cacb200_set_nodal_energy_weight(cacb200_ctx *ctx, double w) {
  API_BEGIN
  c.nodal_energy_weight = w;
  c.gen++;
  API_END
}

int cacb200_set_neighbor(cacb200_ctx *ctx, double skin, int every) {
  API_BEGIN
  if (!(skin >= 0.0) || every < 0) throw Error(CACB200_EINVAL, "invalid neighbour settings");
  c.skin = skin;
  c.every = every;
  c.lists_valid = false;
  c.planned = false;
  c.gen++;
  API_END
}

int cacb200_run_nve_host(cacb200_ctx *ctx, int nsteps, double dt, double *x, double *v, double *nodex,
                         double *nodev) {
  API_BEGIN
  run_nve_host(c, nsteps, dt, x, v, nodex, nodev);
  API_END
}

int cacb200_set_neighbor_modify(cacb200_ctx *ctx, int delay, int check) {
  API_BEGIN
  if (delay < 0 || (check != 0 && check != 1)) throw Error(CACB200_EINVAL, "invalid delay or check");
  c.delay = delay;
  c.dist_check = check;
  API_END
}

int cacb200_build_lists(cacb200_ctx *ctx, int want_half) {
  API_BEGIN
  build(c, want_half != 0);
  API_END
}

int cacb200_list_size(cacb200_ctx *ctx, int half, int64_t *nentries, int *nsites) {
  API_BEGIN
  int64_t n = 0;
  neigh_download(c, half != 0, nullptr, nullptr, nullptr, nullptr, nullptr, &n);
  if (nentries) *nentries = n;
  if (nsites) *nsites = c.nsite_i();
  API_END
}

int cacb200_get_list(cacb200_ctx *ctx, int half, int64_t *offset, int8_t *kind, int32_t *idx, int32_t *site,
                     int8_t *img) {
  API_BEGIN
  if (!offset || !kind || !idx || !site || !img) throw Error(CACB200_EINVAL, "null output array");
  int64_t n = 0;
  neigh_download(c, half != 0, offset, kind, idx, site, img, &n);
  API_END
}

int cacb200_interpolate(cacb200_ctx *ctx) {
  API_BEGIN
  c.check_system();
  interpolate_sites(c);
  API_END
}

int cacb200_compute_pair(cacb200_ctx *ctx, int eflag, int vflag) {
  API_BEGIN
  pair_compute(c, eflag, vflag);
  API_END
}

int cacb200_assemble_nodef(cacb200_ctx *ctx) {
  API_BEGIN
  c.check_system();
  assemble_nodef(c);
  API_END
}

int cacb200_compute_forces(cacb200_ctx *ctx, int eflag, int vflag) {
  API_BEGIN
  c.check_system();
  if (!c.lists_valid) build(c, false);
  forces(c, eflag, vflag);
  API_END
}

int cacb200_nve_initial(cacb200_ctx *ctx, double dt) {
  API_BEGIN
  c.check_system();
  nve_initial(c, dt);
  API_END
}

int cacb200_nve_final(cacb200_ctx *ctx, double dt) {
  API_BEGIN
  c.check_system();
  nve_final(c, dt);
  API_END
}

int cacb200_setup(cacb200_ctx *ctx) {
  API_BEGIN
  setup(c);
  API_END
}

int cacb200_run_begin(cacb200_ctx *ctx, int nsteps, double dt, int eflag, int vflag) {
  API_BEGIN
  run_begin(c, nsteps, dt, eflag, vflag);
  API_END
}

int cacb200_run_steps(cacb200_ctx *ctx, int nsteps, double dt, int eflag, int vflag) {
  API_BEGIN
  run_steps(c, nsteps, dt, eflag, vflag);
  API_END
}

int cacb200_run_nve(cacb200_ctx *ctx, int nsteps, double dt, int eflag, int vflag) {
  API_BEGIN
  run_nve(c, nsteps, dt, eflag, vflag);
  API_END
}

int cacb200_set_fire_params(cacb200_ctx *ctx, int delaystep, double dtgrow, double dtshrink, double alpha0,
                            double alphashrink, double tmax, double tmin, double dmax, int halfstepback,
                            int delaystep_start, int max_vdotf_negatif) {
  API_BEGIN
  if (delaystep < 0 || !(dtgrow >= 1.0) || !(dtshrink > 0.0 && dtshrink <= 1.0) || !(alpha0 >= 0.0) ||
      !(alphashrink > 0.0 && alphashrink <= 1.0) || !(tmax >= 1.0) || !(tmin > 0.0 && tmin <= 1.0) ||
      !(dmax > 0.0))
    throw Error(CACB200_EINVAL, "invalid FIRE parameters");
  c.fire.delaystep = delaystep;
  c.fire.dtgrow = dtgrow;
  c.fire.dtshrink = dtshrink;
  c.fire.alpha0 = alpha0;
  c.fire.alphashrink = alphashrink;
  c.fire.tmax = tmax;
  c.fire.tmin = tmin;
  c.fire.dmax = dmax;
  c.fire.halfstepback = halfstepback ? 1 : 0;
  c.fire.delaystep_start = delaystep_start ? 1 : 0;
  c.fire.max_vdotf_negatif = max_vdotf_negatif;
  API_END
}

int cacb200_minimize_fire(cacb200_ctx *ctx, double etol, double ftol, int maxiter, double dt, int normstyle,
                          int *stop_code, int *niter, double *energy, double *fnorm) {
  API_BEGIN
  if (!stop_code || !niter || !energy || !fnorm) throw Error(CACB200_EINVAL, "null output");
  minimize_fire(c, etol, ftol, maxiter, dt, normstyle, stop_code, niter, energy, fnorm);
  API_END
}

int cacb200_snapshot(cacb200_ctx *ctx) {
  API_BEGIN
  snapshot(c);
  API_END
}

int cacb200_restore(cacb200_ctx *ctx) {
  API_BEGIN
  restore(c);
  API_END
}

int cacb200_profile(cacb200_ctx *ctx, int enable) {
  API_BEGIN
  auto &pend = pending_for(c);
  flush_profile(c, pend);
  c.prof.enabled = enable != 0;
  c.prof.names.clear();
  c.prof.ms.clear();
  c.prof.launches.clear();
  API_END
}

int cacb200_profile_read(cacb200_ctx *ctx, int max, char *names, double *total_ms, int64_t *launches,
                         int *count) {
  API_BEGIN
  auto &pend = pending_for(c);
  flush_profile(c, pend);
  int n = (int)c.prof.names.size();
  if (count) *count = n;
  for (int k = 0; k < n && k < max; k++) {
    if (names) {
      std::memset(names + 32 * k, 0, 32);
      std::strncpy(names + 32 * k, c.prof.names[k].c_str(), 31);
    }
    if (total_ms) total_ms[k] = c.prof.ms[k];
    if (launches) launches[k] = c.prof.launches[k];
  }
  API_END
}

}  // extern "C"
