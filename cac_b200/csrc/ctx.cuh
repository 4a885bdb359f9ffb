// Internal state of a cacb200 context: device buffers, parameters and helpers.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/cacb200.h"

namespace cacb200 {

constexpr int NC = 9;           // lattice sites per element edge
constexpr int NU = NC * NC * NC;  // lattice sites per element (729)
constexpr int NPE = 8;          // nodes per element
constexpr int NG = 8;           // Gauss points per element (the nodes)
constexpr int IMG_BITS = 5;     // periodic image code 0..26 in the low bits of a list entry
constexpr int IMG_ZERO = 13;    // image (0, 0, 0)

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define CACB200_CUDA(call)                                                             \
  do {                                                                                 \
    cudaError_t err_ = (call);                                                         \
    if (err_ != cudaSuccess)                                                           \
      throw ::cacb200::Error(CACB200_ECUDA, std::string(#call) + ": " +                \
                                                cudaGetErrorString(err_));             \
  } while (0)

// Simple owning device buffer.
template <class T>
struct DBuf {
  T *p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  // grow to at least m elements (contents not preserved)
  void reserve(size_t m) {
    if (m <= n && p) return;
    release();
    size_t bytes = (m ? m : 1) * sizeof(T);
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
      cudaGetLastError();
      throw Error(CACB200_ENOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed");
    }
    n = m ? m : 1;
  }
};

// Atom bins of the reference (NBinStandard::setup_bins, nbin_standard.cpp:84-128):
// used only for the half-list storage rule.
struct RefBins {
  double lo[3], hi[3], inv[3];
  int nbin[3];
};

// Uniform periodic cell grid over wrapped coordinates (candidate search).
struct Grid {
  int nc[3];
  double inv[3];   // 1 / cell size
  int ncell;
};

// Orthogonal periodic box.
struct BoxD {
  double lo[3], hi[3], L[3];
};

// One replica of a batch (a single system is a batch of one): its box, its
// two candidate grids and where their cells start in the batch-wide cell
// numbering, and the element radius its grids were planned for.
struct Rep {
  BoxD b;
  Grid ag, eg;
  int abase, ebase;
  double reach_budget;
  float fmargin;      // bound on the error of FP32 separations in this box (A)
  double qscale[3];   // mixed form: fixed-point scale 2^k per dimension ...
  float qinv[3];      // ... and 2^-k
  int Lq[3];          // rint(L 2^k)
};

struct PairParams {
  int style = CACB200_PAIR_NONE;
  double cut = 0.0;          // force cutoff
  // LJ
  double lj1 = 0, lj2 = 0, lj3 = 0, lj4 = 0, offset = 0;
  // EAM
  int nrho = 0, nr = 0;
  double drho = 0, dr = 0, rdr = 0, rdrho = 0, rhomax = 0;
};

// FIRE parameters (Min defaults, min.cpp:33-47) and run settings
struct FireParams {
  int delaystep = 20;
  double dtgrow = 1.1, dtshrink = 0.5, alpha0 = 0.25, alphashrink = 0.99;
  double tmax = 10.0, tmin = 0.02, dmax = 0.1;
  int halfstepback = 1, delaystep_start = 1, max_vdotf_negatif = 2000;
  double etol = 0.0, ftol = 0.0;
  int maxiter = 1000, normstyle = 0;  // 0 two-norm squared, 1 max per-site |f|^2, 2 inf (max component)^2
  double dtmax = 0.0, dtmin = 0.0, mass = 1.0;
};

// FIRE iteration state, kept in device memory and advanced by the control kernel
struct FireState {
  double dt, alpha, dtv, halfback, s1, s2, vdotf, ecur, eprev, fnorm;
  long long step, last_negative, start;
  int vdotf_neg, reset, mix, apply, status, iter;
};

// fix langevin parameters (FixLangevin, fix_langevin.cpp:40-214), CONSTANT style
struct LangevinParams {
  bool on = false;
  double t_start = 0, t_stop = 0, t_period = 1;
  int seed = 0;
  bool zero = false;
};

// fix deform, orthogonal box (FixDeform, fix_deform.cpp:40-372): per
// dimension a style with its arguments (box units) and, for volume, the
// dimensions it is linked to
struct DeformDim {
  enum { ONE_FROM_ONE, ONE_FROM_TWO, TWO_FROM_ONE };
  int style = CACB200_DEFORM_NONE;
  double a = 0, b = 0;
  int substyle = 0, fixed = 0, dynamic1 = 0, dynamic2 = 0;
};
struct DeformParams {
  bool on = false;
  int nevery = 1;
  bool remap_x = true;
  DeformDim dim[3];
  long begin = 0, end = 0;   // the current run's first and last step
};
// per replica: the run's start and stop boxes (FixDeform::Set)
struct DeformRep {
  double lo_start[3], hi_start[3], lo_stop[3], hi_stop[3], vol_start[3];
};

struct Profile {
  bool enabled = false;
  std::vector<std::string> names;
  std::vector<double> ms;
  std::vector<int64_t> launches;
};

struct Ctx {
  int device = 0;
  int num_sms = 148;             // multiprocessors of the device (persistent launches)
  cudaStream_t stream = nullptr;
  // second stream for work that overlaps inside one stage (the Gauss-point
  // list build beside the atom list build), forked from and joined back to
  // `stream` with events, so it is part of the same order and of graphs
  cudaStream_t side = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr, items_ev = nullptr;
  cudaStream_t copy = nullptr;   // host copies overlapped with the last step's forces
  cudaEvent_t pos_ev = nullptr;
  std::string last_error;
  int precision = CACB200_FP64;

  // system (a batch of nrep independent replicas, stored one after another:
  // replica r owns atoms [rep_aoff[r], +rep_na[r]) and elements
  // [rep_eoff[r], +rep_ne[r]); boxlo/boxhi/prd are replica 0's box)
  int na = 0, ne = 0;
  int nrep = 1;
  std::vector<int> rep_na, rep_ne, rep_aoff, rep_eoff;
  std::vector<Rep> rep_h;        // descriptors as last planned
  DBuf<Rep> rep_d;
  DBuf<int> site_rep;            // [nsite_i] replica of each i-site (batches only)
  DBuf<int> elem_rep;            // [ne] replica of each element (batches only)
  DBuf<int> acell_rep;           // [atom cells] replica of each atom cell (batches only)
  DBuf<unsigned long long> reach_bits;   // [nrep] element reach (double bits)
  double boxlo[3] = {0, 0, 0}, boxhi[3] = {0, 0, 0}, prd[3] = {0, 0, 0};
  double mass = 1.0;
  bool have_system = false;

  // sites table S: [atoms | Gauss points (8 per element) | active lattice sites]
  // xs[k] = (x, y, z, w) with w = F'(rho) for EAM
  DBuf<double4> xs;
  int nact = 0;                  // active non-Gauss lattice sites (host copy, valid if nact_known)
  bool nact_known = true;
  DBuf<int> dev_nact;            // device count written by each rebuild
  size_t ns_cap = 0;             // site-table capacity (every lattice site active)
  DBuf<int> act_gid;             // [nact] e*729 + u
  DBuf<int> act_off;             // [ne+1] CSR of active sites by element (into act_gid)
  int nsite_i() const { return na + NG * ne; }

  DBuf<double> v, f;             // atoms [na*3]
  DBuf<double> stage;            // [na*3] host-transfer staging for positions
  DBuf<double> stage_nodes;      // [ne*24] the same for node positions
  DBuf<int> state_changed;       // set_state: did any position change
  DBuf<double4> snap_x;          // device snapshot of the state (cacb200_snapshot)
  DBuf<double> snap_v, snap_nodex, snap_nodev;
  bool have_snapshot = false;
  DBuf<double> nodex, nodev, nodef, gaussf;  // [ne*8*3]
  DBuf<double> rho;              // [na + 8*ne]: atoms then nodes (node order)
  DBuf<double> phi_site;         // [nsite_i] embedding energy F(rho) per i-site (EAM, eflag)
  // energy / virial
  DBuf<double> eatom, vatom, enode, vnode;   // per-site outputs
  DBuf<double> partial;          // per-block partial sums [nblocks*7]
  DBuf<double> ev_out;           // [7]: energy, virial[6]
  double energy = 0.0, virial[6] = {0, 0, 0, 0, 0, 0};
  bool have_peratom_e = false, have_peratom_v = false;
  bool ev_pending = false;       // ev_out holds a result not yet copied to energy/virial
  // step of the last evaluation that tallied the global energy / virial and
  // the per-site energy / virial (-1: none since the system was set)
  long tally_step_e = -1, tally_step_v = -1, tally_step_ae = -1, tally_step_av = -1;
  long step = 0, last_build_step = 0;
  double nodal_energy_weight = -1.0;

  // element geometry (per rebuild)
  DBuf<double4> ecenter;         // reference centre (x, y, z, R_e)
  DBuf<double4> ewrap;           // wrapped centre, w = bitcast of packed wrap counts
  DBuf<double> eframe;           // [ne*28]: element frame (layout at k_elem_geom, neigh.cu)
  double emax_reach = 0.0;

  // atom cell grid (candidate search)
  Grid agrid{}, egrid{};
  DBuf<int> acell_start;         // [ncell+1]
  DBuf<int> acell_atoms;         // [na] atom ids sorted by cell
  DBuf<double4> acell_pos;       // [na] wrapped positions sorted by cell, w = bitcast(id)
  DBuf<float4> acell_pos32;      // [na] the same as floats, w = bitcast(int id)
  DBuf<int> acell_of;            // [na] cell of each sorted atom
  DBuf<int> ecell_start, ecell_elems;
  DBuf<int> cell_key, cell_key2, idx_tmp;
  DBuf<int> atom_work, atom_nwork;   // atoms with element sites in reach (rebuild work list)
  DBuf<int2> items;                  // [slots][item_cap] element boxes to test, per query
  DBuf<int> nitems;                  // [slots]
  int item_cap = 48;
  // list slot -> atom (atoms sorted by cell at the last rebuild; slots past
  // the atoms are Gauss points in site-table order).  Lists, counts and the
  // pair kernels' threads are indexed by slot, so a warp covers a compact
  // group of atoms.
  DBuf<int> slot_atom;
  DBuf<int> atom_slot;           // atom -> list slot
  // pair table: the site table in list-slot order, [atoms by slot | Gauss
  // points | active lattice sites], refreshed each step before the pair
  // kernels; list entries index it, so the neighbours a warp gathers lie in
  // few cache lines.  w = F' for EAM.
  DBuf<double4> xss;
  DBuf<unsigned char> cub_tmp;
  size_t cub_bytes = 0;
  int sort_bits_a = 1, sort_bits_e = 1;
  double reach_budget = 0.0;
  bool planned = false, plan_half = false;
  int plan_na = -1, plan_ne = -1;
  RefBins rbins{};

  // neighbour lists: transposed [cap][nsite_i] packed entries (sidx << 5 | img)
  double skin = 1.0, cutneigh = 0.0, cutneighsq = 0.0;
  int every = 10;
  int delay = 0;                 // neigh_modify delay: no rebuild before this many steps
  int dist_check = 0;            // neigh_modify check yes: a due rebuild only after a move > trigger
  std::vector<double> build_box; // [nrep*6] replica boxes (lo, hi) at the last build
  DBuf<int> moved;               // flag of the displacement check
  int cap = 160;
  // full lists, [cap][nsite_i]: a site's num_in entries within cut +
  // inner_margin at the build fill rows [0, num_in) and its other
  // num_full - num_in entries rows [cap - (num_full - num_in), cap); the two
  // segments meet only when a list overflows (then the build is repeated)
  DBuf<int> nbr_full, num_full;
  DBuf<int2> site_from;
  DBuf<unsigned char> ecell_near;   // single systems: element cells with an element in their 27-cell block
  DBuf<unsigned char> acell_near;   // single systems: atom cells with an atom in their 27-cell block
  // inner prefix of the full lists (entries within cutoff + inner_margin at
  // the build, rows [0, num_in)).  inner_ok[replica] (device) is nonzero
  // until positions move other than by the drift (then every site walks its
  // whole list until the next build); while it is set, the drift keeps each
  // site's displacement since the build (xbuild / nodex_build): disp per
  // atom, edisp per element (its largest node displacement, which bounds
  // every lattice site of the element), dmax per replica (the largest of
  // all, as float bits), and a site walks the rest of its list only when
  // its displacement plus dmax could close the margin (PrefixRule)
  double inner_margin = 0.5;
  double inner_margin_set = -1.0;   // cacb200_set_list_prefix (< 0: 0.5 x skin)
  DBuf<int> num_in, inner_ok;
  DBuf<float> disp, edisp;
  DBuf<unsigned> dmax;
  DBuf<double4> xbuild;
  DBuf<double> nodex_build;
  DBuf<int> nbr_half, num_half;
  bool have_half = false, lists_valid = false;
  DBuf<int> raw_full, raw_half;  // build-time element-site entries (full) and half lists before compaction
  DBuf<unsigned char> img_full, img_half;
  DBuf<int> site_flag;           // [ne*729 + 1] marks
  DBuf<int> site_pref;           // [ne*729 + 1] exclusive prefix of the marks
  DBuf<int> overflow;            // [16] device flags (see neigh_check)
  int build_count = 0;

  PairParams pp;
  DBuf<double4> rhor_val, rhor_der, z2r_val, z2r_der, frho_val, frho_der;
  // per r-knot m: [2m] rhor value coefficients, [2m+1] z2r value coefficients
  // (one 64-byte record read by a pair; derivatives follow from them)
  DBuf<double4> rz;
  // mixed precision: FP32 tables, per-site FP32 offsets and packed anchor cells
  DBuf<float4> frho_val32, frho_der32;
  DBuf<float4> rz32;              // the same r-knot records in FP32 (32 bytes)
  bool have_mixed_tables = false;
  DBuf<int4> pos32;              // mixed form: fixed-point site records (qx, qy, qz, F' bits)

  FireParams fire;
  DBuf<FireState> fire_state;
  DBuf<double> fire_partial;

  Profile prof;

  // CUDA graphs of the NVE cycle: [half-kick + drift, rebuild] then [forces,
  // half-kick, every-1 more steps]; valid while `gen` (bumped by anything
  // that moves buffers or changes baked-in parameters), dt and every match
  long gen = 0;
  bool graphs_enabled = true;
  cudaGraphExec_t g_build = nullptr, g_steps = nullptr;
  long graph_gen = -1;
  double graph_dt = 0.0;
  int graph_every = 0;
  long graph_launches = 0;
  // block sizes of the force-only pair passes, chosen by timing (valid for
  // tune_gen == gen); FP64 and mixed forms
  long tune_gen = -1, tune_gen32 = -1;
  int tb_rho = 128, tb_force = 128, tb_rho32 = 128, tb_force32 = 128;
  // batches, mixed form: persistent work-queue launches of the EAM passes.
  // Items are runs of consecutive list slots of one replica, the largest
  // replicas first; the run length (tile) is chosen per replica size class
  // (i-sites < 8192, < 32768, larger) by timing when the plan changes.
  bool work_queue = true;
  DBuf<int2> work_items;
  DBuf<int> work_counter;
  DBuf<int> sm_counter;   // single systems: run counters of the SM-local ranges (rho, force)
  int nwork_items = 0;
  long work_gen = -1;
  int work_tile[3] = {0, 0, 0};
  double escale_node_last = 0.0;   // node energy scale of the last evaluation
  DBuf<int> rep_meta;              // [4][nrep] aoff, na, eoff, ne (per-replica energy)
  DBuf<double> rep_energy;         // [nrep]
  // thermo read-outs: per-replica offsets and volumes (valid for thermo_gen == gen),
  // block partial sums and results
  long thermo_gen = -1;
  // fix langevin: per-replica random streams (window of the last 97 values
  // and the 96 after it, draws made), the run's step counter, chunk layout
  // and jump coefficients
  LangevinParams lgv;
  DBuf<unsigned> lgv_base, lgv_next, lgv_poly;
  DBuf<unsigned long long> lgv_m;
  DBuf<long long> lgv_ctl;
  DBuf<int2> lgv_chunks, lgv_rchunk;
  DBuf<int4> lgv_meta;
  DBuf<double> lgv_part, lgv_mean, lgv_save;
  int lgv_nchunks = 0, lgv_poly_n = 0;
  // fix deform: parameters, per-replica start/stop boxes, device remap table
  DeformParams dfm;
  std::vector<DeformRep> dfm_rep;
  DBuf<double> dfm_maps;
  bool box_replan = false;        // the next plan follows a box change only
  bool forces_current = false;    // f / nodef are the pair forces of the current positions and box
  long run_left = 0;              // steps left in the run begun by run_begin
  DBuf<int4> thermo_meta;
  DBuf<double> thermo_vol, thermo_part, thermo_out;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;

  Ctx(int dev);
  ~Ctx();
  void check_system() const {
    if (!have_system) throw Error(CACB200_ESTATE, "no system uploaded");
  }
};

// Largest displacement since the build for which the inner prefix still
// holds every pair inside the cutoff: half the margin, less an allowance for
// the FP32 screen of the build's classification.
inline double inner_limit(const Ctx &c) { return 0.5 * (c.inner_margin - 1e-3); }

// The per-site prefix rule as the pair kernels see it.  A pair (i, j) kept
// out of the prefix was at least cutoff + margin apart at the build (less
// the FP32 screen's allowance), so it is still outside the cutoff while
// disp_i + disp_j <= margin less that allowance; disp_j <= dmax.  Site i
// (site-table index) walks its whole list when its replica's flag is clear
// or disp_i + dmax exceeds lim.
struct PrefixRule {
  const int *inner_ok;
  const float *disp, *edisp;
  const unsigned *dmax;
  float lim;
  int na;
};

inline PrefixRule prefix_rule(const Ctx &c) {
  PrefixRule r;
  r.inner_ok = c.inner_ok.p;
  r.disp = c.disp.p;
  r.edisp = c.edisp.p;
  r.dmax = c.dmax.p;
  // twice the per-site allowance of inner_limit, rounded down
  r.lim = std::nextafter((float)(c.inner_margin - 2e-3), 0.0f);
  r.na = c.na;
  return r;
}

// Positions moved by something other than the checked drift: the pair loops
// use the whole lists until the next build.
inline void inner_off(Ctx &c) {
  if (c.inner_ok.p) cudaMemsetAsync(c.inner_ok.p, 0, sizeof(int) * c.inner_ok.n, c.stream);
}

// Host<->device copy ordered on the context's stream and completed on return.
// (The legacy default stream does not order against the context's non-blocking
// stream, so every transfer goes through the stream.)
inline void stream_copy(Ctx &c, void *dst, const void *src, size_t bytes, cudaMemcpyKind kind) {
  if (bytes == 0) return;
  CACB200_CUDA(cudaMemcpyAsync(dst, src, bytes, kind, c.stream));
  CACB200_CUDA(cudaStreamSynchronize(c.stream));
}

// profiling helpers (host)
struct KernelTimer {
  Ctx &c;
  const char *name;
  KernelTimer(Ctx &ctx, const char *n);
  ~KernelTimer();
};

// The replica boxes the lists are built in (the trigger of the displacement
// check shrinks by the box corners' movement since then).
inline void note_build_box(Ctx &c) {
  c.build_box.resize(6 * (size_t)c.rep_h.size());
  for (size_t r = 0; r < c.rep_h.size(); r++)
    for (int d = 0; d < 3; d++) {
      c.build_box[6 * r + d] = c.rep_h[r].b.lo[d];
      c.build_box[6 * r + 3 + d] = c.rep_h[r].b.hi[d];
    }
}

// stages implemented in the .cu files
void neigh_build(Ctx &c, bool want_half);
void neigh_plan(Ctx &c, bool want_half);
void neigh_build_async(Ctx &c, bool want_half);
int neigh_check(Ctx &c);
int device_nact(Ctx &c);
void neigh_download(Ctx &c, bool half, int64_t *offset, int8_t *kind, int32_t *idx, int32_t *site,
                    int8_t *img, int64_t *nentries);
void interpolate_sites(Ctx &c);
void pair_compute(Ctx &c, int eflag, int vflag);
void pair_compute_mixed(Ctx &c, int eflag, int vflag);
// the mixed form's pair table as fixed-point records (interpolate_sites)
void pair_table_mixed(Ctx &c);
void assemble_nodef(Ctx &c);
// prekick: first the previous step's second half-kick (nve_final) on the
// same forces, in the same operations (one pass over the state for both)
void nve_initial(Ctx &c, double dt, bool prekick = false);
bool moved_past_trigger(Ctx &c);
void nve_final(Ctx &c, double dt);
void eam_tables(Ctx &c, const double *frho, const double *rhor, const double *z2r);
void fire_init(Ctx &c, double dt);
void fire_step(Ctx &c);
FireState fire_read(Ctx &c);
void thermo(Ctx &c, int units, double *out);
void langevin_set(Ctx &c, double t_start, double t_stop, double t_period, int seed, int zero);
void langevin_unset(Ctx &c);
void langevin_stream(Ctx &c, long long draws);
void langevin_begin(Ctx &c, long nsteps);
void langevin_post_force(Ctx &c, double dt);
void deform_set(Ctx &c, int nevery, const int *style, const double *a, const double *b, int remap_x);
void deform_unset(Ctx &c);
void deform_begin(Ctx &c, long nsteps, double dt);
void deform_end_of_step(Ctx &c, double dt);
void set_box(Ctx &c, const double *lo, const double *hi);

}  // namespace cacb200
