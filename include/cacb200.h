/*
 * cacb200: B200 (sm_100a) implementation of the CAC per-timestep force path
 * behind a C ABI.
 *
 * One context (cacb200_ctx) holds one system on one GPU: atoms, 8-node Hex
 * elements (apc = 1, 9 lattice sites per edge, 2x2x2 Gauss points = nodes),
 * a periodic orthogonal box, one pair style and the neighbour lists.  State is
 * device-resident; the host copies in and out only through the calls below.
 * All arrays are plain C arrays in the reference's own layouts:
 *   atom x, v, f         [natoms][3]                        (atom.h:36-60)
 *   node x, v, f          [nelements][8 nodes][3]            (element.h:94, apc = 1)
 *   gaussf                [nelements][8 Gauss points][3]
 * Atoms and elements keep the order in which they were uploaded; that order
 * plays the role of the reference's local index order (it decides the
 * "owned j after i" rule of the half list).
 *
 * Every call returns 0 on success or a negative CACB200_E* code; the message
 * is available from cacb200_last_error().  Nothing aborts the process; the
 * reference's styles turn a non-zero status into error->all().
 * A context is driven by one host thread at a time (it owns one stream).
 */
#ifndef CACB200_H
#define CACB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CACB200_OK 0
#define CACB200_EINVAL (-1)      /* bad argument */
#define CACB200_ECUDA (-2)       /* CUDA runtime error */
#define CACB200_ENOMEM (-3)      /* device allocation failed */
#define CACB200_ESTATE (-4)      /* call out of order (e.g. no system yet) */
#define CACB200_EOVERFLOW (-5)   /* a capacity was exceeded and could not grow */
#define CACB200_ETIMEDOUT (-6)   /* a bounded device wait gave up */
#define CACB200_EUNSTABLE (-7)   /* non-finite coordinates or forces */

/* precision forms */
#define CACB200_FP64 0           /* everything in FP64 */
#define CACB200_MIXED 1          /* FP32 pair arithmetic on cell-relative positions */

/* pair styles */
#define CACB200_PAIR_NONE 0
#define CACB200_PAIR_LJ 1
#define CACB200_PAIR_EAM 2

/* energy / virial request bits (force.h:11-20) */
#define CACB200_ENERGY_GLOBAL 1
#define CACB200_ENERGY_ATOM 2
#define CACB200_VIRIAL_GLOBAL 1
#define CACB200_VIRIAL_ATOM 4

typedef struct cacb200_ctx cacb200_ctx;

/* ---------------------------------------------------------------- context */

/* Create a context on CUDA device `device` (replaces the per-run state that
 * Atom/Element/Neighbor/Pair own in the reference, cac.cpp:36-197). */
int cacb200_ctx_create(int device, cacb200_ctx **out);
int cacb200_ctx_destroy(cacb200_ctx *ctx);
const char *cacb200_last_error(const cacb200_ctx *ctx);
/* cudaStream_t the context launches on, as void* */
void *cacb200_stream(cacb200_ctx *ctx);
int cacb200_set_precision(cacb200_ctx *ctx, int form);

/* ----------------------------------------------------------------- system */

/* Upload a system (replaces read_data + AtomVec/ElementVec data parsing,
 * read_data.cpp:339-367, element_vec_cac.cpp:300-395).  Element nodes must be
 * given unwrapped around their element centre; atoms inside the box. */
int cacb200_upload_system(cacb200_ctx *ctx, const double boxlo[3], const double boxhi[3],
                          int natoms, const double *x, const double *v,
                          int nelements, const double *nodex, const double *nodev,
                          double mass);
/* Upload a batch of independent replicas (no reference counterpart: the
 * reference runs one system per process; a batch replaces nreplicas separate
 * runs of the same pair style).  Replica r has natoms[r] atoms,
 * nelements[r] elements and its own periodic box boxlo/boxhi[3r..3r+2];
 * x, v, nodex, nodev concatenate the replicas in order.  Every other call
 * (state, forces, stepping, snapshots) then acts on all replicas at once,
 * arrays concatenated the same way.  Half lists are single-system only. */
int cacb200_upload_batch(cacb200_ctx *ctx, int nreplicas, const int *natoms,
                         const int *nelements, const double *boxlo, const double *boxhi,
                         const double *x, const double *v, const double *nodex,
                         const double *nodev, double mass);
/* Potential energy of each replica (or of the single system) from the last
 * evaluation made with CACB200_ENERGY_ATOM: per-atom energies plus node
 * energies times the node weight, i.e. eng_vdwl split by replica
 * (Pair::ev_tally, pair.cpp:428-482). */
int cacb200_replica_energy(cacb200_ctx *ctx, double *energy /* [nreplicas] */);

/* Thermo read-out reduced on the device, CACB200_THERMO_N doubles per replica
 * in the order below: thermo_style custom temp ke pe etotal press pxx pyy pzz
 * pxy pxz pyz vol with thermo_modify norm no (Thermo::compute_*,
 * thermo.cpp:1642-1936; ComputeTemp, compute_temp.cpp:74-243, CONSISTENT
 * element mass matrix; ComputePressure, compute_pressure.cpp:140-220).
 * Temperature, kinetic energy and volume always come from the current
 * velocities; PotEng and TotEng need the global energy, Press and the tensor
 * the global virial tallied at the current step (per-site energy / virial for
 * a batch).  A quantity not tallied at this step reads NaN, where the
 * reference stops with "Energy (Virial) was not tallied on needed timestep".
 * units: CACB200_UNITS_METAL (pressure in bar) or CACB200_UNITS_METALGPA
 * (GPa), the two pressure units of update.cpp:160-172. */
#define CACB200_UNITS_METAL 0
#define CACB200_UNITS_METALGPA 1
#define CACB200_THERMO_TEMP 0
#define CACB200_THERMO_KE 1
#define CACB200_THERMO_PE 2
#define CACB200_THERMO_ETOTAL 3
#define CACB200_THERMO_PRESS 4
#define CACB200_THERMO_PXX 5
#define CACB200_THERMO_PYY 6
#define CACB200_THERMO_PZZ 7
#define CACB200_THERMO_PXY 8
#define CACB200_THERMO_PXZ 9
#define CACB200_THERMO_PYZ 10
#define CACB200_THERMO_VOL 11
#define CACB200_THERMO_N 12
int cacb200_thermo(cacb200_ctx *ctx, int units, double *out /* [nreplicas][CACB200_THERMO_N] */);

/* Box and mass of a single system (not a batch). */
int cacb200_get_box(cacb200_ctx *ctx, double boxlo[3], double boxhi[3], double *mass);
/* A new periodic box for a single system, sites left where they are (the
 * device side of Domain::set_global_box after a host loop changed the box,
 * domain.cpp:227-238, e.g. the reference's own fix deform between list
 * rebuilds; new positions follow through cacb200_set_state).  Lists are kept;
 * the next rebuild plans its grids for the new box. */
int cacb200_set_box(cacb200_ctx *ctx, const double boxlo[3], const double boxhi[3]);

/* ------------------------------------------------------------- data files */

/* The reference's data-file format (ReadData::command, read_data.cpp:339-367,
 * and the element data parsers, element_vec_cac.cpp:300-470; written as by
 * write_data, element_vec_cac.cpp:1177-1300), restricted to the force path's
 * systems: one atom type, one Hex element type with one atom per cell, 9x9x9
 * lattice sites and 2x2x2 integration points; sections Masses, Element
 * Types, Atoms, Velocities, Elements, Nodes, Node Velocities.  Host-only
 * functions (no device needed) parse and write; cacb200_read_data uploads a
 * file into a context, cacb200_write_data writes a context's state.  Errors
 * return CACB200_EINVAL with the message in cacb200_data_last_error() (a
 * context's own calls report through cacb200_last_error). */
const char *cacb200_data_last_error(void);
int cacb200_data_counts(const char *path, int *natoms, int *nelements, double boxlo[3],
                        double boxhi[3], double *mass);
int cacb200_data_read(const char *path, double *x, double *v, double *nodex, double *nodev);
int cacb200_data_write(const char *path, int natoms, int nelements, const double boxlo[3],
                       const double boxhi[3], double mass, const double *x, const double *v,
                       const double *nodex, const double *nodev);
int cacb200_read_data(cacb200_ctx *ctx, const char *path);
int cacb200_write_data(cacb200_ctx *ctx, const char *path);

/* Overwrite positions/velocities of the current system (same counts; NULL
 * leaves an array unchanged).  Neighbour lists are kept, as the reference
 * keeps them between rebuilds; call cacb200_build_lists after moves larger
 * than half the skin. */
int cacb200_set_state(cacb200_ctx *ctx, const double *x, const double *v,
                      const double *nodex, const double *nodev);
int cacb200_get_state(cacb200_ctx *ctx, double *x, double *v, double *nodex, double *nodev);
/* Forces after the last force evaluation: atom f, nodal f (after assembly),
 * Gauss-point f (before assembly).  Any pointer may be NULL. */
int cacb200_get_forces(cacb200_ctx *ctx, double *f, double *nodef, double *gaussf);
/* Energy and virial of the last evaluation that requested them
 * (Pair::eng_vdwl, Pair::virial, eatom, vatom, enode, vnode). */
int cacb200_get_energy(cacb200_ctx *ctx, double *energy, double virial[6], double *eatom,
                       double *vatom, double *enode, double *vnode);
/* Device address of one of the context's arrays, for consumers on the same
 * GPU (analysis, dumps, another framework's tensors) that should not copy it
 * to the host: compute pe/atom is CACB200_ARRAY_EATOM / ENODE
 * (compute_pe_atom.cpp), compute stress/atom is -nktv2p times
 * CACB200_ARRAY_VATOM / VNODE (compute_stress_atom.cpp:112-330; this
 * reference adds no kinetic term).  *count is the number of doubles.
 * Layouts (atom and element order of the upload):
 *   X      [natoms][4]  x, y, z and a scratch word (positions in the site table)
 *   V, F   [natoms][3]
 *   NODEX, NODEV, NODEF  [nelements][8][3]
 *   EATOM  [natoms], ENODE [nelements][8]      (last evaluation with ENERGY_ATOM)
 *   VATOM  [natoms][6], VNODE [nelements][8][6] (last evaluation with VIRIAL_ATOM)
 * Per-site energies and virials are CACB200_ESTATE until an evaluation has
 * produced them.  The address stays valid until the next upload, list plan
 * or destroy; reads are ordered after the context's stream only once that
 * stream has been synchronised (cacb200_stream gives it). */
#define CACB200_ARRAY_X 0
#define CACB200_ARRAY_V 1
#define CACB200_ARRAY_F 2
#define CACB200_ARRAY_NODEX 3
#define CACB200_ARRAY_NODEV 4
#define CACB200_ARRAY_NODEF 5
#define CACB200_ARRAY_EATOM 6
#define CACB200_ARRAY_ENODE 7
#define CACB200_ARRAY_VATOM 8
#define CACB200_ARRAY_VNODE 9
int cacb200_device_array(cacb200_ctx *ctx, int which, void **ptr, int64_t *count);
int cacb200_counts(cacb200_ctx *ctx, int *natoms, int *nelements, int *nactive_sites);

/* ------------------------------------------------------------- pair styles */

/* pair_style lj/cut + pair_coeff 1 1 eps sigma (pair_lj_cut.cpp:142-215) */
int cacb200_set_lj(cacb200_ctx *ctx, double epsilon, double sigma, double cut);
/* pair_style eam/alloy with one element: the setfl arrays as read from the file
 * (pair_eam_alloy.cpp:100-240): frho[nrho], rhor[nr], z2r[nr] (= r*phi). */
int cacb200_set_eam(cacb200_ctx *ctx, int nrho, double drho, int nr, double dr, double cut,
                    const double *frho, const double *rhor, const double *z2r);
/* Pair::nodal_energy_weight (pair.cpp:38; minimize.cpp:37 sets 1.0): < 0 means
 * the element's nodal weight. */
int cacb200_set_nodal_energy_weight(cacb200_ctx *ctx, double w);

/* --------------------------------------------------------------- neighbour */

/* neighbor SKIN bin + neigh_modify every N delay 0 check no (neighbor.cpp:2043) */
int cacb200_set_neighbor(cacb200_ctx *ctx, double skin, int every);
/* neigh_modify delay D check yes|no (check 1|0; defaults 0 and 0, the
 * settings of cacb200_set_neighbor alone).  A rebuild is due when at least
 * `delay` steps have passed since the last one and their count is a multiple
 * of `every`; with check yes it then happens only when an atom or node has
 * moved more than half the skin since the last build, less the box corners'
 * movement while the box deforms, and otherwise the next one is due `every`
 * steps later (Neighbor::decide / check_distance, neighbor.cpp:1584-1683).
 * The reference's minimiser runs with every 1 delay 0 check yes (Min::init,
 * min.cpp:155-169).  Honoured by cacb200_run_nve / cacb200_run_steps (which
 * replay no graphs under check yes or a delay above every) and
 * cacb200_minimize_fire.  In a batch the rule is applied to the batch as a
 * whole: under check yes one replica that has moved past the trigger
 * rebuilds every replica (a rebuild also wraps positions into the box), and
 * under a deforming box the trigger is the smallest over the replicas, so a
 * batched replica's rebuild steps and wrapped coordinates can differ from
 * the same replica run alone; forces and unwrapped positions agree within
 * the FP64 tolerance.  The bit-for-bit batch-equals-alone property holds
 * under every/delay alone (check no). */
int cacb200_set_neighbor_modify(cacb200_ctx *ctx, int delay, int check);
/* The inner prefix of the lists (no reference counterpart; an evaluation
 * order, not a different result): entries within cutoff + margin at the
 * build are stored first, and a site's pair loop stops after them while its
 * own displacement since the build plus the largest displacement of its
 * system cannot close the margin (the velocity-Verlet drift records them;
 * other moves of the sites send every site to its whole list until the next
 * build, and a FIRE move that takes a site half the margin away does too);
 * every pair inside the cutoff is in the prefix in the same order, so forces
 * and energies are those of the whole lists bit for bit.  margin < 0: 0.5 x skin (default); 0: always the
 * whole lists.  Takes effect at the next list build. */
int cacb200_set_list_prefix(cacb200_ctx *ctx, double margin);
/* Bin and build the lists now (Neighbor::build, neighbor.cpp:1704-1876).
 * The full list (npair_full_bin.cpp) is always built; the half list
 * (npair_half_bin_newton.cpp) only when want_half is non-zero. */
int cacb200_build_lists(cacb200_ctx *ctx, int want_half);
/* Copy a list out in canonical form: per i-site (atoms, then Gauss points
 * natoms + 8*e + igcell) the neighbours (kind 0 atom / 1 lattice site, index,
 * site = -1 or jucell, periodic image sx sy sz).  Call with NULL arrays to get
 * the size; offset has nsites + 1 entries. */
int cacb200_list_size(cacb200_ctx *ctx, int half, int64_t *nentries, int *nsites);
int cacb200_get_list(cacb200_ctx *ctx, int half, int64_t *offset, int8_t *kind, int32_t *idx,
                     int32_t *site, int8_t *img);

/* ------------------------------------------------------------------ steps */

/* Refresh interpolated lattice-site positions (and EAM embedding terms)
 * from the current nodes: the implicit interpolation of
 * npair_half_bin_newton.cpp:284-289 / pair_lj_cut.cpp:364-368 done once. */
int cacb200_interpolate(cacb200_ctx *ctx);
/* Evaluate the pair style (Pair::compute(eflag, vflag)): atom f and gaussf. */
int cacb200_compute_pair(cacb200_ctx *ctx, int eflag, int vflag);
/* Element::compute_nodef, CONSISTENT (element.cpp:2178-2210) */
int cacb200_assemble_nodef(cacb200_ctx *ctx);
/* One force evaluation: interpolate + pair + nodal assembly. */
int cacb200_compute_forces(cacb200_ctx *ctx, int eflag, int vflag);
/* FixNVE::initial_integrate / final_integrate (fix_nve.cpp:62-219) */
int cacb200_nve_initial(cacb200_ctx *ctx, double dt);
int cacb200_nve_final(cacb200_ctx *ctx, double dt);
/* Verlet::setup + nsteps of Verlet::run with fix nve (verlet.cpp:64-360): lists
 * rebuilt every `every` steps (set_neighbor); energy/virial of the final step
 * when eflag/vflag are set.  Runs on the device; the call returns once every
 * step is queued on the context's stream (list rebuilds synchronise). */
int cacb200_setup(cacb200_ctx *ctx);
int cacb200_run_nve(cacb200_ctx *ctx, int nsteps, double dt, int eflag, int vflag);
/* A run from host arrays to host arrays, for a host loop that owns the state
 * between runs (the reference's x / v / nodex / nodev, atom.h:36-60,
 * element.h:94): x, v, nodex, nodev are read (cacb200_set_state), nsteps
 * are run as by cacb200_run_nve (no tallies), and the state is written back
 * into the same arrays (cacb200_get_state).  The positions' copy to the host
 * overlaps the last step's force evaluation (it needs nothing after the
 * drift and the list rebuild); use pinned host memory for copies that run
 * beside the kernels.  Null arrays are neither read nor written. */
int cacb200_run_nve_host(cacb200_ctx *ctx, int nsteps, double dt, double *x, double *v, double *nodex,
                         double *nodev);
/* cacb200_run_nve in two parts, so that a host can act between steps of one
 * run (e.g. print the reference's thermo lines): cacb200_run_begin is
 * Verlet::setup for a run of nsteps (forces of the starting positions, with
 * the tallies eflag / vflag for step-0 output; the thermostat's setup draws;
 * the deformation's start and stop boxes over nsteps), cacb200_run_steps
 * advances that run by some of its steps (tallies on the last of them).
 * cacb200_run_nve(n) = cacb200_run_begin(n, 0, 0) + cacb200_run_steps(n).
 * CACB200_ESTATE when more steps are asked than the run begun has left. */
int cacb200_run_begin(cacb200_ctx *ctx, int nsteps, double dt, int eflag, int vflag);
int cacb200_run_steps(cacb200_ctx *ctx, int nsteps, double dt, int eflag, int vflag);

/* fix ID all langevin t_start t_stop t_period seed [zero yes]
 * (FixLangevin, fix_langevin.cpp:40-214, 266-273, 455-694): drag plus random
 * force on atoms and element nodes (node noise scaled by 1/sqrt(nodal
 * weight)) after each force evaluation of cacb200_run_nve and at the start of
 * each run (the fix's setup), target temperature ramped from t_start to t_stop
 * over each run.  The random numbers are the reference's own RanMars stream
 * (random_mars.cpp:23-90) for `seed`, drawn in its order, so trajectories
 * follow the reference's; replica r of a batch uses seed + r.  The stream
 * starts at this call and continues across runs; a new system (upload) or
 * cacb200_unset_langevin removes the fix.  Snapshots do not rewind the
 * stream.  Not applied during minimisation (the reference's fix has no
 * min_post_force). */
int cacb200_set_langevin(cacb200_ctx *ctx, double t_start, double t_stop, double t_period, int seed,
                         int zero);
/* Position every replica's stream after `draws` uniform() calls of its
 * RanMars (the constructor's warm-up is draw 1; FixLangevin draws 3 per atom
 * and 24 per element each post_force), so that a run continues a stream the
 * reference's own loop has been drawing from (the fix langevin/b200 style). */
int cacb200_set_langevin_stream(cacb200_ctx *ctx, long long draws);
int cacb200_unset_langevin(cacb200_ctx *ctx);

/* fix ID all deform N x|y|z style args ... remap x|none units box on an
 * orthogonal periodic box (FixDeform, fix_deform.cpp:40-487, 698-707,
 * 1020-1240): every N-th step, after the second half-kick, each dimension's
 * box edges move to the style's target for that step of the run (run start
 * box -> stop box, per run as the reference's init does), and with remap x
 * the atoms and nodes follow affinely.  style[d] and its arguments a[d], b[d]
 * (box units):
 *   CACB200_DEFORM_NONE    unchanged
 *   CACB200_DEFORM_FINAL   a = lo, b = hi at the end of the run
 *   CACB200_DEFORM_DELTA   a = dlo, b = dhi added over the run
 *   CACB200_DEFORM_SCALE   a = factor about the centre
 *   CACB200_DEFORM_VEL     a = velocity of the length (distance/time)
 *   CACB200_DEFORM_ERATE   a = engineering strain rate (1/time)
 *   CACB200_DEFORM_TRATE   a = true strain rate (1/time)
 *   CACB200_DEFORM_WIGGLE  a = amplitude, b = period (time)
 *   CACB200_DEFORM_VOLUME  keeps the volume, linked to the other dimensions
 * Replicas of a batch deform alike, each from its own box.  Runs with a
 * deforming box queue their steps without graph replay; the neighbour grids
 * follow the box at each rebuild.  A new system or cacb200_unset_deform
 * removes the fix.  Tilt (triclinic) styles are not offered; the reference's
 * remap v moves neither positions nor velocities (its velocity terms in
 * Domain::remap are commented out, domain.cpp:566-633), so its decks pass
 * remap_x = 0. */
#define CACB200_DEFORM_NONE 0
#define CACB200_DEFORM_FINAL 1
#define CACB200_DEFORM_DELTA 2
#define CACB200_DEFORM_SCALE 3
#define CACB200_DEFORM_VEL 4
#define CACB200_DEFORM_ERATE 5
#define CACB200_DEFORM_TRATE 6
#define CACB200_DEFORM_WIGGLE 7
#define CACB200_DEFORM_VOLUME 8
int cacb200_set_deform(cacb200_ctx *ctx, int nevery, const int style[3], const double a[3],
                       const double b[3], int remap_x);
int cacb200_unset_deform(cacb200_ctx *ctx);

/* ------------------------------------------------------------- minimise */

/* min_modify for FIRE: the parameters of Min (min.h:61-72) with the
 * reference's defaults (min.cpp:33-47): delaystep 20, dtgrow 1.1,
 * dtshrink 0.5, alpha0 0.25, alphashrink 0.99, tmax 10, tmin 0.02, dmax 0.1,
 * halfstepback 1, delaystep_start 1, max_vdotf_negatif 2000. */
int cacb200_set_fire_params(cacb200_ctx *ctx, int delaystep, double dtgrow, double dtshrink,
                            double alpha0, double alphashrink, double tmax, double tmin,
                            double dmax, int halfstepback, int delaystep_start,
                            int max_vdotf_negatif);
/* minimize etol ftol maxiter (Minimize::command, minimize.cpp:21-70, with
 * nodal/weight 1) by a device FIRE iterate over atoms + nodes: FIRE 2.0 of
 * Guenole et al. 2020 with the FIRE parameters and defaults the reference's
 * Min carries (its own min styles are cg and sd, with no FIRE style; the
 * input-deck form is the package's min_style fire/b200, a Min subclass that
 * calls this with the rule Min::init sets, cacb200_set_neighbor_modify).
 * The lists follow cacb200_set_neighbor / _modify.  normstyle: 0 two-norm, 1 max
 * per-site norm, 2 inf norm (min_modify norm two|max|inf).  Returns the stop
 * code of min.h:46-47 (0 MAXITER, 2 ETOL, 3 FTOL, 11 MAXVDOTF), iterations,
 * final energy and force norm (squared, in the chosen style). */
int cacb200_minimize_fire(cacb200_ctx *ctx, double etol, double ftol, int maxiter, double dt,
                          int normstyle, int *stop_code, int *niter, double *energy,
                          double *fnorm);

/* Device-side copy of the state (x, v, nodex, nodev) and its restoration;
 * restoring invalidates the lists (call cacb200_setup before stepping).
 * Serves restarts of short trajectories and job preemption without host
 * traffic. */
int cacb200_snapshot(cacb200_ctx *ctx);
int cacb200_restore(cacb200_ctx *ctx);

/* The same per-replica energies from per-site energies the caller holds on
 * the device, with no device allocation at all: no counterpart in the
 * reference.  For callers that must not allocate device memory (a host
 * program whose GPU memory belongs to another framework's pool, or a loop
 * that cannot afford the device-wide wait of cudaFree beside running
 * streams).  eatom [sum natoms] and enode [sum nelements][8] are device
 * arrays, replicas one after another; natoms, nelements [nreplicas] and
 * energy [nreplicas] are host arrays; node_weight multiplies node energies
 * (729/8 for the UNIFORM Hex element; 1 for EAM during minimisation).  The
 * scratch is one fixed device array of this library for at most
 * CACB200_NOALLOC_MAX_REPLICAS replicas (more: CACB200_EINVAL), held by
 * every GPU that loads the library until exit.  A failed call leaves its
 * reason in cacb200_noalloc_last_error() (per thread; empty after a
 * success).  The
 * first call on a device looks up that array's device address; make it
 * before any stream capture.  The address is kept for the life of the
 * process: a device reset (cudaDeviceReset, or another framework resetting
 * the primary context) after that first call is not supported, since the
 * library's module would be loaded again at another address.  A call copies
 * 16 bytes of offsets and counts per replica.  Every call shares the array, so calls that
 * overlap on the GPU (other streams, other threads) race; each call waits
 * for its stream before returning. */
#define CACB200_NOALLOC_MAX_REPLICAS 4096
int cacb200_replica_energy_noalloc(int device, const double *eatom, const double *enode,
                                   int nreplicas, const int *natoms, const int *nelements,
                                   double node_weight, double *energy /* [nreplicas] */,
                                   void *stream /* cudaStream_t */);
const char *cacb200_noalloc_last_error(void);

/* cacb200_run_nve replays each rebuild cycle (every steps) as two CUDA
 * graphs, with one host wait per cycle to read the rebuild's overflow flags.
 * Enabled by default; disabling runs every launch eagerly (same kernels,
 * same order, same results).  No reference counterpart (Verlet::run,
 * verlet.cpp:192-360, calls the styles step by step). */
int cacb200_set_graphs(cacb200_ctx *ctx, int enable);
/* graph launches made so far by this context */
int cacb200_graph_launches(cacb200_ctx *ctx, long long *count);
/* Block sizes (threads) of the force-only EAM passes of the current precision
 * form: chosen per context by timing 64, 128 and 256 threads on the
 * context's own lists the first time they run (results do not depend on the
 * choice); 128 before that.  No reference counterpart. */
int cacb200_pair_blocks(cacb200_ctx *ctx, int *rho_threads, int *force_threads);
/* Batches in the mixed form run the EAM passes as persistent work-queue
 * launches: resident blocks take items (a run of consecutive list slots of
 * one replica, the largest replicas first) from a counter, so one launch
 * serves replicas of every size without idle tails.  The run length (tile:
 * 128, 512 or 2048 slots) is chosen per replica size class (i-sites below
 * 8,192, below 32,768, larger) by timing the force pass when the capacity
 * plan changes; results do not depend on it (each slot's arithmetic is that
 * of the grid launch).  Single systems run the atom-list build, and in the
 * FP64 form the force-only EAM passes, over SM-local runs instead: the
 * sorted atoms or list slots are cut into runs (32 atoms; 128 slots) and each
 * multiprocessor owns a contiguous range of runs, so the blocks resident on
 * one multiprocessor share their neighbours' data in its L1; a block whose
 * own range is exhausted takes runs from another range (same lists and
 * results as the grid launches, bit for bit).  enable: 1 on (default), 0 off
 * (one grid launch per pass), -1 unchanged; tiles [3] gets the chosen tiles
 * of batches (0: not chosen yet).  No reference counterpart (the reference
 * runs one system per process). */
int cacb200_work_queue(cacb200_ctx *ctx, int enable, int tiles[3]);

/* Kernel timing: when enabled, every launch is bracketed by CUDA events and
 * per-kernel totals accumulate (ms, launches) until reset. */
int cacb200_profile(cacb200_ctx *ctx, int enable);
int cacb200_profile_read(cacb200_ctx *ctx, int max, char *names /* max*32 */,
                         double *total_ms, int64_t *launches, int *count);

/* ---------------------------------------------------------------- serving */

/* A job server (no reference counterpart: the reference runs one input deck
 * per process).  Worker threads each own one context (own CUDA stream,
 * buffers reused across jobs) and take jobs first come first served once the
 * job's device-memory estimate fits the budget, so jobs of any size run
 * concurrently and start as soon as room frees up.  A job is one system plus
 * `run N` under fix nve (CACB200_JOB_NVE, steps = N) or `minimize etol ftol
 * N` with the FIRE iterate and max-norm (CACB200_JOB_FIRE, steps = maxiter);
 * it runs through the same context calls as a single run, so its results
 * equal that run's bit for bit whatever else is being served.  Configure
 * (pair style, neighbour settings) before cacb200_server_start.  Each worker
 * keeps the buffers of the largest job it has run. */
typedef struct cacb200_server cacb200_server;
#define CACB200_JOB_NVE 0
#define CACB200_JOB_FIRE 1
int cacb200_server_create(int device, int nworkers, double budget_bytes, int precision,
                          cacb200_server **out);
int cacb200_server_set_lj(cacb200_server *s, double epsilon, double sigma, double cut);
int cacb200_server_set_eam(cacb200_server *s, int nrho, double drho, int nr, double dr, double cut,
                           const double *frho, const double *rhor, const double *z2r);
int cacb200_server_set_neighbor(cacb200_server *s, double skin, int every);
/* NVE jobs of more than `segment` steps run as trajectories of `segment`
 * steps, each restarted from the job's initial state (device snapshot), the
 * last one ending the job; 0 (default) runs one trajectory. */
int cacb200_server_set_segment(cacb200_server *s, int segment);
int cacb200_server_start(cacb200_server *s);
/* Queue a job (arrays are copied).  CACB200_ENOMEM when the job alone
 * exceeds the budget. */
int cacb200_server_submit(cacb200_server *s, int kind, const double boxlo[3], const double boxhi[3],
                          int natoms, const double *x, const double *v, int nelements,
                          const double *nodex, const double *nodev, double mass, int steps,
                          double dt, double etol, double ftol, int64_t *job);
/* Block until the job ends (timeout_s < 0: no limit); returns its status
 * (CACB200_OK, CACB200_ETIMEDOUT while still queued or running, or the
 * job's error code). */
int cacb200_server_wait(cacb200_server *s, int64_t job, double timeout_s);
/* An NVE job under fix langevin t_start t_stop damp seed [zero yes]
 * (cacb200_set_langevin semantics: the reference's RanMars stream for `seed`,
 * started with the job; with segmented NVE the stream runs on across the
 * restarts).  Its results equal the same run on one context bit for bit. */
int cacb200_server_submit_nvt(cacb200_server *s, const double boxlo[3], const double boxhi[3],
                              int natoms, const double *x, const double *v, int nelements,
                              const double *nodex, const double *nodev, double mass, int steps,
                              double dt, double t_start, double t_stop, double damp, int seed,
                              int zero, int64_t *job);
/* The job's thermo line at its end (cacb200_thermo, metal units:
 * CACB200_THERMO_N doubles), reduced on the device before the state is read
 * back.  NVE jobs tally energy and virial on their last step; FIRE jobs
 * evaluate their final positions once more for the virial. */
int cacb200_server_thermo(cacb200_server *s, int64_t job, double *out /* [CACB200_THERMO_N] */);
/* Final state, energy (eng_vdwl), iterations and FIRE stop code (-1 for
 * NVE), and times in seconds: [queued, running, submit to end] (times are
 * filled for failed jobs too, which return their error code). */
int cacb200_server_result(cacb200_server *s, int64_t job, double *x, double *v, double *nodex,
                          double *nodev, double *energy, int *niter, int *stop_code,
                          double *times /* [3] */);
int cacb200_server_release(cacb200_server *s, int64_t job);
const char *cacb200_server_last_error(const cacb200_server *s);
/* Finish running jobs, drop queued ones, join the workers. */
int cacb200_server_destroy(cacb200_server *s);

#ifdef __cplusplus
}
#endif

#endif
