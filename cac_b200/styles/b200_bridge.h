/*
 * Bridge between the CAC reference's host data (Atom, Element, Domain, Pair)
 * and one cacb200 context (include/cacb200.h).  Used by the /b200 styles of
 * this package; compiled into the reference executable together with them.
 *
 * The bridge owns the device context of one system.  Every force call copies
 * the owned atoms' and elements' positions to the device (the whole system on
 * the first call and whenever the reference has just rebuilt its neighbour
 * lists, Neighbor::ago == 0, so that atom order and ghost images stay in step
 * with the reference), evaluates the pair style there and adds the owned
 * forces, Gauss-point forces, energies and virial back into the reference's
 * arrays.  Ghost sites need nothing: on one rank every ghost is a periodic
 * image, and the device applies the images itself, so owners receive their
 * complete forces and the reference's reverse communication adds zeros.
 */
#ifndef CAC_B200_BRIDGE_H
#define CAC_B200_BRIDGE_H

#include <vector>

#include "pointers.h"

struct cacb200_ctx;

namespace CAC_NS {

// Fixes run_b200 applies on the device besides fix nve (settings read from
// the langevin/b200 and deform/b200 styles)
struct B200Fixes {
  bool langevin = false;
  double t_start = 0, t_stop = 0, t_period = 1;
  int seed = 1, zero = 0;
  long long draws = 1;          // uniform() calls the host generator has made
  bool deform = false;
  int deform_every = 1, deform_remap_x = 1;
  int deform_style[3] = {0, 0, 0};
  double deform_a[3] = {0, 0, 0}, deform_b[3] = {0, 0, 0};
};

// min_style fire/b200: the FIRE parameters of Min (min.h:61-72) with the
// reference's defaults (min.cpp:33-47)
struct B200Fire {
  int delaystep = 20;
  double dtgrow = 1.1, dtshrink = 0.5, alpha0 = 0.25, alphashrink = 0.99;
  double tmax = 10.0, tmin = 0.02, dmax = 0.1;
  int halfstepback = 1, delaystep_start = 1, max_vdotf_negatif = 2000;
};

// The device thermo read-out (cacb200_thermo) of the output step the
// reference's Output is writing during a device run; compute temp/b200 reads
// it instead of the host velocities while `active` and the step matches.
struct B200ThermoNow {
  bool active = false;
  bigint step = -1;
  double v[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
};
extern B200ThermoNow b200_thermo_now;

class B200Bridge : protected Pointers {
 public:
  explicit B200Bridge(class CAC *);
  ~B200Bridge();

  void set_lj(double epsilon, double sigma, double cut);
  void set_eam(int nrho, double drho, int nr, double dr, double cut, const double *frho,
               const double *rhor, const double *z2r);
  // Pair::compute body: fills atom->f, element->gaussf, eng_vdwl, virial and
  // the per-site arrays of `pair` according to its ev flags.
  void compute(class Pair *pair);
  // run N velocity-Verlet steps on the device (run_b200 command, run_style
  // verlet/b200), with the given thermostat / deformation.  Output comes on
  // the reference's schedule through its own Output: at every output step the
  // device's global tallies go into the pair and its thermo read-out to
  // compute temp/b200, so thermo lines copy no per-site data; a dump due at
  // the step (or computes that read host per-site data) bring the state,
  // the forces and the per-site tallies into the reference's arrays.
  // step0_output: also write step 0 (run_b200; under run the integrator's
  // setup did).
  void run_device(int nsteps, double dt, int every, const B200Fixes &fixes, bool step0_output);
  // per-site state copies to the host made for output during device runs
  long long state_copies = 0;
  // a device run copies the state at every output step (computes that read
  // host per-site data are defined)
  bool output_copies_state = false;
  // minimise on the device from the reference's current state (min_style
  // fire/b200) under the reference's current neighbour rule; the final
  // positions come back into atom->x / element->nodex (velocities are left
  // as they are, as by the reference's minimisers)
  void minimize_fire(double etol, double ftol, int maxiter, double dt, int normstyle, const B200Fire &p,
                     int &stop, int &niter, double &energy, double &fnorm);
  // canonical neighbour-list dump (write_b200_neighbor command)
  void dump_list(const char *file, int half);
  // the device's half list into the reference's host list (NPair
  // half/bin/newton/b200 outside a run): its site order, local and ghost
  // indices, lattice-site index of element neighbours
  void fill_host_list(class NeighList *list);

  cacb200_ctx *ctx = nullptr;

 private:
  int pair_style = 0;
  std::vector<double> lj;                 // eps, sigma, cut
  std::vector<double> eam_frho, eam_rhor, eam_z2r;
  int eam_nrho = 0, eam_nr = 0;
  double eam_drho = 0, eam_dr = 0, eam_cut = 0;
  int uploaded_na = -1, uploaded_ne = -1;
  double uploaded_lo[3] = {0, 0, 0}, uploaded_hi[3] = {0, 0, 0};   // box the device holds
  std::vector<double> fbuf, gbuf, ebuf, vbuf, enbuf, vnbuf;

  void check_system();
  void download_state(bool box);
  void download_forces();
  void output_step(bigint step, bool box, bool first);
  void upload(bool with_velocities);
  void configure_pair();
  void status(int rc, const char *what);
};

// The bridge of a /b200 pair style (lj/cut/b200, eam/alloy/b200), else null.
B200Bridge *b200_bridge_of(class Pair *pair);

}  // namespace CAC_NS

#endif
