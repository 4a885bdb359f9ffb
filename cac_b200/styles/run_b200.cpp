#include "run_b200.h"

#include <cstring>
#include <string>

#include "cac.h"
#include "compute_b200.h"
#include "error.h"
#include "fix.h"
#include "fix_deform_b200.h"
#include "fix_langevin_b200.h"
#include "force.h"
#include "modify.h"
#include "neighbor.h"
#include "output.h"
#include "pair_eam_alloy_b200.h"
#include "pair_lj_cut_b200.h"
#include "universe.h"
#include "update.h"

using namespace CAC_NS;

// The fixes a device run applies besides fix nve (fix langevin/b200, fix
// deform/b200), read from the reference's Modify; errors for anything else.
FixLangevinB200 *CAC_NS::b200_device_fixes(CAC *cac, const char *who, B200Fixes &fx)
{
  Modify *modify = cac->modify;
  Error *error = cac->error;
  int nve = 0;
  FixLangevinB200 *lgv = nullptr;
  FixDeformB200 *dfm = nullptr;
  for (int i = 0; i < modify->nfix; i++) {
    Fix *f = modify->fix[i];
    if (strcmp(f->style, "nve") == 0) {
      nve++;
    } else if (auto *l = dynamic_cast<FixLangevinB200 *>(f)) {
      if (lgv) error->all(FLERR, (std::string(who) + " takes one fix langevin/b200").c_str());
      lgv = l;
    } else if (auto *d = dynamic_cast<FixDeformB200 *>(f)) {
      if (dfm) error->all(FLERR, (std::string(who) + " takes one fix deform/b200").c_str());
      dfm = d;
    } else {
      error->all(FLERR, (std::string(who) + " integrates fix nve with fix langevin/b200 and fix deform/b200 only; "
                                            "remove other fixes (use the /b200 forms of langevin and deform)").c_str());
    }
  }
  if (nve != 1) error->all(FLERR, (std::string(who) + " needs exactly one fix nve").c_str());
  fx = B200Fixes();
  if (lgv) {
    if (!lgv->device_ok())
      error->all(FLERR, (std::string(who) + ": fix langevin/b200 needs group all and constant temperatures").c_str());
    fx.langevin = true;
    fx.t_start = lgv->start();
    fx.t_stop = lgv->stop();
    fx.t_period = lgv->damp();
    fx.seed = lgv->seed_value();
    fx.zero = lgv->zero();
    fx.draws = lgv->draws;
  }
  if (dfm) {
    if (!dfm->device_ok())
      error->all(FLERR, (std::string(who) + ": fix deform/b200 needs group all, an orthogonal box, no tilt and "
                                            "remap x, v or none").c_str());
    fx.deform = true;
    fx.deform_every = dfm->every();
    fx.deform_remap_x = dfm->remap_x();
    for (int d = 0; d < 3; d++) {
      fx.deform_style[d] = dfm->device_style(d, fx.deform_a[d], fx.deform_b[d]);
      if (fx.deform_style[d] < 0)
        error->all(FLERR, (std::string(who) + ": fix deform/b200 variable styles are not offered").c_str());
    }
  }
  return lgv;
}

void RunB200::command(int narg, char **arg)
{
  if (narg != 1) error->all(FLERR, "Illegal run_b200 command: run_b200 N");
  int nsteps = universe->inumeric(FLERR, arg[0]);
  if (nsteps < 0) error->all(FLERR, "Illegal run_b200 step count");
  B200Bridge *b = b200_bridge_of(force->pair);
  if (!b) error->all(FLERR, "run_b200 needs pair style lj/cut/b200 or eam/alloy/b200");
  B200Fixes fx;
  FixLangevinB200 *lgv = b200_device_fixes(cac, "run_b200", fx);
  b200_use_device_thermo(cac);
  // the run's bookkeeping as Run::command keeps it (run.cpp:150-200), so
  // that the reference's Output schedules thermo and dumps over this run
  const bigint step0 = update->ntimestep;
  update->whichflag = 1;
  update->nsteps = nsteps;
  update->firststep = update->beginstep = step0;
  update->laststep = update->endstep = step0 + nsteps;
  cac->init();   // pair init_style/init_one push the tables to the bridge
  b->run_device(nsteps, update->dt, neighbor->every, fx, true);
  // the host generator continues after the device's draws: the run's setup
  // call and one call per step
  if (lgv) lgv->advance((long long)(nsteps + 1) * lgv->draws_per_call());
  update->ntimestep = step0 + nsteps;
  update->whichflag = 0;
  update->firststep = update->laststep = 0;
  update->beginstep = update->endstep = 0;
}

void WriteB200Neighbor::command(int narg, char **arg)
{
  if (narg != 2) error->all(FLERR, "Illegal write_b200_neighbor command: FILE half|full");
  int half = strcmp(arg[1], "half") == 0;
  if (!half && strcmp(arg[1], "full") != 0) error->all(FLERR, "write_b200_neighbor: half or full");
  B200Bridge *b = b200_bridge_of(force->pair);
  if (!b) error->all(FLERR, "write_b200_neighbor needs a /b200 pair style");
  cac->init();
  b->dump_list(arg[0], half);
}

void RunStyle::command(int narg, char **arg)
{
  if (narg < 1) error->all(FLERR, "Illegal run_style command: run_style STYLE [args]");
  update->create_integrate(narg, arg, 1);
}
