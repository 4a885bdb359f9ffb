#include "verlet_b200.h"

#include "b200_bridge.h"
#include "compute_b200.h"
#include "error.h"
#include "fix_langevin_b200.h"
#include "force.h"
#include "neighbor.h"
#include "run_b200.h"
#include "update.h"

using namespace CAC_NS;

VerletB200::VerletB200(CAC *cac, int narg, char **arg) : Verlet(cac, narg, arg) {}

void VerletB200::init()
{
  Verlet::init();
  // the thermo's temperature from the device read-out during the run; set
  // before Modify::init and Output::init, which look computes up by ID
  b200_use_device_thermo(cac);
}

void VerletB200::run(int n, int /*flag*/)
{
  B200Bridge *b = force->pair ? b200_bridge_of(force->pair) : nullptr;
  if (!b) error->all(FLERR, "run_style verlet/b200 needs pair style lj/cut/b200 or eam/alloy/b200");
  B200Fixes fx;
  FixLangevinB200 *lgv = b200_device_fixes(cac, "run_style verlet/b200", fx);
  // Verlet::setup drew the thermostat's setup forces on the host; the
  // device's run start draws them again from the same place of the stream
  // (with the pair forces it evaluates there), so its stream starts one call
  // earlier, and afterwards the host generator skips the device's per-step
  // draws
  if (lgv) fx.draws -= lgv->draws_per_call();
  const bigint step0 = update->ntimestep;
  b->run_device(n, update->dt, neighbor->every, fx, false);
  if (lgv) lgv->advance((long long) n * lgv->draws_per_call());
  update->ntimestep = step0 + n;
}
