#include "run_b200.h"

#include <cstring>

#include "cac.h"
#include "error.h"
#include "fix.h"
#include "force.h"
#include "modify.h"
#include "neighbor.h"
#include "pair_eam_alloy_b200.h"
#include "pair_lj_cut_b200.h"
#include "universe.h"
#include "update.h"

using namespace CAC_NS;

namespace {

B200Bridge *bridge_of(Pair *pair)
{
  if (auto *p = dynamic_cast<PairLJCutB200 *>(pair)) return p->bridge;
  if (auto *p = dynamic_cast<PairEAMAlloyB200 *>(pair)) return p->bridge;
  return nullptr;
}

}  // namespace

void RunB200::command(int narg, char **arg)
{
  if (narg != 1) error->all(FLERR, "Illegal run_b200 command: run_b200 N");
  int nsteps = universe->inumeric(FLERR, arg[0]);
  if (nsteps < 0) error->all(FLERR, "Illegal run_b200 step count");
  B200Bridge *b = bridge_of(force->pair);
  if (!b) error->all(FLERR, "run_b200 needs pair style lj/cut/b200 or eam/alloy/b200");
  int nve = 0;
  for (int i = 0; i < modify->nfix; i++) {
    if (strcmp(modify->fix[i]->style, "nve") == 0) nve++;
    else error->all(FLERR, "run_b200 integrates fix nve only; remove other fixes");
  }
  if (nve != 1) error->all(FLERR, "run_b200 needs exactly one fix nve");
  cac->init();   // pair init_style/init_one push the tables to the bridge
  b->run_nve(nsteps, update->dt, neighbor->every);
  update->ntimestep += nsteps;
}

void WriteB200Neighbor::command(int narg, char **arg)
{
  if (narg != 2) error->all(FLERR, "Illegal write_b200_neighbor command: FILE half|full");
  int half = strcmp(arg[1], "half") == 0;
  if (!half && strcmp(arg[1], "full") != 0) error->all(FLERR, "write_b200_neighbor: half or full");
  B200Bridge *b = bridge_of(force->pair);
  if (!b) error->all(FLERR, "write_b200_neighbor needs a /b200 pair style");
  cac->init();
  b->dump_list(arg[0], half);
}
