#include "pair_lj_cut_b200.h"

#include "atom.h"
#include "error.h"

using namespace CAC_NS;

PairLJCutB200::PairLJCutB200(CAC *cac) : PairLJCut(cac) { bridge = new B200Bridge(cac); }

PairLJCutB200::~PairLJCutB200() { delete bridge; }

void PairLJCutB200::init_style()
{
  // no host list: the device lists follow Neighbor::ago
  cut_respa = nullptr;
}

double PairLJCutB200::init_one(int i, int j)
{
  double c = PairLJCut::init_one(i, j);
  if (atom->ntypes != 1) error->all(FLERR, "pair lj/cut/b200 supports one atom type");
  bridge->set_lj(epsilon[1][1], sigma[1][1], cut[1][1]);
  return c;
}

void PairLJCutB200::compute(int eflag, int vflag)
{
  ev_init(eflag, vflag);
  bridge->compute(this);
}
