#include "pair_lj_cut_b200.h"

#include "atom.h"
#include "error.h"
#include "neighbor.h"

using namespace CAC_NS;

PairLJCutB200::PairLJCutB200(CAC *cac) : PairLJCut(cac) { bridge = new B200Bridge(cac); }

PairLJCutB200::~PairLJCutB200() { delete bridge; }

void PairLJCutB200::init_style()
{
  // the default half list (as PairLJCut::init_style requests it); the NPair
  // class serving it (half/bin/newton/b200) stores nothing during a run:
  // the device lists follow Neighbor::ago.  The requestor is the Pair
  // subobject: Neighbor::init casts it back to Pair *.
  neighbor->request(static_cast<Pair *>(this), instance_me);
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
