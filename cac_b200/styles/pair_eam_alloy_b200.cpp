#include "pair_eam_alloy_b200.h"

#include "atom.h"
#include "error.h"
#include "neighbor.h"

using namespace CAC_NS;

PairEAMAlloyB200::PairEAMAlloyB200(CAC *cac) : PairEAM(cac), PairEAMAlloy(cac)
{
  bridge = new B200Bridge(cac);
}

PairEAMAlloyB200::~PairEAMAlloyB200() { delete bridge; }

void PairEAMAlloyB200::init_style()
{
  // tables as PairEAM::init_style builds them (pair_eam.cpp:310-318), and
  // its default half list request; the NPair class serving it
  // (half/bin/newton/b200) stores nothing during a run.  The requestor is
  // the Pair subobject: Neighbor::init casts it back to Pair *.
  file2array();
  array2spline();
  neighbor->request(static_cast<Pair *>(this), instance_me);
  if (setfl == nullptr || setfl->nelements != 1)
    error->all(FLERR, "pair eam/alloy/b200 needs a one-element setfl file");
  bridge->set_eam(nrho, drho, nr, dr, setfl->cut, &frho[0][1], &rhor[0][1], &z2r[0][1]);
}

void PairEAMAlloyB200::compute(int eflag, int vflag)
{
  ev_init(eflag, vflag);
  bridge->compute(this);
}
