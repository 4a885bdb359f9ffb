#include "fix_langevin_b200.h"

#include "atom.h"
#include "element.h"
#include "random_mars.h"

using namespace CAC_NS;

FixLangevinB200::FixLangevinB200(CAC *cac, int narg, char **arg) : FixLangevin(cac, narg, arg) {}

// FixLangevin::post_force draws 3 values per atom, then 3 per node of every
// element (fix_langevin.cpp:538-646)
void FixLangevinB200::post_force(int vflag)
{
  FixLangevin::post_force(vflag);
  draws += draws_per_call();
}

long long FixLangevinB200::draws_per_call() const
{
  long long n = 3LL * atom->nlocal;
  for (int i = 0; i < element->nlocal; i++)
    n += 3LL * element->npe[element->etype[i]] * element->apc[element->etype[i]];
  return n;
}

void FixLangevinB200::advance(long long n)
{
  for (long long k = 0; k < n; k++) random->uniform();
  draws += n;
}
