#include "compute_b200.h"

#include <cstring>
#include <string>

#include "atom.h"
#include "b200_bridge.h"
#include "cacb200.h"
#include "domain.h"
#include "element.h"
#include "error.h"
#include "force.h"
#include "group.h"
#include "memory.h"
#include "modify.h"
#include "pair.h"
#include "update.h"

using namespace CAC_NS;

/* ------------------------------------------------------------ temp/b200 */

ComputeTempB200::ComputeTempB200(CAC *cac, int narg, char **arg) : ComputeTemp(cac, narg, arg) {}

// The device read-out serves group all with the default options only (the
// device reduces the whole system with the CONSISTENT element mass matrix);
// any other use is ComputeTemp's own.
double ComputeTempB200::compute_scalar()
{
  if (b200_thermo_now.active && b200_thermo_now.step == update->ntimestep && igroup == 0 && !accurate_flag &&
      nodal_force_style == Element::CONSISTENT) {
    invoked_scalar = update->ntimestep;
    scalar = b200_thermo_now.v[CACB200_THERMO_TEMP];
    return scalar;
  }
  return ComputeTemp::compute_scalar();
}

void ComputeTempB200::compute_vector()
{
  if (b200_thermo_now.active && b200_thermo_now.step == update->ntimestep && igroup == 0 && !accurate_flag &&
      nodal_force_style == Element::CONSISTENT && force->pair) {
    invoked_vector = update->ntimestep;
    // the kinetic tensor (mvv2e sum m v v, compute_temp.cpp:160-243) from the
    // device pressure tensor P = (K + W) / V * nktv2p (compute_pressure.cpp:
    // 190-220) less the pair virial W of the same step
    const double vol = domain->xprd * domain->yprd * domain->zprd;
    const double *w = force->pair->virial;
    for (int k = 0; k < 6; k++) vector[k] = b200_thermo_now.v[CACB200_THERMO_PXX + k] * vol / force->nktv2p - w[k];
    return;
  }
  ComputeTemp::compute_vector();
}

/* ------------------------------------------------------- per-site computes */

static B200Bridge *bridge_for(Pair *pair, Error *error, const char *style)
{
  B200Bridge *b = pair ? b200_bridge_of(pair) : nullptr;
  if (!b || !b->ctx) {
    std::string msg = std::string("compute ") + style + " needs a /b200 pair style that has evaluated forces";
    error->all(FLERR, msg.c_str());
  }
  return b;
}

ComputePEAtomB200::ComputePEAtomB200(CAC *cac, int narg, char **arg) : Compute(cac, narg, arg)
{
  if (narg != 3) error->all(FLERR, "Illegal compute pe/atom/b200 command");
  peratom_flag = 1;
  size_peratom_cols = 0;
  element_data_style = NODE;
  peatomflag = 1;   // the integrator tallies per-site energy on the steps this compute is invoked
  timeflag = 1;
}

ComputePEAtomB200::~ComputePEAtomB200()
{
  memory->destroy(atom_energy);
  memory->destroy(node_energy);
}

void ComputePEAtomB200::compute_peratom()
{
  invoked_peratom = update->ntimestep;
  if (update->eflag_atom != invoked_peratom)
    error->all(FLERR, "Per-atom atom_energy was not tallied on needed timestep");
  B200Bridge *b = bridge_for(force->pair, error, "pe/atom/b200");
  if (atom->nmax > atom_nmax) {
    memory->destroy(atom_energy);
    atom_nmax = atom->nmax;
    memory->create(atom_energy, atom_nmax, "pe/atom/b200:atom_energy");
  }
  if (element->nmax > elem_nmax) {
    memory->destroy(node_energy);
    elem_nmax = element->nmax;
    memory->create(node_energy, elem_nmax, element->maxapc, element->maxnpe, "pe/atom/b200:node_energy");
  }
  vector_atom = atom_energy;
  vector_node = node_energy;
  const int na = atom->nlocal, ne = element->nlocal;
  ebuf.resize(std::max(na, 1));
  enbuf.resize(8 * (size_t) std::max(ne, 1));
  double e = 0.0;
  if (cacb200_get_energy(b->ctx, &e, nullptr, ebuf.data(), nullptr, enbuf.data(), nullptr) != CACB200_OK)
    error->all(FLERR, (std::string("compute pe/atom/b200: ") + cacb200_last_error(b->ctx)).c_str());
  int *amask = atom->mask, *emask = element->mask;
  for (int i = 0; i < na; i++) atom_energy[i] = (amask[i] & groupbit) ? ebuf[i] : 0.0;
  for (int i = 0; i < ne; i++)
    for (int n = 0; n < 8; n++) node_energy[i][0][n] = (emask[i] & groupbit) ? enbuf[8 * (size_t) i + n] : 0.0;
}

double ComputePEAtomB200::memory_usage()
{
  return sizeof(double) * ((double) atom_nmax + (double) elem_nmax * element->maxapc * element->maxnpe);
}

ComputeStressAtomB200::ComputeStressAtomB200(CAC *cac, int narg, char **arg) : Compute(cac, narg, arg)
{
  // compute ID group stress/atom/b200 NULL [pair | virial]: the reference's
  // form without a temperature (its kinetic term is not offered there either)
  if (narg < 4 || strcmp(arg[3], "NULL") != 0) error->all(FLERR, "Illegal compute stress/atom/b200 command");
  for (int iarg = 4; iarg < narg; iarg++)
    if (strcmp(arg[iarg], "pair") != 0 && strcmp(arg[iarg], "virial") != 0)
      error->all(FLERR, "Illegal compute stress/atom/b200 command");
  peratom_flag = 1;
  size_peratom_cols = 6;
  element_data_style = NODE;
  pressatomflag = 1;   // the integrator tallies per-site virial on the steps this compute is invoked
  timeflag = 1;
}

ComputeStressAtomB200::~ComputeStressAtomB200()
{
  memory->destroy(atom_stress);
  memory->destroy(node_stress);
}

void ComputeStressAtomB200::compute_peratom()
{
  invoked_peratom = update->ntimestep;
  if (update->vflag_atom != invoked_peratom)
    error->all(FLERR, "Per-atom virial was not tallied on needed timestep");
  B200Bridge *b = bridge_for(force->pair, error, "stress/atom/b200");
  if (atom->nmax > atom_nmax) {
    memory->destroy(atom_stress);
    atom_nmax = atom->nmax;
    memory->create(atom_stress, atom_nmax, 6, "stress/atom/b200:atom_stress");
  }
  if (element->nmax > elem_nmax) {
    memory->destroy(node_stress);
    elem_nmax = element->nmax;
    memory->create(node_stress, elem_nmax, element->maxapc, element->maxnpe, 6, "stress/atom/b200:node_stress");
  }
  array_atom = atom_stress;
  array_node = node_stress;
  const int na = atom->nlocal, ne = element->nlocal;
  vbuf.resize(6 * (size_t) std::max(na, 1));
  vnbuf.resize(48 * (size_t) std::max(ne, 1));
  double e = 0.0;
  if (cacb200_get_energy(b->ctx, &e, nullptr, nullptr, vbuf.data(), nullptr, vnbuf.data()) != CACB200_OK)
    error->all(FLERR, (std::string("compute stress/atom/b200: ") + cacb200_last_error(b->ctx)).c_str());
  // stress = -nktv2p x per-site virial (compute_stress_atom.cpp:300-330)
  const double s = -force->nktv2p;
  int *amask = atom->mask, *emask = element->mask;
  for (int i = 0; i < na; i++)
    for (int k = 0; k < 6; k++) atom_stress[i][k] = (amask[i] & groupbit) ? s * vbuf[6 * (size_t) i + k] : 0.0;
  for (int i = 0; i < ne; i++)
    for (int n = 0; n < 8; n++)
      for (int k = 0; k < 6; k++)
        node_stress[i][0][n][k] = (emask[i] & groupbit) ? s * vnbuf[48 * (size_t) i + 6 * n + k] : 0.0;
}

double ComputeStressAtomB200::memory_usage()
{
  return 6.0 * sizeof(double) * ((double) atom_nmax + (double) elem_nmax * element->maxapc * element->maxnpe);
}

/* -------------------------------------------------------------- helpers */

void CAC_NS::b200_use_device_thermo(CAC *cac)
{
  Modify *modify = cac->modify;
  int i = modify->find_compute("thermo_temp");
  if (i < 0) return;
  Compute *c = modify->compute[i];
  if (strcmp(c->style, "temp") != 0) return;   // temp/b200 already, or replaced by the deck
  std::string gname = cac->group->names[c->igroup];
  modify->delete_compute("thermo_temp");
  char *args[3] = {(char *) "thermo_temp", (char *) gname.c_str(), (char *) "temp/b200"};
  modify->add_compute(3, args);
}

bool CAC_NS::b200_device_output_safe(CAC *cac)
{
  Modify *modify = cac->modify;
  for (int i = 0; i < modify->ncompute; i++) {
    const Compute *c = modify->compute[i];
    const char *id = c->id, *st = c->style;
    bool ok = strcmp(st, "temp/b200") == 0 || strcmp(st, "pe/atom/b200") == 0 ||
              strcmp(st, "stress/atom/b200") == 0 ||
              (strcmp(id, "thermo_press") == 0 && strcmp(st, "pressure") == 0) ||
              (strcmp(id, "thermo_pe") == 0 && strcmp(st, "pe") == 0);
    if (!ok) return false;
  }
  return true;
}
