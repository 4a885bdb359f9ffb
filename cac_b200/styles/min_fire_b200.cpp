#include "min_fire_b200.h"

#include "atom.h"
#include "b200_bridge.h"
#include "element.h"
#include "error.h"
#include "force.h"
#include "modify.h"
#include "output.h"
#include "pair.h"
#include "update.h"

using namespace CAC_NS;

MinFireB200::MinFireB200(CAC *cac) : Min(cac)
{
  searchflag = 0;   // damped dynamics (no line search)
  xvec = fvec = nullptr;
}

MinFireB200::~MinFireB200()
{
  delete[] xvec;
  delete[] fvec;
}

void MinFireB200::setup_style()
{
  if (!b200_bridge_of(force->pair))
    error->all(FLERR, "min_style fire/b200 needs pair style lj/cut/b200 or eam/alloy/b200");
}

// The combined vectors of MinLineSearch::reset_vectors
// (min_linesearch.cpp:118-143): atoms, then every element's nodes.
void MinFireB200::reset_vectors()
{
  nvec = 3 * (atom->nlocal + element->count_nodes(1));
  delete[] xvec;
  delete[] fvec;
  xvec = new double[nvec > 0 ? nvec : 1];
  fvec = new double[nvec > 0 ? nvec : 1];
}

// xvec -> atom->x + element->nodex, fvec -> atom->f + element->nodef
// (the layout of MinLineSearch::copy_vectors, min_linesearch.cpp:1027-1067)
void MinFireB200::copy_vectors()
{
  int n = 0;
  for (int i = 0; i < atom->nlocal; i++)
    for (int d = 0; d < 3; d++, n++) {
      atom->x[i][d] = xvec[n];
      atom->f[i][d] = fvec[n];
    }
  for (int i = 0; i < element->nlocal; i++) {
    const int et = element->etype[i];
    for (int j = 0; j < element->apc[et]; j++)
      for (int k = 0; k < element->npe[et]; k++)
        for (int d = 0; d < 3; d++, n++) {
          element->nodex[i][j][k][d] = xvec[n];
          element->nodef[i][j][k][d] = fvec[n];
        }
  }
}

// atom->x + element->nodex -> xvec, atom->f + element->nodef -> fvec
// (MinLineSearch::copy_force, min_linesearch.cpp:972-1012)
void MinFireB200::copy_force()
{
  int n = 0;
  for (int i = 0; i < atom->nlocal; i++)
    for (int d = 0; d < 3; d++, n++) {
      xvec[n] = atom->x[i][d];
      fvec[n] = atom->f[i][d];
    }
  for (int i = 0; i < element->nlocal; i++) {
    const int et = element->etype[i];
    for (int j = 0; j < element->apc[et]; j++)
      for (int k = 0; k < element->npe[et]; k++)
        for (int d = 0; d < 3; d++, n++) {
          xvec[n] = element->nodex[i][j][k][d];
          fvec[n] = element->nodef[i][j][k][d];
        }
  }
}

// Up to maxiter FIRE iterations on the device from the state Min::setup
// evaluated, with the neighbour rule Min::init set (every 1 delay 0 check
// yes).  Returns the stop code of min.h (MAXITER, ETOL, FTOL or MAXVDOTF).
int MinFireB200::iterate(int maxiter)
{
  B200Bridge *b = b200_bridge_of(force->pair);
  if (force->pair->nodal_energy_weight != 1.0)
    error->all(FLERR, "min_style fire/b200 minimises with nodal/weight 1 (the minimize default)");
  B200Fire p;
  p.delaystep = delaystep;
  p.dtgrow = dtgrow;
  p.dtshrink = dtshrink;
  p.alpha0 = alpha0;
  p.alphashrink = alphashrink;
  p.tmax = tmax;
  p.tmin = tmin;
  p.dmax = dmax;
  p.halfstepback = halfstepback_flag;
  p.delaystep_start = delaystep_start_flag;
  p.max_vdotf_negatif = max_vdotf_negatif;
  int stop = MAXITER, it = 0;
  double energy = 0.0, fnorm = 0.0;
  b->minimize_fire(update->etol, update->ftol, maxiter, update->dt, normstyle, p, stop, it, energy, fnorm);
  niter = it;
  neval = it;
  update->ntimestep += it;
  copy_force();   // xvec holds the final positions (energy_force starts from it)
  if (stop == MAXITER) {
    // what Min::run does after an early stop: output of the final state
    if (update->restrict_output == 0) {
      for (int idump = 0; idump < output->ndump; idump++) output->next_dump[idump] = update->ntimestep;
      output->next_dump_any = update->ntimestep;
    }
    output->next_thermo = update->ntimestep;
    modify->addstep_compute_all(update->ntimestep);
    ecurrent = energy_force(0);
    output->write(update->ntimestep);
  }
  return stop;
}
