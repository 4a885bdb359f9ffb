/*
 * Computes that read the device instead of the host arrays.
 *
 * compute ID group temp/b200 [args of temp]: ComputeTemp (compute_temp.cpp:
 *   74-243) whose scalar and kinetic tensor come from the device thermo
 *   read-out (cacb200_thermo) while a device run writes an output step;
 *   otherwise ComputeTemp itself.  run_style verlet/b200 and run_b200 put it
 *   in place of the thermo's own thermo_temp, so thermo lines during a device
 *   run need no host copy of the velocities.
 *
 * compute ID group pe/atom/b200 and compute ID group stress/atom/b200 NULL:
 *   per-site potential energy (ComputePEAtom, compute_pe_atom.cpp) and
 *   stress (ComputeStressAtom, compute_stress_atom.cpp:235-330: -nktv2p x
 *   per-site virial, no kinetic term, as in this reference's pair-only form)
 *   of atoms and nodes, copied from the device's per-site tallies of the
 *   current step (the /b200 pair style's context) instead of the pair's host
 *   arrays.
 */
#ifdef COMPUTE_CLASS

ComputeStyle(temp/b200, ComputeTempB200)
ComputeStyle(pe/atom/b200, ComputePEAtomB200)
ComputeStyle(stress/atom/b200, ComputeStressAtomB200)

#else

#ifndef CAC_COMPUTE_B200_H
#define CAC_COMPUTE_B200_H

#include <vector>

#include "compute.h"
#include "compute_temp.h"

namespace CAC_NS {

class ComputeTempB200 : public ComputeTemp {
 public:
  ComputeTempB200(class CAC *, int, char **);
  double compute_scalar() override;
  void compute_vector() override;
};

class ComputePEAtomB200 : public Compute {
 public:
  ComputePEAtomB200(class CAC *, int, char **);
  ~ComputePEAtomB200() override;
  void init() override {}
  void compute_peratom() override;
  double memory_usage() override;

 private:
  int atom_nmax = 0, elem_nmax = 0;
  double *atom_energy = nullptr;
  double ***node_energy = nullptr;
  std::vector<double> ebuf, enbuf;
};

class ComputeStressAtomB200 : public Compute {
 public:
  ComputeStressAtomB200(class CAC *, int, char **);
  ~ComputeStressAtomB200() override;
  void init() override {}
  void compute_peratom() override;
  double memory_usage() override;

 private:
  int atom_nmax = 0, elem_nmax = 0;
  double **atom_stress = nullptr;
  double ****node_stress = nullptr;
  std::vector<double> vbuf, vnbuf;
};

// Put compute temp/b200 in place of the thermo's thermo_temp (same group);
// no-op when it is there already or the deck replaced thermo_temp.
void b200_use_device_thermo(class CAC *cac);

// True when every compute defined is one the device output path serves
// (temp/b200, thermo_press, thermo_pe, the /b200 per-site computes): then an
// output step of a device run needs no host copy of the state.  Otherwise
// the state is copied at every output step.  Variables are not inspected (the
// reference keeps their count private): thermo keywords and equal-style
// variables of thermo keywords are served; an atom-style variable printed by
// thermo would read the state of the last copy.
bool b200_device_output_safe(class CAC *cac);

}  // namespace CAC_NS

#endif
#endif
