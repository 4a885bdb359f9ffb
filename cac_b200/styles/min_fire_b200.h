/*
 * min_style fire/b200: the whole minimisation of `minimize etol ftol maxiter
 * maxeval` on the device, as FIRE 2.0 (Guenole et al. 2020) with the FIRE
 * parameters and defaults the reference's Min carries (min.h:61-72,
 * min.cpp:33-47; min_modify norm / alpha0 / dmax).  It fits the reference's
 * Min interface (setup_style / reset_vectors / iterate, min.h:36-44): Min's
 * own setup evaluates the start, iterate() hands atoms + nodes to the device
 * and returns Min's stop code, and the final positions come back into
 * atom->x / element->nodex with forces, energy and the combined vectors
 * refreshed through Min::energy_force, so Min::run, Min::cleanup and Finish
 * report as for the reference's own styles.  The device loop writes no
 * intermediate thermo or dump output; the last iteration's is written.
 */
#ifdef MINIMIZE_CLASS

MinimizeStyle(fire/b200, MinFireB200)

#else

#ifndef CAC_MIN_FIRE_B200_H
#define CAC_MIN_FIRE_B200_H

#include "min.h"

namespace CAC_NS {

class MinFireB200 : public Min {
 public:
  MinFireB200(class CAC *);
  ~MinFireB200() override;
  void setup_style() override;
  void reset_vectors() override;
  int iterate(int) override;

 protected:
  void copy_vectors() override;
  void copy_force() override;
};

}  // namespace CAC_NS

#endif
#endif
