/*
 * run_style verlet/b200: the reference's Verlet (verlet.cpp:64-360) with its
 * step loop on the device.  Setup is Verlet::setup unchanged (host comm,
 * the /b200 pair style's first force evaluation, the output of step 0);
 * Verlet::run's loop -- fix nve's kicks and drift (fix_nve.cpp:62-219), list
 * rebuilds on the deck's neigh_modify rule, pair forces, nodal assembly,
 * fix langevin/b200 and fix deform/b200 -- runs on the device, and the
 * reference's own Output writes every thermo and dump step from device
 * read-outs (compute temp/b200 in place of thermo_temp, the pair's global
 * tallies); the state comes back into the reference's arrays at dump steps
 * and at the end of the run.  So a deck that says
 *
 *     run_style verlet/b200
 *     run N
 *
 * with fix nve and a /b200 pair style runs device-resident with the
 * reference's own run command.
 */
#ifdef INTEGRATE_CLASS

IntegrateStyle(verlet/b200, VerletB200)

#else

#ifndef CAC_VERLET_B200_H
#define CAC_VERLET_B200_H

#include "verlet.h"

namespace CAC_NS {

class VerletB200 : public Verlet {
 public:
  VerletB200(class CAC *, int, char **);
  void init() override;
  void run(int, int) override;
};

}  // namespace CAC_NS

#endif
#endif
