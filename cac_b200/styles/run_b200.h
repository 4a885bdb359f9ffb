/*
 * run_b200 N: N steps of velocity Verlet (Verlet::run with fix nve,
 * verlet.cpp:218-360, fix_nve.cpp:62-219) entirely on the device for the
 * system of the current /b200 pair style; lists are rebuilt at the reference's
 * neigh_modify every interval.  Positions, velocities and forces are copied
 * back into the reference's arrays at the end and the step counter advances.
 *
 * write_b200_neighbor FILE half|full: the device's neighbour list in the
 * canonical text form (tags, lattice site, periodic image) for comparison
 * with the reference's own list.
 *
 * run_style STYLE: choose the integrator of later runs (verlet, verlet/b200).
 */
#ifdef COMMAND_CLASS

CommandStyle(run_b200, RunB200)
CommandStyle(write_b200_neighbor, WriteB200Neighbor)
CommandStyle(run_style, RunStyle)

#else

#ifndef CAC_RUN_B200_H
#define CAC_RUN_B200_H

#include "pointers.h"

namespace CAC_NS {

struct B200Fixes;
class FixLangevinB200;

// The fixes a device run applies besides fix nve (fix langevin/b200, fix
// deform/b200) into `fx`; the langevin/b200 fix (to advance its generator
// after the run) or null.  `who` names the command in errors.
FixLangevinB200 *b200_device_fixes(class CAC *cac, const char *who, B200Fixes &fx);

class RunB200 : protected Pointers {
 public:
  RunB200(class CAC *cac) : Pointers(cac) {}
  void command(int, char **);
};

class WriteB200Neighbor : protected Pointers {
 public:
  WriteB200Neighbor(class CAC *cac) : Pointers(cac) {}
  void command(int, char **);
};

// run_style STYLE [args]: the integrator the next runs use, by its
// IntegrateStyle name (Update::create_integrate, update.cpp:301); the
// reference registers integrators (style_integrate.h) but reads no command
// that selects one, so its runs are always verlet.  run_style verlet/b200
// puts the device loop under the reference's run command.
class RunStyle : protected Pointers {
 public:
  RunStyle(class CAC *cac) : Pointers(cac) {}
  void command(int, char **);
};

}  // namespace CAC_NS

#endif
#endif
