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
 */
#ifdef COMMAND_CLASS

CommandStyle(run_b200, RunB200)
CommandStyle(write_b200_neighbor, WriteB200Neighbor)

#else

#ifndef CAC_RUN_B200_H
#define CAC_RUN_B200_H

#include "pointers.h"

namespace CAC_NS {

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

}  // namespace CAC_NS

#endif
#endif
