/*
 * Oracle read-out commands compiled into the CAC reference executable
 * (test infrastructure only; built by oracle/Makefile into oracle/_ref/).
 *
 *   oracle_dump FILE state     atoms and nodes as they are now (x, v, f, gaussf)
 *   oracle_dump FILE compute   rebuild ghosts and lists exactly as
 *                              Verlet::setup does (verlet.cpp:64-152), evaluate
 *                              the pair style with global+per-atom energy and
 *                              virial, fold ghost contributions into owners,
 *                              assemble nodal forces, then dump
 *   oracle_dump_neigh FILE [binary]
 *                              dump the pair style's neighbour list as
 *                              canonical keys (atom tag or element tag + lattice
 *                              site) with the periodic image of every neighbour;
 *                              binary: sorted rows of 7 int32 (i-site, j kind,
 *                              j tag-1, j site, sx, sy, sz) for large systems
 */
#ifdef COMMAND_CLASS

CommandStyle(oracle_dump, OracleDump)
CommandStyle(oracle_dump_neigh, OracleDumpNeigh)

#else

#ifndef CACB200_ORACLE_DUMP_H
#define CACB200_ORACLE_DUMP_H

#include "pointers.h"

namespace CAC_NS {

class OracleDump : protected Pointers {
 public:
  OracleDump(class CAC *);
  void command(int, char **);

 private:
  void setup_and_compute();
  void write(const char *file, int with_energy, int binary);
};

class OracleDumpNeigh : protected Pointers {
 public:
  OracleDumpNeigh(class CAC *);
  void command(int, char **);
};

}  // namespace CAC_NS

#endif
#endif
