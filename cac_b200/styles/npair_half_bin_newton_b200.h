/*
 * NPair half/bin/newton/b200: the half list of a /b200 pair style, in place
 * of NPairHalfBinNewton (npair_half_bin_newton.cpp:25-392, mask
 * npair_half_bin_newton.h:3-6) with the NP_B200 bit added (b200_neigh.h).
 *
 * The device builds its own lists (the same sets as the reference's, bit for
 * bit) whenever the pair style evaluates forces, so inside a run or a
 * minimisation this class stores nothing on the host and the reference's
 * list build costs only its binning.  Outside one -- a command that builds
 * the list and reads it, such as the reference's write_dump_neighbor_debug
 * -- it fills the host NeighList from the device's half list, with the
 * reference's local and ghost indices and its site order (atoms, then each
 * element's Gauss points).  The order of the neighbours within one site's
 * list is the device's.
 */
#ifdef NPAIR_CLASS

// mask: NPairHalfBinNewton's plus NP_B200 (= NP_NOINNER << 1, b200_neigh.h)
NPairStyle(half/bin/newton/b200,
           NPairHalfBinNewtonB200,
           NP_HALF | NP_BIN | NP_NEWTON |
           NP_ORTHO | NP_ATOM | NP_GAUSS | (NP_NOINNER << 1))

#else

#ifndef CAC_NPAIR_HALF_BIN_NEWTON_B200_H
#define CAC_NPAIR_HALF_BIN_NEWTON_B200_H

#include "npair.h"
#include "b200_neigh.h"

namespace CAC_NS {

class NPairHalfBinNewtonB200 : public NPair {
 public:
  NPairHalfBinNewtonB200(class CAC *);
  ~NPairHalfBinNewtonB200() override {}
  void build(class NeighList *) override;
};

}  // namespace CAC_NS

#endif
#endif
