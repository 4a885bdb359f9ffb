/*
 * pair_style eam/alloy/b200: PairEAMAlloy (pair_eam.cpp:618-1031 with the
 * setfl tables of pair_eam_alloy.cpp:100-240) evaluated on a B200 through the
 * cacb200 C ABI.  Same pair_coeff * * FILE El command; one element.  Energies
 * are the embedding energies on the F(rho) spline row (the reference's
 * compute_fp with its coefficient pointer returned); forces are the
 * reference's.
 */
#ifdef PAIR_CLASS

PairStyle(eam/alloy/b200, PairEAMAlloyB200)

#else

#ifndef CAC_PAIR_EAM_ALLOY_B200_H
#define CAC_PAIR_EAM_ALLOY_B200_H

#include "pair_eam_alloy.h"
#include "b200_bridge.h"

namespace CAC_NS {

class PairEAMAlloyB200 : public PairEAMAlloy {
 public:
  PairEAMAlloyB200(class CAC *);
  ~PairEAMAlloyB200() override;
  void compute(int, int) override;
  void init_style() override;
  B200Bridge *bridge;
};

}  // namespace CAC_NS

#endif
#endif
