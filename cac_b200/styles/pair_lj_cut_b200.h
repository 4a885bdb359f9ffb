/*
 * pair_style lj/cut/b200: PairLJCut (pair_lj_cut.cpp:227-417) evaluated on a
 * B200 through the cacb200 C ABI.  Same settings/coeff commands as lj/cut;
 * no host neighbour list is requested (the device builds its own lists at the
 * steps where the reference reneighbours).
 */
#ifdef PAIR_CLASS

PairStyle(lj/cut/b200, PairLJCutB200)

#else

#ifndef CAC_PAIR_LJ_CUT_B200_H
#define CAC_PAIR_LJ_CUT_B200_H

#include "pair_lj_cut.h"
#include "b200_bridge.h"

namespace CAC_NS {

class PairLJCutB200 : public PairLJCut {
 public:
  PairLJCutB200(class CAC *);
  ~PairLJCutB200() override;
  void compute(int, int) override;
  void init_style() override;
  double init_one(int, int) override;
  B200Bridge *bridge;
};

}  // namespace CAC_NS

#endif
#endif
