/*
 * pair_style lj/cut/fulllist: the reference's lj/cut evaluated over the full
 * neighbour list (NPairFullBin, npair_full_bin.cpp:23-358) instead of the
 * half list.  Test infrastructure only: it exposes the reference's full list
 * to oracle_dump_neigh, and its forces (each site sums every neighbour, no
 * reaction) cross-check the half-list forces of lj/cut.
 */
#ifdef PAIR_CLASS

PairStyle(lj/cut/fulllist, PairLJCutFullList)

#else

#ifndef CACB200_PAIR_LJ_CUT_FULLLIST_H
#define CACB200_PAIR_LJ_CUT_FULLLIST_H

#include "pair_lj_cut.h"

namespace CAC_NS {

class PairLJCutFullList : public PairLJCut {
 public:
  PairLJCutFullList(class CAC *cac) : PairLJCut(cac) {}
  void init_style() override;
  void compute(int, int) override;
};

}  // namespace CAC_NS

#endif
#endif
