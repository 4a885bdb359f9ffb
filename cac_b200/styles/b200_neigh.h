/*
 * Selection of the /b200 NPair classes (no style registration here, so the
 * reference's neighbor.cpp may include it at file scope).
 *
 * The reference picks one NPair class per list request by matching the
 * request against each class's bit mask (Neighbor::choose_pair,
 * neighbor.cpp:1407-1500; masks neighbor.h:211-232).  The /b200 classes
 * carry one more bit, NP_B200, the bit after the reference's last
 * (NP_NOINNER, 1 << 21), and choose_pair takes them exactly for requests made
 * by a /b200 pair style.  A maintainer adds, in choose_pair after the
 * NP_HALF_FULL test,
 *
 *     if (!b200_device_list_request(rq) != !(mask & NP_B200)) continue;
 *
 * and includes this header in neighbor.cpp.
 */
#ifndef CAC_B200_NEIGH_H
#define CAC_B200_NEIGH_H

#include "neighbor.h"

namespace CAC_NS {

constexpr int NP_B200 = NeighConst::NP_NOINNER << 1;

class NeighRequest;

// true when the request comes from a /b200 pair style
bool b200_device_list_request(NeighRequest *rq);

}  // namespace CAC_NS

#endif
