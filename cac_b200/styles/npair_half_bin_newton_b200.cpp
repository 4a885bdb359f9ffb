#include "npair_half_bin_newton_b200.h"

#include "b200_bridge.h"
#include "force.h"
#include "neigh_list.h"
#include "neigh_request.h"
#include "pair.h"
#include "update.h"

using namespace CAC_NS;

bool CAC_NS::b200_device_list_request(NeighRequest *rq)
{
  // the /b200 pair styles make their requests with their Pair subobject
  return rq && rq->pair && rq->requestor && b200_bridge_of(static_cast<Pair *>(rq->requestor)) != nullptr;
}

NPairHalfBinNewtonB200::NPairHalfBinNewtonB200(CAC *cac) : NPair(cac) {}

void NPairHalfBinNewtonB200::build(NeighList *list)
{
  B200Bridge *b = force->pair ? b200_bridge_of(force->pair) : nullptr;
  // inside run / minimize (update->whichflag 1 or 2) the device's own lists
  // serve the pair style; the host list stays empty
  if (update->whichflag != 0 || b == nullptr) {
    list->inum = list->ainum = list->einum = list->ginum = list->ninum = 0;
    return;
  }
  b->fill_host_list(list);
}
