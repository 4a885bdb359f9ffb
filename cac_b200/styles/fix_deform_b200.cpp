#include "fix_deform_b200.h"

#include "cacb200.h"
#include "domain.h"

using namespace CAC_NS;

namespace {
// FixDeform's style numbering (fix_deform.cpp:28)
enum { R_NONE = 0, R_FINAL, R_DELTA, R_SCALE, R_VEL, R_ERATE, R_TRATE, R_VOLUME, R_WIGGLE, R_VARIABLE };
}  // namespace

FixDeformB200::FixDeformB200(CAC *cac, int narg, char **arg) : FixDeform(cac, narg, arg) {}

int FixDeformB200::device_style(int d, double &a, double &b) const
{
  const Set &s = set[d];
  a = b = 0.0;
  switch (s.style) {
    case R_NONE: return CACB200_DEFORM_NONE;
    case R_FINAL: a = s.flo; b = s.fhi; return CACB200_DEFORM_FINAL;
    case R_DELTA: a = s.dlo; b = s.dhi; return CACB200_DEFORM_DELTA;
    case R_SCALE: a = s.scale; return CACB200_DEFORM_SCALE;
    case R_VEL: a = s.vel; return CACB200_DEFORM_VEL;
    case R_ERATE: a = s.rate; return CACB200_DEFORM_ERATE;
    case R_TRATE: a = s.rate; return CACB200_DEFORM_TRATE;
    case R_VOLUME: return CACB200_DEFORM_VOLUME;
    case R_WIGGLE: a = s.amplitude; b = s.tperiod; return CACB200_DEFORM_WIGGLE;
    default: return -1;
  }
}

bool FixDeformB200::device_ok() const
{
  if (domain->triclinic || igroup != 0) return false;
  for (int d = 3; d < 6; d++)
    if (set[d].style != R_NONE) return false;
  // remap v moves nothing in this reference: the velocity terms of
  // Domain::remap are commented out (domain.cpp:566-633) and the border
  // packing only affects ghost velocities, which no /b200 pair style reads;
  // the device runs it as remap none
  return remapflag == Domain::X_REMAP || remapflag == Domain::NO_REMAP || remapflag == Domain::V_REMAP;
}

int FixDeformB200::remap_x() const { return remapflag == Domain::X_REMAP; }
