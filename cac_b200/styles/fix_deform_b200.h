/*
 * fix ID all deform/b200 N x|y|z style args ... : FixDeform (fix_deform.cpp)
 * unchanged inside the reference's own loop, plus its per-dimension settings
 * in the package's numbering for run_b200, which applies the same
 * deformation on the device (orthogonal boxes, remap x or none).
 */
#ifdef FIX_CLASS

FixStyle(deform/b200, FixDeformB200)

#else

#ifndef CAC_FIX_DEFORM_B200_H
#define CAC_FIX_DEFORM_B200_H

#include "fix_deform.h"

namespace CAC_NS {

class FixDeformB200 : public FixDeform {
 public:
  FixDeformB200(class CAC *, int, char **);

  // CACB200_DEFORM_* style of dimension d (0..2) with its arguments in box
  // units, or -1 when the device does not offer it (variable styles)
  int device_style(int d, double &a, double &b) const;
  // tilt styles, a triclinic box or remap v
  bool device_ok() const;
  int every() const { return nevery; }
  int remap_x() const;
};

}  // namespace CAC_NS

#endif
#endif
