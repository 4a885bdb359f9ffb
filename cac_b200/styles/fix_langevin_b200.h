/*
 * fix ID all langevin/b200 Tstart Tstop damp seed [zero yes|no]: FixLangevin
 * (fix_langevin.cpp) unchanged inside the reference's own loop, plus what
 * run_b200 needs to apply the same thermostat on the device: its settings
 * and how many draws its RanMars generator has made, so that the device
 * continues that stream; after run_b200 the host generator is advanced past
 * the device's draws, so a later `run` continues the stream too.
 */
#ifdef FIX_CLASS

FixStyle(langevin/b200, FixLangevinB200)

#else

#ifndef CAC_FIX_LANGEVIN_B200_H
#define CAC_FIX_LANGEVIN_B200_H

#include "fix_langevin.h"

namespace CAC_NS {

class FixLangevinB200 : public FixLangevin {
 public:
  FixLangevinB200(class CAC *, int, char **);
  void post_force(int) override;

  // settings for the device (constant target ramp only)
  bool device_ok() const { return tstr == nullptr && igroup == 0; }
  double start() const { return t_start; }
  double stop() const { return t_stop; }
  double damp() const { return t_period; }
  int seed_value() const { return seed; }
  int zero() const { return zeroflag; }

  // uniform() calls made by the generator, its construction included
  long long draws = 1;
  // draws of one post_force over the current atoms and elements
  long long draws_per_call() const;
  // advance the host generator by n draws
  void advance(long long n);
};

}  // namespace CAC_NS

#endif
#endif
