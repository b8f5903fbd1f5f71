// TEST INFRASTRUCTURE -- not part of the product.  The device dt_select body
// (gemini_b200/csrc/gem_clock.cuh) compiled for the host, so that it can be checked against the
// oracle on a CPU.
#include "../gemini_b200/csrc/gem_clock.cuh"

extern "C" double hc_dt_select(double dtcfl, double t, double tout, double tglowout, int flagglow, long long it,
                               double dtprev) {
  return gemt::dt_select(dtcfl, t, tout, tglowout, flagglow, it, dtprev);
}
