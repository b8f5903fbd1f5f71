// Device-resident time stepping: dt_select and the clock update after each step, so that a
// loop of steps needs no host round trip for dt (and can be captured in one CUDA graph).
// Included by gem_fluid.cu.

#include "gem_clock.cuh"

namespace gemk {

__global__ void kt_dt_select(gem_clock* c, int flagglow, double* dt) {
  if (blockIdx.x == 0 && threadIdx.x == 0)
    *dt = gemt::dt_select(c->dtcfl, c->t, c->tout, c->tglowout, flagglow, c->it, *dt);
}

__global__ void kt_clock_advance(gem_clock* c, const double* dt) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    c->t = c->t + *dt;  // app/main.f90:233
    c->it = c->it + 1;
  }
}

}  // namespace gemk

extern "C" {

int gem_dt_select_dev(const gem_cfg* cfg, const gem_grid* g, const double* fluidvars, gem_work* w, gem_clock* clock,
                      double* dt, void* stream) {
  if (!cfg || check_grid(g) || !fluidvars || !w || !clock || !dt) return set_err(GEM_EINVAL, "null argument");
  const int rc = gem_dt_calc_dev(g, cfg->tcfl, fluidvars, w, &clock->dtcfl, stream);
  if (rc != GEM_OK) return rc;
  gemk::kt_dt_select<<<1, 32, 0, S(stream)>>>(clock, cfg->flagglow, dt);
  GEM_LAUNCHED("kt_dt_select");
  return GEM_OK;
}

int gem_clock_advance_dev(gem_clock* clock, const double* dt, void* stream) {
  if (!clock || !dt) return set_err(GEM_EINVAL, "null argument");
  gemk::kt_clock_advance<<<1, 32, 0, S(stream)>>>(clock, dt);
  GEM_LAUNCHED("kt_clock_advance");
  return GEM_OK;
}

}  // extern "C"
