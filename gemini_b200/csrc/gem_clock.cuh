// The time-step selection after the CFL step (libgemini_mpi.f90:450-483 dt_select with
// temporal_mpi.f90:27-84 dt_comm on a single rank) as one body for the device and the host:
// clip so that t + dt does not pass the next GLOW output (when flagglow) and then the next
// output, floor at 1e-6, and from the second iteration on (get_it() > 1) grow by at most
// dtscale = 2 (libgemini_mpi.f90:38) over the previous step.  Plain IEEE arithmetic in the
// reference's order, so both builds give the reference's bits.
#pragma once

#ifdef __CUDACC__
#define GEMT_HD __host__ __device__ __forceinline__
#else
#define GEMT_HD inline
#endif

namespace gemt {

GEMT_HD double dt_select(double dtcfl, double t, double tout, double tglowout, int flagglow, long long it,
                         double dtprev) {
  double dt = dtcfl;
  if (flagglow != 0 && t + dt > tglowout) dt = tglowout - t;
  if (t + dt > tout) dt = tout - t;
  dt = (dt > 1e-6) ? dt : 1e-6;
  const double dtscale = 2;
  if (it > 1 && dt / dtprev > dtscale) dt = dtscale * dtprev;
  return dt;
}

}  // namespace gemt
