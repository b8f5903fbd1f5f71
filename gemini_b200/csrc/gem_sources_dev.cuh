// Device form of the source/loss solves (multifluid.f90:474-549): one thread per cell of the
// ghosted block running the per-cell bodies of gem_sources.cuh, behind the C ABI
// (include/gem_fluid.h).  Included by gem_fluid.cu (one translation unit with the plain path).

#include "gem_sources.cuh"

namespace gemk {

__global__ void ks_mass(gems::View v, double* __restrict__ Pr, const double* __restrict__ Lo,
                        const double* __restrict__ Prprecip, double* __restrict__ ns,
                        const double* __restrict__ dtp) {
  const double dt = *dtp;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < v.ng; k += (long long)gridDim.x * blockDim.x)
    gems::mass_cell(v, k, dt, Pr, Lo, Prprecip, ns);
}
__global__ void ks_momentum(gems::View v, const double* __restrict__ Pr, const double* __restrict__ Lo,
                            const double* __restrict__ ns, double* __restrict__ rhovs1, double* __restrict__ vs1,
                            const double* __restrict__ dtp) {
  const double dt = *dtp;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < v.ng; k += (long long)gridDim.x * blockDim.x)
    gems::momentum_cell(v, k, dt, Pr, Lo, ns, rhovs1, vs1);
}
__global__ void ks_energy(gems::View v, double* __restrict__ Pr, const double* __restrict__ Lo,
                          const double* __restrict__ Qeprecip, double* __restrict__ rhoes, double* __restrict__ Ts,
                          const double* __restrict__ ns, const double* __restrict__ dtp) {
  const double dt = *dtp;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < v.ng; k += (long long)gridDim.x * blockDim.x)
    gems::energy_cell(v, k, dt, Pr, Lo, Qeprecip, rhoes, Ts, ns);
}

gems::View src_view(const gem_grid* g) {
  const Dims& d = g->dev.d;
  gems::View v;
  v.lx1 = d.lx1;
  v.lx2 = d.lx2;
  v.lx3 = d.lx3;
  v.s2 = d.s2;
  v.s3 = d.s3;
  v.ng = d.ng;
  const double ms[LSP] = {16.0 * AMU, 30.0 * AMU, 28.0 * AMU, 32.0 * AMU, 14.0 * AMU, 1.0 * AMU, 5.485799090e-4 * AMU};
  const double gam[LSP] = {5.0 / 3, 7.0 / 5, 7.0 / 5, 7.0 / 5, 5.0 / 3, 5.0 / 3, 5.0 / 3};
  for (int s = 0; s < LSP; ++s) {
    v.ms[s] = ms[s];
    v.qs[s] = (s < LSP - 1) ? 1.0 * ELCHRG : -1.0 * ELCHRG;
    v.gam[s] = gam[s];
  }
  return v;
}

}  // namespace gemk

extern "C" {

int gem_mass_source_loss_solve_dev(const gem_grid* g, const double* dt, double* Pr, const double* Lo,
                                   const double* Prprecip, double* fluidvars, void* stream) {
  if (check_grid(g) || !dt || !Pr || !Lo || !Prprecip || !fluidvars) return set_err(GEM_EINVAL, "null argument");
  const gems::View v = gemk::src_view(g);
  gemk::ks_mass<<<grid_for(v.ng, 256), 256, 0, S(stream)>>>(v, Pr, Lo, Prprecip, fluidvars, dt);
  GEM_LAUNCHED("ks_mass");
  return GEM_OK;
}

int gem_momentum_source_loss_solve_dev(const gem_grid* g, const double* dt, const double* Pr, const double* Lo,
                                       double* fluidvars, double* fluidauxvars, void* stream) {
  if (check_grid(g) || !dt || !Pr || !Lo || !fluidvars || !fluidauxvars) return set_err(GEM_EINVAL, "null argument");
  const gems::View v = gemk::src_view(g);
  gemk::ks_momentum<<<grid_for(v.ng, 256), 256, 0, S(stream)>>>(v, Pr, Lo, fluidvars, fluidauxvars,
                                                                 fluidvars + LSP * v.ng, dt);
  GEM_LAUNCHED("ks_momentum");
  return GEM_OK;
}

int gem_energy_source_loss_solve_dev(const gem_grid* g, const double* dt, double* Pr, const double* Lo,
                                     const double* Qeprecip, double* fluidvars, double* fluidauxvars, void* stream) {
  if (check_grid(g) || !dt || !Pr || !Lo || !Qeprecip || !fluidvars || !fluidauxvars)
    return set_err(GEM_EINVAL, "null argument");
  const gems::View v = gemk::src_view(g);
  gemk::ks_energy<<<grid_for(v.ng, 256), 256, 0, S(stream)>>>(v, Pr, Lo, Qeprecip, fluidauxvars + LSP * v.ng,
                                                               fluidvars + 4 * LSP * v.ng, fluidvars, dt);
  GEM_LAUNCHED("ks_energy");
  return GEM_OK;
}

}  // extern "C"
