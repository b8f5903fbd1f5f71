// Device form of the production/loss rates (sources.f90): one thread per interior cell for
// the continuity chemistry, one per (cell, species) for the energy and momentum exchange,
// running the bodies of gem_rates.cuh, behind the C ABI (include/gem_fluid.h).  Included by
// gem_fluid.cu (one translation unit with the plain path).

#include "gem_rates.cuh"

namespace gemk {

struct RateIn {  // interior neutral inputs
  const double *nn, *vn1, *vn2, *vn3, *Tn;
};

__global__ void kr_continuity(gemr::View v, RateIn in, const double* __restrict__ fv, double* __restrict__ Pr,
                              double* __restrict__ Lo) {
  const long long n = gemr::ncell(v);
  const double *ns = fv, *vs1 = fv + LSP * v.ng, *vs2 = fv + 2 * LSP * v.ng, *vs3 = fv + 3 * LSP * v.ng,
               *Ts = fv + 4 * LSP * v.ng;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
    gemr::continuity_cell(v, c, in.nn, in.vn1, in.vn2, in.vn3, in.Tn, ns, vs1, vs2, vs3, Ts, Pr, Lo);
}

__global__ void kr_energy(gemr::View v, RateIn in, const double* __restrict__ fv, double* __restrict__ Pr,
                          double* __restrict__ Lo) {
  const long long n = gemr::ncell(v) * LSP;
  const double *ns = fv, *vs1 = fv + LSP * v.ng, *vs2 = fv + 2 * LSP * v.ng, *vs3 = fv + 3 * LSP * v.ng,
               *Ts = fv + 4 * LSP * v.ng;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    gemr::energy_rate(v, t, in.nn, in.vn1, in.vn2, in.vn3, in.Tn, ns, vs1, vs2, vs3, Ts, Pr, Lo);
}

__global__ void kr_momentum(gemr::View v, RateIn in, const double* __restrict__ fv, const double* __restrict__ E1,
                            const double* __restrict__ Q, const double* __restrict__ alt,
                            const double* __restrict__ g1, double* __restrict__ Pr, double* __restrict__ Lo) {
  const long long n = gemr::ncell(v) * LSP;
  const double *ns = fv, *vs1 = fv + LSP * v.ng, *vs2 = fv + 2 * LSP * v.ng, *vs3 = fv + 3 * LSP * v.ng,
               *Ts = fv + 4 * LSP * v.ng;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    gemr::momentum_rate(v, t, in.nn, in.vn1, in.Tn, ns, vs1, vs2, vs3, Ts, E1, Q, alt, g1, Pr, Lo);
}

gemr::View rate_view(const gem_grid* g) {
  const GridDev& G = g->dev;
  const Dims& d = G.d;
  gemr::View v;
  v.lx1 = d.lx1;
  v.lx2 = d.lx2;
  v.lx3 = d.lx3;
  v.s2 = d.s2;
  v.s3 = d.s3;
  v.ng = d.ng;
  v.c3 = G.c3;
  v.h1 = G.unit ? nullptr : G.h1;
  v.h2 = G.unit ? nullptr : G.h2;
  v.h3 = G.unit ? nullptr : G.h3;
  v.dx1 = G.L[0].dx;
  const double ms[LSP] = {16.0 * AMU, 30.0 * AMU, 28.0 * AMU, 32.0 * AMU, 14.0 * AMU, 1.0 * AMU, 5.485799090e-4 * AMU};
  const double gam[LSP] = {5.0 / 3, 7.0 / 5, 7.0 / 5, 7.0 / 5, 5.0 / 3, 5.0 / 3, 5.0 / 3};
  for (int s = 0; s < LSP; ++s) {
    v.ms[s] = ms[s];
    v.qs[s] = (s < LSP - 1) ? 1.0 * ELCHRG : -1.0 * ELCHRG;
    v.gam[s] = gam[s];
  }
  v.pi = 4 * std::atan(1.0);  // phys_consts.in.f90:20, on the host
  return v;
}

}  // namespace gemk

extern "C" {

int gem_srcs_continuity_dev(const gem_grid* g, const double* nn, const double* vn1, const double* vn2,
                            const double* vn3, const double* Tn, const double* fluidvars, double* Pr, double* Lo,
                            void* stream) {
  if (check_grid(g) || !nn || !vn1 || !vn2 || !vn3 || !Tn || !fluidvars || !Pr || !Lo)
    return set_err(GEM_EINVAL, "null argument");
  const gemr::View v = gemk::rate_view(g);
  const long long n = gemr::ncell(v);
  gemk::kr_continuity<<<grid_for(n, 128), 128, 0, S(stream)>>>(v, gemk::RateIn{nn, vn1, vn2, vn3, Tn}, fluidvars,
                                                                  Pr, Lo);
  GEM_LAUNCHED("kr_continuity");
  return GEM_OK;
}

int gem_srcs_energy_dev(const gem_grid* g, const double* nn, const double* vn1, const double* vn2, const double* vn3,
                        const double* Tn, const double* fluidvars, double* Pr, double* Lo, void* stream) {
  if (check_grid(g) || !nn || !vn1 || !vn2 || !vn3 || !Tn || !fluidvars || !Pr || !Lo)
    return set_err(GEM_EINVAL, "null argument");
  const gemr::View v = gemk::rate_view(g);
  const long long n = gemr::ncell(v) * LSP;
  gemk::kr_energy<<<grid_for(n, 128), 128, 0, S(stream)>>>(v, gemk::RateIn{nn, vn1, vn2, vn3, Tn}, fluidvars, Pr,
                                                              Lo);
  GEM_LAUNCHED("kr_energy");
  return GEM_OK;
}

int gem_srcs_momentum_dev(const gem_grid* g, const double* nn, const double* vn1, const double* Tn,
                          const double* fluidvars, const double* electrovars, const double* Q, const double* alt,
                          const double* g1, double* Pr, double* Lo, void* stream) {
  if (check_grid(g) || !nn || !vn1 || !Tn || !fluidvars || !electrovars || !Q || !alt || !g1 || !Pr || !Lo)
    return set_err(GEM_EINVAL, "null argument");
  if (g->dev.d.lx1 < 2) return set_err(GEM_EINVAL, "the x1 gradients need lx1 >= 2");
  const gemr::View v = gemk::rate_view(g);
  const long long n = gemr::ncell(v) * LSP;
  gemk::kr_momentum<<<grid_for(n, 128), 128, 0, S(stream)>>>(v, gemk::RateIn{nn, vn1, nullptr, nullptr, Tn},
                                                                fluidvars, electrovars, Q, alt, g1, Pr, Lo);
  GEM_LAUNCHED("kr_momentum");
  return GEM_OK;
}

}  // extern "C"
