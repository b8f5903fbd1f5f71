// Device form of the compression sub-step (app/main.f90:320-338): one thread per index of
// the per-index bodies in gem_compression.cuh, behind the C ABI (include/gem_fluid.h).
// Included by gem_fluid.cu (one translation unit with the plain path).

#include "gem_compression.cuh"

namespace gemk {

__global__ void kc_artvisc(gemc::View v, long long n, const double* __restrict__ ns,
                           const double* __restrict__ vs1, double* __restrict__ Q) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    gemc::artvisc(v, t, ns, vs1, Q);
}
__global__ void kc_rk2_x1(gemc::View v, long long n, double* vs1) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    gemc::rk2_x1(v, t, vs1);
}
__global__ void kc_rk2_x2(gemc::View v, long long n, double* vs1, double* vs2, double* vs3) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    gemc::rk2_x2(v, t, vs1, vs2, vs3);
}
__global__ void kc_rk2_x3(gemc::View v, long long n, double* vs1, double* vs2, double* vs3) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    gemc::rk2_x3(v, t, vs1, vs2, vs3);
}
__global__ void kc_compression(gemc::View v, long long n, const double* __restrict__ vs1,
                               const double* __restrict__ vs2, const double* __restrict__ vs3,
                               const double* __restrict__ Q, double* rhoes, const double* __restrict__ dtp) {
  const double dt = *dtp;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    gemc::cmp(v, t, vs1, vs2, vs3, Q, rhoes, dt);
}

// the View of a grid: device metric tables (null on unit-metric grids) and the species
// constants from the same literal expressions as the device constants
gemc::View cmp_view(const gem_grid* g) {
  const GridDev& G = g->dev;
  const Dims& d = G.d;
  gemc::View v;
  v.lx1 = d.lx1;
  v.lx2 = d.lx2;
  v.lx3 = d.lx3;
  v.flagper = G.flagper;
  v.s2 = d.s2;
  v.s3 = d.s3;
  v.ng = d.ng;
  v.c3 = G.c3;
  v.h1 = G.unit ? nullptr : G.h1;
  v.h2 = G.unit ? nullptr : G.h2;
  v.h3 = G.unit ? nullptr : G.h3;
  v.dx1 = G.L[0].dx;
  v.dx2 = G.L[1].dx;
  v.dx3 = G.L[2].dx;
  const double ms[LSP] = {16.0 * AMU, 30.0 * AMU, 28.0 * AMU, 32.0 * AMU, 14.0 * AMU, 1.0 * AMU, 5.485799090e-4 * AMU};
  const double gam[LSP] = {5.0 / 3, 7.0 / 5, 7.0 / 5, 7.0 / 5, 5.0 / 3, 5.0 / 3, 5.0 / 3};
  for (int s = 0; s < LSP; ++s) {
    v.ms[s] = ms[s];
    v.gm1[s] = gam[s] - 1;
  }
  return v;
}

}  // namespace gemk

extern "C" {

int gem_vnricht_artvisc_dev(const gem_grid* g, const double* fluidvars, double* Q, void* stream) {
  if (check_grid(g) || !fluidvars || !Q) return set_err(GEM_EINVAL, "null argument");
  const gemc::View v = gemk::cmp_view(g);
  const long long n = gemc::ncell(v) * LSP;
  gemk::kc_artvisc<<<grid_for(n, 256), 256, 0, S(stream)>>>(v, n, fluidvars, fluidvars + LSP * v.ng, Q);
  GEM_LAUNCHED("kc_artvisc");
  return GEM_OK;
}

int gem_rk2_global_boundary_allspec_dev(const gem_grid* g, double* fluidvars, void* stream) {
  if (check_grid(g) || !fluidvars) return set_err(GEM_EINVAL, "null argument");
  const gemc::View v = gemk::cmp_view(g);
  double* vs1 = fluidvars + LSP * v.ng;
  double* vs2 = fluidvars + 2 * LSP * v.ng;
  double* vs3 = fluidvars + 3 * LSP * v.ng;
  cudaStream_t st = S(stream);
  const long long n1 = (long long)(v.lx2 + 4) * (v.lx3 + 4) * LSP;
  gemk::kc_rk2_x1<<<grid_for(n1, 256), 256, 0, st>>>(v, n1, vs1);
  GEM_LAUNCHED("kc_rk2_x1");
  const long long n2 = (long long)(v.lx1 + 4) * (v.lx3 + 4) * LSP * 3;
  gemk::kc_rk2_x2<<<grid_for(n2, 256), 256, 0, st>>>(v, n2, vs1, vs2, vs3);
  GEM_LAUNCHED("kc_rk2_x2");
  if (!v.flagper) {
    const long long n3 = (long long)(v.lx1 + 4) * (v.lx2 + 4) * LSP * 3;
    gemk::kc_rk2_x3<<<grid_for(n3, 256), 256, 0, st>>>(v, n3, vs1, vs2, vs3);
    GEM_LAUNCHED("kc_rk2_x3");
  }
  return GEM_OK;
}

int gem_compression_dev(const gem_grid* g, const double* fluidvars, double* fluidauxvars, const double* Q,
                        const double* dt, void* stream) {
  if (check_grid(g) || !fluidvars || !fluidauxvars || !Q || !dt) return set_err(GEM_EINVAL, "null argument");
  const gemc::View v = gemk::cmp_view(g);
  const long long n = gemc::ncell(v) * LSP;
  gemk::kc_compression<<<grid_for(n, 256), 256, 0, S(stream)>>>(v, n, fluidvars + LSP * v.ng,
                                                                  fluidvars + 2 * LSP * v.ng,
                                                                  fluidvars + 3 * LSP * v.ng, Q,
                                                                  fluidauxvars + LSP * v.ng, dt);
  GEM_LAUNCHED("kc_compression");
  return GEM_OK;
}

}  // extern "C"
