// Device form of the production/loss rates (sources.f90): one thread per interior cell for
// the continuity chemistry, one per (cell, species) for the energy and momentum exchange
// (a warp per species over 32 cells, the charged pairs shared within the block),
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

// The energy and momentum exchange run one block per 32 interior cells, one warp per
// species (a thread per (cell, species), 32 consecutive cells of one species per warp).  Each of the 21 unordered charged pairs of a cell has its symmetric part (Teff**1.5,
// Phi, Psi) evaluated once, by warp i for the pairs (i, i+1), (i, i+2), (i, i+3) mod 7, and
// shared through shared memory: the bits are those of evaluating it in both threads.
constexpr int kRateCells = 32;
constexpr int kRateThreads = LSP * kRateCells;
constexpr int kPairs = LSP * (LSP - 1) / 2;

struct PairTab {
  double P[kPairs][kRateCells], Phi[kPairs][kRateCells], Psi[kPairs][kRateCells], yP[kPairs][kRateCells];
};

// slot of the unordered pair {i, j}, i != j: owner i with offset d = j - i mod 7 in 1..3
__device__ __forceinline__ int pair_slot(int i, int j) {
  int d = j - i;
  if (d < 0) d += LSP;
  return (d <= 3) ? i * 3 + d - 1 : j * 3 + (LSP - d) - 1;
}

struct SmemPairs {
  const PairTab* tab;
  int lane;
  __device__ __forceinline__ gemr::CoulPair operator()(const gemr::View&, int isp, int isp2, double, double, double,
                                                       double) const {
    const int p = pair_slot(isp, isp2);
    return gemr::CoulPair{tab->P[p][lane], tab->Phi[p][lane], tab->Psi[p][lane], tab->yP[p][lane]};
  }
};

// this thread's three pairs of cell c (ghosted index k), into the table
__device__ __forceinline__ void fill_pairs(const gemr::View& v, int isp, int lane, long long k,
                                           const double* __restrict__ vs1, const double* __restrict__ Ts,
                                           PairTab& tab) {
  const double t1 = Ts[isp * v.ng + k], u1 = vs1[isp * v.ng + k];
#pragma unroll
  for (int d = 1; d <= 3; ++d) {
    const int j = (isp + d < LSP) ? isp + d : isp + d - LSP;
    const gemr::CoulPair q = gemr::coulomb_pair(v, isp, j, t1, Ts[j * v.ng + k], u1, vs1[j * v.ng + k]);
    const int p = isp * 3 + d - 1;
    tab.P[p][lane] = q.P;
    tab.Phi[p][lane] = q.Phi;
    tab.Psi[p][lane] = q.Psi;
    tab.yP[p][lane] = q.yP;
  }
}

// Five 7-warp blocks per SM (56 registers, 112 bytes spilled): 11.2 -> 10.3 ms on the
// 384x192x192 dipole grid against its natural 72 registers and four blocks.
__global__ void __launch_bounds__(kRateThreads, 5) kr_energy(gemr::View v, RateIn in, const double* __restrict__ fv,
                                                          double* __restrict__ Pr, double* __restrict__ Lo) {
  __shared__ PairTab tab;
  const int isp = threadIdx.x / kRateCells, lane = threadIdx.x % kRateCells;
  const long long nc = gemr::ncell(v);
  const long long c = (long long)blockIdx.x * kRateCells + lane;
  const double *ns = fv, *vs1 = fv + LSP * v.ng, *vs2 = fv + 2 * LSP * v.ng, *vs3 = fv + 3 * LSP * v.ng,
               *Ts = fv + 4 * LSP * v.ng;
  if (c < nc) {
    int i1, i2, i3;
    gemr::cell_of(v, c, i1, i2, i3);
    fill_pairs(v, isp, lane, gemr::gix(v, i1, i2, i3), vs1, Ts, tab);
  }
  __syncthreads();
  if (c < nc)
    gemr::energy_rate(v, isp * nc + c, in.nn, in.vn1, in.vn2, in.vn3, in.Tn, ns, vs1, vs2, vs3, Ts, Pr, Lo,
                      SmemPairs{&tab, lane});
}

// x1 log-gradient terms from values the block formed once: the electrons' ambipolar term
// of the cell (shared memory, written by the electron warp) and this species' log(n kB T) at
// the cell and its x1 neighbours (taken by the neighbouring lanes)
struct SharedX1 {
  double epol_v, lm, l0, lp;
  __device__ __forceinline__ double epol(const gemr::View&, const double*, const double*, int, long long, long long,
                                         long long, const gemr::X1Div&) const {
    return epol_v;
  }
  __device__ __forceinline__ double pg(const gemr::View& v, const double*, const double*, long long, int i1, long long,
                                       long long, long long, const gemr::X1Div& q) const {
    return gemr::dx1_line(v, i1, lm, l0, lp, q);
  }
};

// Each lane forms log(n kB T) of its own cell once; a cell's x1 neighbours on the same line
// are the adjacent lanes (c +- 1), except across the block's edges (lanes 0 and 31), which
// form that one neighbour's log themselves.  At the line ends the missing side is the cell
// itself, as the direct form's clamped neighbour index gives.
// Five 7-warp blocks per SM (56 registers, 132 bytes spilled): each SM sub-partition holds a
// quarter of the register file, so at its natural 93 registers (96 allocated) only 5 warps
// fit per sub-partition and two blocks per SM (16.2 ms on the 384x192x192 dipole grid;
// 72 registers, four blocks: 10.1 ms; 56: 9.95 ms).
__global__ void __launch_bounds__(kRateThreads, 5) kr_momentum(gemr::View v, RateIn in, const double* __restrict__ fv,
                                                            const double* __restrict__ E1,
                                                            const double* __restrict__ Q,
                                                            const double* __restrict__ alt,
                                                            const double* __restrict__ g1, double* __restrict__ Pr,
                                                            double* __restrict__ Lo) {
  __shared__ PairTab tab;
  __shared__ double s_epol[kRateCells];
  const int isp = threadIdx.x / kRateCells, lane = threadIdx.x % kRateCells;
  const long long nc = gemr::ncell(v);
  const long long c = (long long)blockIdx.x * kRateCells + lane;
  const bool ok = c < nc;
  const double *ns = fv, *vs1 = fv + LSP * v.ng, *vs2 = fv + 2 * LSP * v.ng, *vs3 = fv + 3 * LSP * v.ng,
               *Ts = fv + 4 * LSP * v.ng;
  const long long s0 = (long long)isp * v.ng;
  int i1 = 1, i2 = 1, i3 = 1;
  long long kg = 0;
  double l0 = 0.0;
  if (ok) {
    gemr::cell_of(v, c, i1, i2, i3);
    kg = gemr::gix(v, i1, i2, i3);
    fill_pairs(v, isp, lane, kg, vs1, Ts, tab);
    l0 = log(ns[s0 + kg] * gemr::KB_ * Ts[s0 + kg]);
  }
  double lm = __shfl_up_sync(0xffffffffu, l0, 1), lp = __shfl_down_sync(0xffffffffu, l0, 1);
  if (ok) {
    if (i1 == 1) lm = l0;
    if (i1 == v.lx1) lp = l0;
    const bool edge_m = lane == 0 && i1 > 1, edge_p = lane == kRateCells - 1 && i1 < v.lx1;
    if (edge_m || edge_p) {
      const long long kk = gemr::gix(v, edge_m ? i1 - 1 : i1 + 1, i2, i3);
      const double x = log(ns[s0 + kk] * gemr::KB_ * Ts[s0 + kk]);
      if (edge_m)
        lm = x;
      else
        lp = x;
    }
    if (isp == LSP - 1)
      s_epol[lane] = gemr::KB_ * Ts[s0 + kg] / v.qs[LSP - 1] *
                     gemr::dx1_line(v, i1, lm, l0, lp, gemr::x1_div(v, i1, i2, i3));
  }
  __syncthreads();
  if (ok)
    gemr::momentum_rate(v, isp * nc + c, in.nn, in.vn1, in.Tn, ns, vs1, vs2, vs3, Ts, E1, Q, alt, g1, Pr, Lo,
                        SmemPairs{&tab, lane}, SharedX1{s_epol[lane], lm, l0, lp});
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
  v.yh1 = G.unit ? nullptr : G.yh1;
  v.dx1 = G.L[0].dx;
  const double ms[LSP] = {16.0 * AMU, 30.0 * AMU, 28.0 * AMU, 32.0 * AMU, 14.0 * AMU, 1.0 * AMU, 5.485799090e-4 * AMU};
  const double gam[LSP] = {5.0 / 3, 7.0 / 5, 7.0 / 5, 7.0 / 5, 5.0 / 3, 5.0 / 3, 5.0 / 3};
  for (int s = 0; s < LSP; ++s) {
    v.ms[s] = ms[s];
    v.qs[s] = (s < LSP - 1) ? 1.0 * ELCHRG : -1.0 * ELCHRG;
    v.gam[s] = gam[s];
  }
  v.pi = 4 * std::atan(1.0);  // phys_consts.in.f90:20, on the host
  // the divisors ms_i + mn_j and ms_i + ms_j exactly as the device forms them
  const double mn[gemr::NNEU] = {16 * gemr::AMU_, 28 * gemr::AMU_, 32 * gemr::AMU_, 1 * gemr::AMU_};  // Coll::mn
  for (int i = 0; i < LSP; ++i) {
    for (int j = 0; j < gemr::NNEU; ++j) v.ymn[i][j] = 1.0 / (v.ms[i] + mn[j]);
    for (int j = 0; j < LSP; ++j) v.yms[i][j] = 1.0 / (v.ms[i] + v.ms[j]);
  }
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
  const long long nb = (gemr::ncell(v) + gemk::kRateCells - 1) / gemk::kRateCells;
  gemk::kr_energy<<<(unsigned)nb, gemk::kRateThreads, 0, S(stream)>>>(v, gemk::RateIn{nn, vn1, vn2, vn3, Tn}, fluidvars, Pr,
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
  const long long nb = (gemr::ncell(v) + gemk::kRateCells - 1) / gemk::kRateCells;
  gemk::kr_momentum<<<(unsigned)nb, gemk::kRateThreads, 0, S(stream)>>>(v, gemk::RateIn{nn, vn1, nullptr, nullptr, Tn},
                                                                fluidvars, electrovars, Q, alt, g1, Pr, Lo);
  GEM_LAUNCHED("kr_momentum");
  return GEM_OK;
}

}  // extern "C"
