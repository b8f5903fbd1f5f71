// Device code of the B200 fluid-advance library: the MC-limited advection sweeps, the
// ghost fill that replaces the MPI halo, the state conversions / clean_param epilogues, the
// warp-parallel TRBDF2 field-aligned diffusion and the CFL reduction.
//
// Layout: the reference's Fortran blocks (x1 fastest, 2 ghosts per side, species slowest),
// so a Fortran or C caller's cudaMalloc'd blocks are used in place.
//
// Arithmetic: the advection, ghost fill, conversions and clean-up reproduce the reference's
// operation order exactly (compiled with -fmad=false; IEEE division and sqrt), so for
// identical inputs they are bit-identical to the Fortran routines they restate.  The
// diffusion assembles the same coefficients with reordered divisions and solves the
// tridiagonal systems without pivoting; its results agree with an extended-precision
// solution of the reference's discrete equations to ~1e-13 relative.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "gem_diffusion_lu.cuh"

namespace gemk {

constexpr int LSP = 7;
constexpr double KB = 1.38064852e-23;     // phys_consts.in.f90:24
constexpr double ELCHRG = 1.60217662e-19;  // phys_consts.in.f90:25
constexpr double AMU = 1.660539040e-27;    // phys_consts.in.f90:26
constexpr double MINDENS = 1.0e-100;       // phys_consts.in.f90:82-84
constexpr double MINDENSNULL = 1.0e-20;
constexpr double MINDENSDIV = 1.0e-5;

// phys_consts.in.f90:43-53; collisions.f90:51-53 (default-REAL literals widened)
__constant__ double c_ms[LSP] = {16.0 * AMU, 30.0 * AMU, 28.0 * AMU, 32.0 * AMU,
                                 14.0 * AMU, 1.0 * AMU,  5.485799090e-4 * AMU};
// correctly rounded reciprocals of the masses (constant-folded in IEEE double)
__constant__ double c_yms[LSP] = {1.0 / (16.0 * AMU), 1.0 / (30.0 * AMU), 1.0 / (28.0 * AMU),
                                  1.0 / (32.0 * AMU), 1.0 / (14.0 * AMU), 1.0 / (1.0 * AMU),
                                  1.0 / (5.485799090e-4 * AMU)};
__constant__ double c_qs[LSP] = {1.0 * ELCHRG, 1.0 * ELCHRG, 1.0 * ELCHRG, 1.0 * ELCHRG,
                                 1.0 * ELCHRG, 1.0 * ELCHRG, -1.0 * ELCHRG};
__constant__ double c_gammas[LSP] = {5.0 / 3, 7.0 / 5, 7.0 / 5, 7.0 / 5, 5.0 / 3, 5.0 / 3, 5.0 / 3};
// gammas-1, (gammas-1)/kB and the electron charge with its correctly rounded reciprocal,
// each the IEEE value of the expression (constant-folded in double), so a kernel reading one
// gets the bits its runtime evaluation would give
#define GEM_G53 (5.0 / 3 - 1)
#define GEM_G75 (7.0 / 5 - 1)
__constant__ double c_gm1[LSP] = {GEM_G53, GEM_G75, GEM_G75, GEM_G75, GEM_G53, GEM_G53, GEM_G53};
__constant__ double c_gm1kb[LSP] = {GEM_G53 / KB, GEM_G75 / KB, GEM_G75 / KB, GEM_G75 / KB,
                                    GEM_G53 / KB, GEM_G53 / KB, GEM_G53 / KB};
constexpr double QE = -1.0 * ELCHRG;
constexpr double YQE = 1.0 / (-1.0 * ELCHRG);
__constant__ double c_tcoef[LSP - 1] = {(double)0.1019e-12f, (double)0.0747e-12f,
                                        (double)0.0754e-12f, (double)0.0701e-12f,
                                        (double)0.1068e-12f, (double)0.3986e-12f};

struct Dims {
  int lx1, lx2, lx3;
  long long s2, s3, ng;
};

inline Dims make_dims(int lx1, int lx2, int lx3) {
  Dims d;
  d.lx1 = lx1;
  d.lx2 = lx2;
  d.lx3 = lx3;
  d.s2 = lx1 + 4;
  d.s3 = (long long)(lx1 + 4) * (lx2 + 4);
  d.ng = d.s3 * (lx3 + 4);
  return d;
}

// ghosted (-1:lx1+2,-1:lx2+2,-1:lx3+2)
__device__ __forceinline__ long long gi(const Dims& d, int i1, int i2, int i3) {
  return (long long)(i1 + 1) + d.s2 * (i2 + 1) + d.s3 * (i3 + 1);
}
// interior (1:lx1,1:lx2,1:lx3)
__device__ __forceinline__ long long ci(const Dims& d, int i1, int i2, int i3) {
  return (long long)(i1 - 1) + (long long)d.lx1 * ((i2 - 1) + (long long)d.lx2 * (i3 - 1));
}
__host__ __device__ __forceinline__ long long nci(const Dims& d) { return (long long)d.lx1 * d.lx2 * d.lx3; }
// faces
__device__ __forceinline__ long long f1i(const Dims& d, int i1, int i2, int i3) {
  return (long long)(i1 - 1) + (long long)(d.lx1 + 1) * ((i2 - 1) + (long long)d.lx2 * (i3 - 1));
}
__host__ __device__ __forceinline__ long long nf1(const Dims& d) { return (long long)(d.lx1 + 1) * d.lx2 * d.lx3; }
__device__ __forceinline__ long long f2i(const Dims& d, int i1, int i2, int i3) {
  return (long long)(i1 - 1) + (long long)d.lx1 * ((i2 - 1) + (long long)(d.lx2 + 1) * (i3 - 1));
}
__host__ __device__ __forceinline__ long long nf2(const Dims& d) { return (long long)d.lx1 * (d.lx2 + 1) * d.lx3; }
__device__ __forceinline__ long long f3i(const Dims& d, int i1, int i2, int i3) {
  return (long long)(i1 - 1) + (long long)d.lx1 * ((i2 - 1) + (long long)d.lx2 * (i3 - 1));
}
__host__ __device__ __forceinline__ long long nf3(const Dims& d) { return (long long)d.lx1 * d.lx2 * (d.lx3 + 1); }

// Block coordinate of a kernel body: the launch's own blockIdx / gridDim for the plain
// kernels, or the (block, per-instance grid extent) of a work item for the batched ones.
struct VB {
  int bx, by, gx;
};

// 1-D tables of one sweep direction (meshobj.f90:356-389 differences and their correctly
// rounded reciprocals, for the exact reciprocal-corrected division mdiv below)
struct Line1D {
  const double *dx, *ydx;    // dx(j), j = 0..l+2, at [j]
  const double *dxs, *ydxs;  // dx(j) + dx(j+1), j = 0..l+1, at [j]
  const double *dxi, *ydxi;  // dxi(j), j = 1..l, at [j-1]
};

// face tables of one sweep direction: ha2i for frank 0 and 1, the advected-direction metric
// h1i and its reciprocal (advec.f90:302-304, 333-340, 369-376).  Face (i1,i2,i3) of the
// family is at (i1-1)*t1 + (i2-1)*t2 + (i3-1)*t3.
struct FaceTab {
  const double *ha2i0, *ha2i1, *hc, *yhc;
  long long t1, t2, t3;
};

struct GridDev {
  Dims d;
  int gridflag, flagper, unit, has_null;
  long long c3;  // x3 stride of the cell metric tables: d.s3, or 0 when they do not vary in x3
  Line1D L[3];
  const double *h1, *h2, *h3, *yh1;               // cell metric factors (ghosted), 1/h1
  const double *ha1_0, *ha1_1, *yha1_0, *yha1_1;  // h1*h2*h3, h1*h1*h2*h3 and reciprocals
  const double *dl[3], *ydl[3];                   // dx{d}i*h{d} per cell and reciprocals
  int dl3_tab;                                    // dl[2]/ydl[2] present (else formed in the kernel)
  FaceTab F[3];
  const unsigned char* nullpts;
};

// cell metric index (ghosted indices; x3 stride 0 for x3-invariant metrics)
__device__ __forceinline__ long long cmi(const GridDev& G, int i1, int i2, int i3) {
  return (long long)(i1 + 1) + G.d.s2 * (i2 + 1) + G.c3 * (i3 + 1);
}
__device__ __forceinline__ long long fmi(const FaceTab& F, int i1, int i2, int i3) {
  return (long long)(i1 - 1) * F.t1 + (long long)(i2 - 1) * F.t2 + (long long)(i3 - 1) * F.t3;
}

// Metric loads; UNIT grids return exactly 1 (products with 1 are exact, results match).
template <bool UNIT>
__device__ __forceinline__ double ldm(const double* p, long long k) {
  if (UNIT) return 1.0;
  return __ldg(p + k);
}

// a/b from y = RN(1/b) with one exact correction (Markstein's theorem): q0 = RN(a*y),
// r = a - b*q0 (exact with fma), q = RN(q0 + r*y) equals the IEEE quotient RN(a/b) as long
// as nothing over- or underflows, which |a| in (2^-500, 2^500) and |y| in [2^-400, 2^400]
// guarantee (q0 and the remainder stay normal).  Every y mdiv receives comes from a grid
// table that gem_grid_create has checked to lie in [2^-400, 2^400] (or is 1), so only the
// numerator's exponent is tested (integer pipe).  A zero numerator returns q0 = a*y, the
// correctly signed zero of a/b; anything else out of range takes the IEEE division.
__device__ __noinline__ double slow_div(double a, double b) { return a / b; }
__device__ __forceinline__ double mdiv(double a, double b, double y) {
  const double q0 = a * y;
  const double r = __fma_rn(-q0, b, a);
  const double q1 = __fma_rn(r, y, q0);
  const unsigned ha = (unsigned)__double2hiint(a) & 0x7fffffffu;
  if (ha - (523u << 20) < (1000u << 20)) return q1;
  if (a == 0.0) return q0;
  return slow_div(a, b);
}

// mdiv without the fallback: clears ok when the quotient must be recomputed as a/b
__device__ __forceinline__ double mdiv_try(double a, double b, double y, bool& ok) {
  const double q0 = a * y;
  const double r = __fma_rn(-q0, b, a);
  const double q1 = __fma_rn(r, y, q0);
  const unsigned ha = (unsigned)__double2hiint(a) & 0x7fffffffu;
  const unsigned hy = (unsigned)__double2hiint(y) & 0x7fffffffu;
  const bool zero = a == 0.0;
  ok = ok && (hy - (623u << 20) < (800u << 20)) && ((ha - (523u << 20) < (1000u << 20)) || zero);
  return zero ? q0 : q1;
}

__device__ __forceinline__ bool is_null(const GridDev& G, int i1, int i2, int i3) {
  return G.has_null && G.nullpts[ci(G.d, i1, i2, i3)];
}

// advec.f90:438-447
__device__ __forceinline__ double minmod(double a, double b) {
  if (a * b <= 0.0) return 0.0;
  if (fabs(a) < fabs(b)) return a;
  return b;
}
__device__ __forceinline__ double fmin_f(double a, double b) { return (a < b) ? a : b; }
__device__ __forceinline__ double fmax_f(double a, double b) { return (a > b) ? a : b; }

// fluidvar_pointers / fluidauxvar_pointers (libgemini.f90:462-500)
struct Blocks {
  double* F;  // fluidvars
  double* A;  // fluidauxvars
  long long ng;
  __device__ __forceinline__ double* ns(int s) const { return F + (long long)s * ng; }
  __device__ __forceinline__ double* vs1(int s) const { return F + (long long)(LSP + s) * ng; }
  __device__ __forceinline__ double* vs2(int s) const { return F + (long long)(2 * LSP + s) * ng; }
  __device__ __forceinline__ double* vs3(int s) const { return F + (long long)(3 * LSP + s) * ng; }
  __device__ __forceinline__ double* Ts(int s) const { return F + (long long)(4 * LSP + s) * ng; }
  __device__ __forceinline__ double* rv(int s) const { return A + (long long)s * ng; }
  __device__ __forceinline__ double* re(int s) const { return A + (long long)(LSP + s) * ng; }
};

// v12rhov1 and T2rhoe on one value (multifluid.f90:193-214)
__device__ __forceinline__ double conv_rv(double n, double v1, int s) { return n * c_ms[s] * v1; }
__device__ __forceinline__ double conv_re(double n, double T, int s) { return n * KB * T / c_gm1[s]; }

// ======================================================================================
// 2. Elementwise conversions over the full ghosted arrays (multifluid.f90:179-233)
// ======================================================================================
__global__ void k_v12rhov1(Blocks B) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < B.ng;
       k += (long long)gridDim.x * blockDim.x)
    for (int s = 0; s < LSP; ++s) B.rv(s)[k] = conv_rv(B.ns(s)[k], B.vs1(s)[k], s);
}

__global__ void k_T2rhoe(Blocks B) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < B.ng;
       k += (long long)gridDim.x * blockDim.x)
    for (int s = 0; s < LSP; ++s) B.re(s)[k] = conv_re(B.ns(s)[k], B.Ts(s)[k], s);
}

__global__ void k_rhoe2T(Blocks B) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < B.ng;
       k += (long long)gridDim.x * blockDim.x)
    for (int s = 0; s < LSP; ++s) {
      const double T = c_gm1kb[s] * B.re(s)[k] / fmax_f(B.ns(s)[k], MINDENSDIV);
      B.Ts(s)[k] = fmax_f(T, 100.0);
    }
}

__global__ void k_rhov12v1(Blocks B) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < B.ng;
       k += (long long)gridDim.x * blockDim.x) {
    double chrg = 0.0, nsum = 0.0;
    for (int s = 0; s < LSP - 1; ++s) {
      const double n = B.ns(s)[k];
      const double v = B.rv(s)[k] / (c_ms[s] * fmax_f(n, MINDENSDIV));
      B.vs1(s)[k] = v;
      chrg = chrg + n * c_qs[s] * v;
      nsum = nsum + n;
    }
    B.ns(LSP - 1)[k] = nsum;
    B.vs1(LSP - 1)[k] = mdiv(-1 / fmax_f(nsum, MINDENSDIV), QE, YQE) * chrg;
  }
}

// ======================================================================================
// 3. clean_param (multifluid.f90:553-688)
// ======================================================================================
__device__ __forceinline__ void decode_cell(const Dims& d, long long k, int& i1, int& i2, int& i3) {
  const long long a = k / d.s2;
  i1 = (int)(k - a * d.s2) - 1;
  const long long b = a / (d.lx2 + 4);
  i2 = (int)(a - b * (d.lx2 + 4)) - 1;
  i3 = (int)b - 1;
}

__device__ __forceinline__ bool is_ghost(const Dims& d, int i1, int i2, int i3) {
  return i1 < 1 || i1 > d.lx1 || i2 < 1 || i2 > d.lx2 || i3 < 1 || i3 > d.lx3;
}

// The ghost shell, enumerated: the four x3 ghost planes (i1 fastest), then the four x2 ghost
// rows of every interior x3 index, then the four x1 ghosts of every interior column --
// nghost(d) = ng - lx1*lx2*lx3 cells, each once.
__device__ __forceinline__ long long nghost(const Dims& d) {
  const long long a1 = d.lx1 + 4, a2 = d.lx2 + 4;
  return 4 * (a1 * a2 + a1 * d.lx3 + (long long)d.lx2 * d.lx3);
}
__device__ __forceinline__ void ghost_cell(const Dims& d, long long q, int& i1, int& i2, int& i3) {
  const long long a1 = d.lx1 + 4, a2 = d.lx2 + 4;
  const long long np = 4 * a1 * a2, nr = 4 * a1 * d.lx3;
  if (q < np) {
    const long long p = q / (a1 * a2), rem = q - p * (a1 * a2);
    i3 = (p < 2) ? (int)p - 1 : d.lx3 + (int)p - 1;
    i2 = (int)(rem / a1) - 1;
    i1 = (int)(rem - (rem / a1) * a1) - 1;
    return;
  }
  q -= np;
  if (q < nr) {
    const long long row = q / a1;
    i1 = (int)(q - row * a1) - 1;
    const int g = (int)(row & 3);
    i2 = (g < 2) ? g - 1 : d.lx2 + g - 1;
    i3 = (int)(row >> 2) + 1;
    return;
  }
  q -= nr;
  const int g = (int)(q & 3);
  const long long col = q >> 2;
  i1 = (g < 2) ? g - 1 : d.lx1 + g - 1;
  i2 = (int)(col % d.lx2) + 1;
  i3 = (int)(col / d.lx2) + 1;
}

// param: the 4-D block of ns (1), vs1 (2) or Ts (3), all lsp species
__global__ void k_clean_elementwise(GridDev G, double* param, int iparm) {
  const Dims d = G.d;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < d.ng;
       k += (long long)gridDim.x * blockDim.x) {
    int i1, i2, i3;
    decode_cell(d, k, i1, i2, i3);
    const bool ghost = is_ghost(d, i1, i2, i3);
    const bool nul = !ghost && is_null(G, i1, i2, i3);
    if (iparm == 1) {
      double acc = 0.0;
      for (int s = 0; s < LSP - 1; ++s) {
        const double v = fmax_f(param[s * d.ng + k], MINDENS);
        param[s * d.ng + k] = v;
        acc = acc + v;
      }
      param[(LSP - 1) * d.ng + k] = acc;
      if (nul)
        for (int s = 0; s < LSP; ++s) param[s * d.ng + k] = (s == 0) ? MINDENSNULL * 1e-2 : MINDENSNULL;
      if (ghost)
        for (int s = 0; s < LSP; ++s) param[s * d.ng + k] = MINDENSDIV;
    } else if (iparm == 2) {
      if (nul)
        for (int s = 0; s < LSP; ++s) param[s * d.ng + k] = 0;
    } else {
      for (int s = 0; s < LSP; ++s) param[s * d.ng + k] = fmax_f(param[s * d.ng + k], 100.0);
      if (nul || ghost)
        for (int s = 0; s < LSP; ++s) param[s * d.ng + k] = 100;
    }
  }
}

// clean_param(2) border fix along field lines (multifluid.f90:614-654), one thread per
// (column, species).  The null-point scan reproduces the reference's loop bounds exactly.
__device__ __forceinline__ void b_clean_vel_edges(const GridDev& G, double* vs1, const VB vb) {
  const Dims d = G.d;
  const long long ncol = (long long)d.lx2 * d.lx3;
  for (long long t = vb.bx * (long long)blockDim.x + threadIdx.x; t < ncol * LSP;
       t += (long long)vb.gx * blockDim.x) {
    const int s = (int)(t / ncol);
    const long long c = t - s * ncol;
    const int i2 = (int)(c % d.lx2) + 1, i3 = (int)(c / d.lx2) + 1;
    double* p = vs1 + s * d.ng;
    if (G.gridflag == 0) {
      int beg = 1;
      while (!is_null(G, beg, i2, i3) && beg < d.lx1) beg = beg + 1;
      int end = beg;
      while (is_null(G, end, i2, i3) && end < d.lx1) end = end + 1;
      if (beg != d.lx1) p[gi(d, beg, i2, i3)] = p[gi(d, beg + 1, i2, i3)];
      if (end != d.lx1) p[gi(d, end, i2, i3)] = p[gi(d, end - 1, i2, i3)];
    } else if (G.gridflag == 1) {
      int end = 1;
      while (!is_null(G, end, i2, i3) && end < d.lx1) end = end + 1;
      if (end != d.lx1) p[gi(d, end, i2, i3)] = p[gi(d, end - 1, i2, i3)];
    }
  }
}

__global__ void k_clean_vel_edges(GridDev G, double* vs1) {
  b_clean_vel_edges(G, vs1, VB{(int)blockIdx.x, (int)blockIdx.y, (int)gridDim.x});
}


// ======================================================================================
// 4. Global-boundary ghost fill (advec.f90:21-149) and the single-grid halo
//    (mpihalo.f90:147-151), split into the reference's three passes so no thread reads a
//    value another thread of the same pass writes:
//      A  x1 ghosts of every source column (column-owned, in-thread order as the reference)
//      B  x2 ghost rows copied from the edge rows (all x1, all x3)
//      C  x3 ghost slabs copied from the edge slabs (non-periodic) or wrapped (periodic)
//    CONV: the fused step has not materialised rhovs1/rhoes yet (v12rhov1/T2rhoe are folded
//    into the passes and into the x3 sweep), so interior momentum/energy values are formed
//    from ns, vs1, Ts on the fly with the reference's conversion arithmetic.
// ======================================================================================
struct GhostSrc {
  // momentum / energy density of species s at a cell, converted or read
  template <bool CONV>
  __device__ __forceinline__ static double rv(const Blocks& B, int s, long long k) {
    if (CONV) return conv_rv(B.ns(s)[k], B.vs1(s)[k], s);
    return B.rv(s)[k];
  }
  template <bool CONV>
  __device__ __forceinline__ static double re(const Blocks& B, int s, long long k) {
    if (CONV) return conv_re(B.ns(s)[k], B.Ts(s)[k], s);
    return B.re(s)[k];
  }
};

// Pass A.  One thread per (column, species).  interior columns get advec.f90:42-79
// (density extrapolation, reflected momentum from the stale v1i, constant-T energy); ghost
// columns (only those later used as sources) get the same statements applied to their
// own values, as the reference's full-slice assignments do.  In CONV mode the column's
// interior momentum/energy values are also materialised for ghost columns (pass B/C read
// them), interior columns keep them implicit.
template <bool CONV>
__device__ __forceinline__ void b_ghost_x1(const GridDev& G, const Blocks& B, const double* __restrict__ vs1i, int lsp, const VB vb) {
  const Dims d = G.d;
  const int n2 = d.lx2 + 4, n3 = d.lx3 + 4;
  const long long ncol = (long long)n2 * n3;
  for (long long t = vb.bx * (long long)blockDim.x + threadIdx.x; t < ncol * lsp;
       t += (long long)vb.gx * blockDim.x) {
    const int s = (int)(t / ncol);
    const long long c = t - s * ncol;
    const int j2 = (int)(c % n2) - 1, j3 = (int)(c / n2) - 1;
    const bool in2 = j2 >= 1 && j2 <= d.lx2, in3 = j3 >= 1 && j3 <= d.lx3;
    const bool interior = in2 && in3;
    // source columns: interior columns, plus x3-ghost columns with interior x2 when the
    // grid is periodic (the x3 copy is skipped there and the x2 copy reads them)
    if (!interior && !(G.flagper && in2 && !in3)) continue;
    double* n = B.ns(s);
    double* rvp = B.rv(s);
    double* rep = B.re(s);
    const double* v1 = B.vs1(s);
    const double msp = c_ms[s];
    const int lx1 = d.lx1;
    auto at = [&](int i1) { return gi(d, i1, j2, j3); };
    if (!interior && CONV) {
      for (int i1 = 1; i1 <= lx1; ++i1) {
        const long long k = at(i1);
        rvp[k] = GhostSrc::rv<true>(B, s, k);
        rep[k] = GhostSrc::re<true>(B, s, k);
      }
    }
    // ---- bottom (advec.f90:42-60)
    {
      double n0, nm1, r0;
      if (interior) {
        const double coeff = n[at(2)] / n[at(3)];
        n0 = fmin_f(coeff * n[at(1)], n[at(1)]);
        nm1 = fmin_f(coeff * n0, n0);
        r0 = 2 * vs1i[(long long)s * nf1(d) + f1i(d, 1, j2, j3)] - v1[at(1)];
      } else {
        n0 = n[at(0)];
        nm1 = n[at(-1)];
        r0 = GhostSrc::rv<CONV>(B, s, at(0));
      }
      const double rm1 = r0 + r0 - v1[at(1)];
      n[at(0)] = n0;
      n[at(-1)] = nm1;
      rvp[at(-1)] = rm1 * nm1 * msp;
      rvp[at(0)] = r0 * n0 * msp;
      const double e1 = interior ? GhostSrc::re<CONV>(B, s, at(1)) : rep[at(1)];
      const double Tb = e1 / n[at(1)];
      rep[at(0)] = Tb * n0;
      rep[at(-1)] = Tb * nm1;
    }
    // ---- top (advec.f90:61-79)
    {
      double n1, n2v, r1;
      if (interior) {
        const double coeff = n[at(lx1 - 1)] / n[at(lx1 - 2)];
        n1 = fmin_f(coeff * n[at(lx1)], n[at(lx1)]);
        n2v = fmin_f(coeff * n1, n1);
        r1 = 2 * vs1i[(long long)s * nf1(d) + f1i(d, lx1 + 1, j2, j3)] - v1[at(lx1)];
      } else {
        n1 = n[at(lx1 + 1)];
        n2v = n[at(lx1 + 2)];
        r1 = GhostSrc::rv<CONV>(B, s, at(lx1 + 1));
      }
      const double r2 = r1 + r1 - v1[at(lx1)];
      n[at(lx1 + 1)] = n1;
      n[at(lx1 + 2)] = n2v;
      rvp[at(lx1 + 1)] = r1 * n1 * msp;
      rvp[at(lx1 + 2)] = r2 * n2v * msp;
      const double el = interior ? GhostSrc::re<CONV>(B, s, at(lx1)) : rep[at(lx1)];
      const double Tb = el / n[at(lx1)];
      rep[at(lx1 + 1)] = Tb * n1;
      rep[at(lx1 + 2)] = Tb * n2v;
    }
  }
}

template <bool CONV>
__global__ void k_ghost_x1(GridDev G, Blocks B, const double* __restrict__ vs1i, int lsp) {
  b_ghost_x1<CONV>(G, B, vs1i, lsp, VB{(int)blockIdx.x, (int)blockIdx.y, (int)gridDim.x});
}


// Pass B (advec.f90:83-104): x2 ghost rows := edge rows, for vs2, ns, rhovs1, rhoes, every
// x1 (incl. ghosts) and every x3 (incl. ghosts).  One thread per (i1, i3, species).
template <bool CONV>
__device__ __forceinline__ void b_ghost_x2(const GridDev& G, const Blocks& B, int lsp, const VB vb) {
  const Dims d = G.d;
  const int n1 = d.lx1 + 4, n3 = d.lx3 + 4;
  const long long nrow = (long long)n1 * n3;
  for (long long t = vb.bx * (long long)blockDim.x + threadIdx.x; t < nrow * lsp;
       t += (long long)vb.gx * blockDim.x) {
    const int s = (int)(t / nrow);
    const long long c = t - s * nrow;
    const int i1 = (int)(c % n1) - 1, i3 = (int)(c / n1) - 1;
    const bool src_implicit = CONV && i1 >= 1 && i1 <= d.lx1 && i3 >= 1 && i3 <= d.lx3;
    const long long lo = gi(d, i1, 1, i3), hi = gi(d, i1, d.lx2, i3);
    const double v2l = B.vs2(s)[lo], v2h = B.vs2(s)[hi];
    const double nl = B.ns(s)[lo], nh = B.ns(s)[hi];
    const double rl = src_implicit ? GhostSrc::rv<true>(B, s, lo) : B.rv(s)[lo];
    const double rh = src_implicit ? GhostSrc::rv<true>(B, s, hi) : B.rv(s)[hi];
    const double el = src_implicit ? GhostSrc::re<true>(B, s, lo) : B.re(s)[lo];
    const double eh = src_implicit ? GhostSrc::re<true>(B, s, hi) : B.re(s)[hi];
    for (int g = 0; g < 2; ++g) {
      const long long kl = gi(d, i1, -g, i3), kh = gi(d, i1, d.lx2 + 1 + g, i3);
      B.vs2(s)[kl] = v2l;
      B.ns(s)[kl] = nl;
      B.rv(s)[kl] = rl;
      B.re(s)[kl] = el;
      B.vs2(s)[kh] = v2h;
      B.ns(s)[kh] = nh;
      B.rv(s)[kh] = rh;
      B.re(s)[kh] = eh;
    }
  }
}

template <bool CONV>
__global__ void k_ghost_x2(GridDev G, Blocks B, int lsp) {
  b_ghost_x2<CONV>(G, B, lsp, VB{(int)blockIdx.x, (int)blockIdx.y, (int)gridDim.x});
}


// Pass C.  Non-periodic (advec.f90:107-132): x3 ghost slabs := edge slabs for vs3, ns,
// rhovs1, rhoes over every x1 and x2.  Periodic with WRAP (the halo_fluidvars self-wrap,
// mpihalo.f90:147-151, lhalo = 2): rows 1:lx2, every x1, for ns, rhovs1, rhoes, vs2, vs3.
// One thread per (i1, i2, species).
template <bool CONV, bool WRAP>
__device__ __forceinline__ void b_ghost_x3(const GridDev& G, const Blocks& B, int lsp, const VB vb) {
  const Dims d = G.d;
  const int n1 = d.lx1 + 4, n2 = d.lx2 + 4;
  const long long nrow = (long long)n1 * n2;
  for (long long t = vb.bx * (long long)blockDim.x + threadIdx.x; t < nrow * lsp;
       t += (long long)vb.gx * blockDim.x) {
    const int s = (int)(t / nrow);
    const long long c = t - s * nrow;
    const int i1 = (int)(c % n1) - 1, i2 = (int)(c / n1) - 1;
    const bool in1 = i1 >= 1 && i1 <= d.lx1, in2 = i2 >= 1 && i2 <= d.lx2;
    if (!WRAP) {
      const bool src_implicit = CONV && in1 && in2;
      const long long lo = gi(d, i1, i2, 1), hi = gi(d, i1, i2, d.lx3);
      const double v3l = B.vs3(s)[lo], v3h = B.vs3(s)[hi];
      const double nl = B.ns(s)[lo], nh = B.ns(s)[hi];
      const double rl = src_implicit ? GhostSrc::rv<true>(B, s, lo) : B.rv(s)[lo];
      const double rh = src_implicit ? GhostSrc::rv<true>(B, s, hi) : B.rv(s)[hi];
      const double el = src_implicit ? GhostSrc::re<true>(B, s, lo) : B.re(s)[lo];
      const double eh = src_implicit ? GhostSrc::re<true>(B, s, hi) : B.re(s)[hi];
      for (int g = 0; g < 2; ++g) {
        const long long kl = gi(d, i1, i2, -g), kh = gi(d, i1, i2, d.lx3 + 1 + g);
        B.vs3(s)[kl] = v3l;
        B.ns(s)[kl] = nl;
        B.rv(s)[kl] = rl;
        B.re(s)[kl] = el;
        B.vs3(s)[kh] = v3h;
        B.ns(s)[kh] = nh;
        B.rv(s)[kh] = rh;
        B.re(s)[kh] = eh;
      }
    } else {
      if (!in2) continue;
      const bool src_implicit = CONV && in1;
      // param(:,1:lx2,-1:0) = param(:,1:lx2,lx3-1:lx3); param(:,1:lx2,lx3+1:lx3+2) = param(:,1:lx2,1:2)
      const int dst[4] = {-1, 0, d.lx3 + 1, d.lx3 + 2};
      const int src[4] = {d.lx3 - 1, d.lx3, 1, 2};
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const long long ks = gi(d, i1, i2, src[q]), kd = gi(d, i1, i2, dst[q]);
        B.ns(s)[kd] = B.ns(s)[ks];
        B.rv(s)[kd] = src_implicit ? GhostSrc::rv<true>(B, s, ks) : B.rv(s)[ks];
        B.re(s)[kd] = src_implicit ? GhostSrc::re<true>(B, s, ks) : B.re(s)[ks];
        B.vs2(s)[kd] = B.vs2(s)[ks];
        B.vs3(s)[kd] = B.vs3(s)[ks];
      }
    }
  }
}

template <bool CONV, bool WRAP>
__global__ void k_ghost_x3(GridDev G, Blocks B, int lsp) {
  b_ghost_x3<CONV, WRAP>(G, B, lsp, VB{(int)blockIdx.x, (int)blockIdx.y, (int)gridDim.x});
}


// Halo wrap only (standalone halo_allparams / halo_fluidvars): rows 1:lx2, all x1.
__global__ void k_halo_wrap(GridDev G, Blocks B, int with_v23) {
  const Dims d = G.d;
  const int n1 = d.lx1 + 4;
  const long long nrow = (long long)n1 * d.lx2;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nrow * LSP;
       t += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(t / nrow);
    const long long c = t - s * nrow;
    const int i1 = (int)(c % n1) - 1, i2 = (int)(c / n1) + 1;
    const int dst[4] = {-1, 0, d.lx3 + 1, d.lx3 + 2};
    const int src[4] = {d.lx3 - 1, d.lx3, 1, 2};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const long long ks = gi(d, i1, i2, src[q]), kd = gi(d, i1, i2, dst[q]);
      B.ns(s)[kd] = B.ns(s)[ks];
      B.rv(s)[kd] = B.rv(s)[ks];
      B.re(s)[kd] = B.re(s)[ks];
      if (with_v23) {
        B.vs2(s)[kd] = B.vs2(s)[ks];
        B.vs3(s)[kd] = B.vs3(s)[ks];
      }
    }
  }
}

// ======================================================================================
// 5. Interface velocities (advec.f90:155-229), standalone form
// ======================================================================================
// One thread per face of the three families (enumerated back to back, 32-bit indices: the
// per-species face counts stay below 2^31), blockIdx.y the species.
__global__ void k_interface_vels(GridDev G, Blocks B, double* vs1i, double* vs2i, double* vs3i) {
  const Dims d = G.d;
  const int n1 = (int)nf1(d), n2 = (int)nf2(d), n3 = (int)nf3(d);
  const int s = blockIdx.y;
  const int per = n1 + n2 + n3;
  for (int q0 = blockIdx.x * blockDim.x + threadIdx.x; q0 < per; q0 += gridDim.x * blockDim.x) {
    int q = q0;
    if (q < n1) {
      const int i1 = q % (d.lx1 + 1) + 1;
      const int r = q / (d.lx1 + 1);
      const int i2 = r % d.lx2 + 1, i3 = r / d.lx2 + 1;
      const double* v = B.vs1(s);
      double val;
      if (i1 >= 2 && i1 <= d.lx1) {
        val = 0.5 * (v[gi(d, i1 - 1, i2, i3)] + v[gi(d, i1, i2, i3)]);
      } else if (i1 == 1) {
        if (G.gridflag == 1)
          val = fmin_f(0.5 * (v[gi(d, 1, i2, i3)] + v[gi(d, 2, i2, i3)]), 0.0);
        else
          val = v[gi(d, 1, i2, i3)];
      } else {
        if (G.gridflag == 0 || G.gridflag == 1)
          val = v[gi(d, d.lx1, i2, i3)];
        else
          val = fmax_f(0.5 * (v[gi(d, d.lx1 - 1, i2, i3)] + v[gi(d, d.lx1, i2, i3)]), 0.0);
      }
      vs1i[(long long)s * n1 + q] = val;
      continue;
    }
    q -= n1;
    if (q < n2) {
      const int i1 = q % d.lx1 + 1;
      const int r = q / d.lx1;
      const int i2 = r % (d.lx2 + 1) + 1, i3 = r / (d.lx2 + 1) + 1;
      const double* v = B.vs2(s);
      vs2i[(long long)s * n2 + q] = 0.5 * (v[gi(d, i1, i2 - 1, i3)] + v[gi(d, i1, i2, i3)]);
      continue;
    }
    q -= n2;
    {
      const int i1 = q % d.lx1 + 1;
      const int r = q / d.lx1;
      const int i2 = r % d.lx2 + 1, i3 = r / d.lx2 + 1;
      const double* v = B.vs3(s);
      vs3i[(long long)s * n3 + q] = 0.5 * (v[gi(d, i1, i2, i3 - 1)] + v[gi(d, i1, i2, i3)]);
    }
  }
}

// ======================================================================================
// 6. The advection sweeps (advec.f90:233-435 through multifluid.f90:49-126).
//
//    Divisions use mdiv with correctly rounded reciprocals of the grid divisors (1-D tables
//    and per-cell/per-face metric tables), so every update is bit-identical to the
//    reference's a/b chain.  Two kernels:
//      k_sweep_march<DIM=2|3>: one thread per (x2 or x3 line, species), a warp covering 32
//        adjacent x1 -- every copy is a coalesced 256-byte row; the thread marches along its
//        line with the running state of its fields in registers, its warp staging the
//        values of step j+4 by cp.async into a shared ring while computing step j, and
//        writes cell j-1 in place.
//      k_sweep_x1: one warp per (x1 column, species), lanes along the contiguous x1, the
//        column processed in chunks of 32 cells with neighbours exchanged by shuffles, the
//        next chunk staged by cp.async into a shared ring while the current one computes.
//    Standalone (FUSED=false): one field set (which: 0 ns, 1 rhovs1 (frank 1), 2 rhoes),
//    interface velocities from the work arrays, ghosts from memory.
//    Fused x3: v12rhov1/T2rhoe folded in, x3 ghosts and vs3i formed on the fly.
//    Fused x1: vs1i formed on the fly (boundary faces stored for the next step), the
//    halo_allparams self-wrap of the swept values written directly.
//    Fused x2: rhov12v1, clean_param(1,2,3) element parts and rhoe2T applied to each
//    finished cell (species exchanged through shared memory).
// ======================================================================================
struct SweepArgs {
  GridDev G;
  Blocks B;
  const double* vsi;  // standalone: vs{dim}i (all species)
  double* vs1i;       // fused x1: boundary faces written here
  const double* dtp;
  double* dtp_w;  // writable alias of dtp (batched dt finalize); unused by the sweeps
  int which;      // standalone field set
};

// Running state of one field while marching j = 0..lx+1 along a line:
//   fp = f(j-1), fc = f(j), ls = lslope, slp = slope(j-1), php = phi(j-1)
struct FieldRun {
  double fp, fc, ls, slp, php;
};

// Face quantities shared by the fields of one species at face j:
//   v = v1i(j), hv = 0.5*v, qp = dx(j) + v/h1i(j)*dt, qm = dx(j) - v/h1i(j)*dt
struct Face {
  double v, hv, qp, qm;
};

__device__ __forceinline__ Face make_face(double v, double hc, double yhc, double dxj, double dt) {
  Face f;
  f.v = v;
  f.hv = 0.5 * v;
  const double q = mdiv(v, hc, yhc) * dt;
  f.qp = dxj + q;
  f.qm = dxj - q;
  return f;
}

// slope(j) (advec.f90:407-414): needs f(j-1), f(j), f(j+1) and lslope = rslope(j-1)
__device__ __forceinline__ double mc_slope(double fm, double f0, double fpl, double ls, const Line1D& L,
                                           int j, double& rs) {
  rs = mdiv(fpl - f0, __ldg(L.dx + j + 1), __ldg(L.ydx + j + 1));
  const double cs = mdiv(fpl - fm, __ldg(L.dxs + j), __ldg(L.ydxs + j));
  return minmod(cs, minmod(2 * ls, 2 * rs));
}

// phi(j) (advec.f90:418-424)
__device__ __forceinline__ double mc_phi(double fjm1, double fj, double sljm1, double slj, const Face& F) {
  if (F.v < 0) return fj * F.v - F.hv * F.qp * slj;
  return fjm1 * F.v + F.hv * F.qm * sljm1;
}

// updated cell value (advec.f90:427): f - dt*(Pr - Pl)/dxi/ha1 with P = ha2i*phi
__device__ __forceinline__ double mc_update(double f, double Pr, double Pl, double dt, double dxi, double ydxi,
                                            double ha1, double yha1) {
  return f - mdiv(mdiv(dt * (Pr - Pl), dxi, ydxi), ha1, yha1);
}

template <bool UNIT>
__device__ __forceinline__ void cell_metric(const GridDev& G, long long k, int frank, double& ha1, double& yha1) {
  if (UNIT) {
    ha1 = 1.0;
    yha1 = 1.0;
  } else if (frank == 0) {
    ha1 = __ldg(G.ha1_0 + k);
    yha1 = __ldg(G.yha1_0 + k);
  } else {
    ha1 = __ldg(G.ha1_1 + k);
    yha1 = __ldg(G.yha1_1 + k);
  }
}

// ---- x2 / x3 sweeps ---------------------------------------------------------------------
// asynchronous global -> shared copies (cp.async, 8 bytes per thread) and their groups
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
// the same with zero fill when !valid (no bytes read; src must still be a valid address)
__device__ __forceinline__ void cp_async8z(void* smem, const void* gmem, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(valid ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// PERM: the x3 periodicity of the fused x3 sweep, 0 / 1 known at compile time (the plain
// launch: the wrap values stay out of the registers of non-periodic lines), 2 read from G.
// KEEPRE (fused x2 only): the epilogue stops after rhov12v1 and clean_param(1), (2) and
// stores the swept energy densities instead of converting them (rhoe2T and clean_param(3)
// come after the compression sub-step).
template <int DIM, bool UNIT, bool FUSED, int PERM = 2, bool KEEPRE = false>
__device__ __forceinline__ void b_sweep_march(const SweepArgs& P, const VB vb) {
  const GridDev& G = P.G;
  const Dims d = G.d;
  const Blocks& B = P.B;
  const double dt = *P.dtp;
  const int s = threadIdx.y;
  const Line1D& L = G.L[DIM - 1];
  const FaceTab& FT = G.F[DIM - 1];
  // line coordinates: DIM3 (i1, i2), DIM2 (i1, i3)
  const int a = vb.bx * 32 + threadIdx.x + 1;
  const int b = vb.by + 1;
  const bool valid = a <= d.lx1;
  const int aa = valid ? a : d.lx1;  // idle lanes read a valid line
  const int lx = (DIM == 3) ? d.lx3 : d.lx2;
  const long long stride = (DIM == 3) ? d.s3 : d.s2;
  const long long base = (DIM == 3) ? gi(d, aa, b, 0) - d.s3 : gi(d, aa, 0, b) - d.s2;
  auto cell = [&](int j) -> long long { return base + (long long)(j + 1) * stride; };
  auto cmet = [&](int j) -> long long { return (DIM == 3) ? cmi(G, aa, b, j) : cmi(G, aa, j, b); };
  auto fmet = [&](int j) -> long long { return (DIM == 3) ? fmi(FT, aa, b, j) : fmi(FT, aa, j, b); };
  auto fvel = [&](int j) -> long long {  // face j in the work arrays (full 3-D layout)
    return (DIM == 3) ? f3i(d, aa, b, j) : f2i(d, aa, j, b);
  };

  int nf;
  double* fld[3];
  int frank[3];
  if (FUSED) {
    if (s < LSP - 1) {
      nf = 3;
      fld[0] = B.ns(s); fld[1] = B.rv(s); fld[2] = B.re(s);
      frank[0] = 0; frank[1] = 1; frank[2] = 0;
    } else {
      nf = 1;
      fld[0] = B.re(s); fld[1] = fld[0]; fld[2] = fld[0];
      frank[0] = 0; frank[1] = 0; frank[2] = 0;
    }
  } else {
    nf = 1;
    fld[0] = (P.which == 0) ? B.ns(s) : (P.which == 1) ? B.rv(s) : B.re(s);
    fld[1] = fld[0]; fld[2] = fld[0];
    frank[0] = (P.which == 1) ? 1 : 0; frank[1] = frank[0]; frank[2] = frank[0];
  }
  const bool per = (PERM == 2) ? (G.flagper != 0) : (PERM == 1);
  auto map3 = [&](int j) -> int {  // x3 ghosts after set_global_boundaries / the self-wrap
    if (j >= 1 && j <= lx) return j;
    if (per) return (j < 1) ? j + lx : j - lx;
    return (j < 1) ? 1 : lx;
  };
  // raw loads of line index j (FUSED x3 converts ns, vs1, Ts into the three fields)
  struct Raw {
    double x[3];
  };
  auto load_raw = [&](int j) -> Raw {
    Raw r;
    if (FUSED && DIM == 3) {
      const long long k = cell(map3(j));
      r.x[0] = B.ns(s)[k];
      r.x[1] = (s < LSP - 1) ? B.vs1(s)[k] : 0.0;
      r.x[2] = B.Ts(s)[k];
    } else {
#pragma unroll
      for (int f = 0; f < 3; ++f) r.x[f] = (f < nf) ? fld[f][cell(j)] : 0.0;
    }
    return r;
  };
  auto fields_of = [&](const Raw& r, double* out) {
    if (FUSED && DIM == 3) {
      if (s < LSP - 1) {
        out[0] = r.x[0];
        out[1] = conv_rv(r.x[0], r.x[1], s);
        out[2] = conv_re(r.x[0], r.x[2], s);
      } else {
        out[0] = conv_re(r.x[0], r.x[2], s);
        out[1] = out[0];
        out[2] = out[0];
      }
    } else {
      out[0] = r.x[0]; out[1] = r.x[1]; out[2] = r.x[2];
    }
  };

  if (lx <= 1) {
    // advec1D_MC_curv passes a single-cell line through; the fused x3 sweep still
    // materialises the converted momentum/energy densities
    if (FUSED && DIM == 3 && valid) {
      const long long k = cell(1);
      B.rv(s)[k] = conv_rv(B.ns(s)[k], B.vs1(s)[k], s);
      B.re(s)[k] = conv_re(B.ns(s)[k], B.Ts(s)[k], s);
    }
    return;
  }

  // periodic fused x3: keep the pre-sweep values the tail of the line wraps to
  double wrap1[3], wrap2[3];
  if (FUSED && DIM == 3 && per) {
    fields_of(load_raw(1), wrap1);
    fields_of(load_raw(2), wrap2);
  }
  FieldRun run[3];
  {
    double fm1[3], f0[3];
    fields_of(load_raw(-1), fm1);
    fields_of(load_raw(0), f0);
    const double dx0 = __ldg(L.dx);
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      run[f].fp = fm1[f];
      run[f].fc = f0[f];
      run[f].ls = mdiv(f0[f] - fm1[f], dx0, __ldg(L.ydx));
      run[f].slp = 0.0;
      run[f].php = 0.0;
    }
  }
  double ha2prev0 = 0.0, ha2prev1 = 0.0;
  // prefetch pipeline: each warp stages, three steps ahead, the raw values of f(jj) and the
  // velocity of step jj-1 (fused: the cell velocity v(jj-1); unfused: the face velocity
  // of face jj-1) by cp.async into slot jj&3 of a 4-slot shared ring of its own; step j
  // reads slot (j+1)&3.  The sweep writes cell j-1 in place at step j, behind every staged
  // index (up to j+4).  vprev = v(j-1).
  double vprev = 0.0;
  __shared__ double xm_f[LSP][4][4][32];
  auto stage = [&](int jj) {
    if (jj >= 1 && jj <= lx + 2) {
      double* sl = &xm_f[s][jj & 3][0][threadIdx.x];
      if constexpr (FUSED && DIM == 3) {
        const long long k = cell(map3(jj));
        cp_async8(sl, B.ns(s) + k);
        if (s < LSP - 1) cp_async8(sl + 32, B.vs1(s) + k);
        cp_async8(sl + 64, B.Ts(s) + k);
        cp_async8(sl + 96, B.vs3(s) + cell(map3(jj - 1)));
      } else {
#pragma unroll
        for (int f = 0; f < 3; ++f)
          if (f < nf) cp_async8(sl + 32 * f, fld[f] + cell(jj));
        if constexpr (FUSED) {
          const int jv = (jj - 1 < 1) ? 1 : (jj - 1 > lx ? lx : jj - 1);
          cp_async8(sl + 96, B.vs2(s) + cell(jv));
        } else if (jj >= 2) {
          cp_async8(sl + 96, P.vsi + (long long)s * ((DIM == 3) ? nf3(d) : nf2(d)) + fvel(jj - 1));
        }
      }
    }
  };
  // Fused x2 on non-unit grids: the metrics change from cell to cell along x2 and the 7
  // species warps of the block read the same ones, so the block fetches them once, three
  // steps ahead, into a 4-slot shared ring (cp.async; warp s copies table s, warp 0 also
  // table 7): step j reads slot j&3 -- face j's hc, yhc, ha2i0, ha2i1 and cell j-1's ha1,
  // yha1 for frank 0 and 1.  Every step ends in a block barrier (the epilogue's, or its
  // own for j < 2), and a thread waits for its copies two steps old before it, so step j+3's
  // slot is complete and visible when step j+3 starts, and the slot written during step j
  // was last read during step j-1, before that step's barrier.
  constexpr bool SMETA = FUSED && DIM == 2 && !UNIT;
  __shared__ double sh_m[SMETA ? 4 : 1][SMETA ? 8 : 1][32];
  auto meta_issue = [&](int jj) {
    if constexpr (SMETA) {
      if (jj >= 1 && jj <= lx + 1) {
        double* slot = &sh_m[jj & 3][0][0];
        auto one = [&](int t) {
          const double* src;
          if (t < 4) {
            const long long fk = fmet(jj);
            src = (t == 0 ? FT.hc : t == 1 ? FT.yhc : t == 2 ? FT.ha2i0 : FT.ha2i1) + fk;
          } else {
            if (jj < 2) return;
            const long long ck = cmet(jj - 1);
            src = (t == 4 ? G.ha1_0 : t == 5 ? G.yha1_0 : t == 6 ? G.ha1_1 : G.yha1_1) + ck;
          }
          cp_async8(slot + t * 32 + threadIdx.x, src);
        };
        one(s);
        if (s == 0) one(7);
      }
    }
  };
  // one cp.async group per step: the group committed at step j holds the metrics of step
  // j+3 and the staged values of slot (j+4)&3 (read at step j+3); the prologue commits the
  // groups that steps 0..2 read
  meta_issue(1);
  stage(1);
  cp_async_commit();
  meta_issue(2);
  stage(2);
  cp_async_commit();
  stage(3);
  cp_async_commit();
  if constexpr (SMETA) {
    cp_async_wait<0>();
    __syncthreads();
  }

  for (int j = 0; j <= lx + 1; ++j) {
    // values of this step
    double fn[3];
    double vc = 0.0;  // fused: v(j); unfused: the velocity of face j
    {
      __syncwarp();  // every lane is done with the slot staged below (read at step j-1)
      meta_issue(j + 3);
      stage(j + 4);
      cp_async_commit();
      cp_async_wait<3>();  // this thread's copies of step j-3's group (slot (j+1)&3)
      __syncwarp();
      const double* sl = &xm_f[s][(j + 1) & 3][0][threadIdx.x];
      if (FUSED && DIM == 3 && j + 1 > lx) {
#pragma unroll
        for (int f = 0; f < 3; ++f) fn[f] = per ? ((j + 1 == lx + 1) ? wrap1[f] : wrap2[f]) : run[f].fc;
      } else {
        Raw nx;
        nx.x[0] = sl[0];
        nx.x[1] = (FUSED && DIM == 3) ? ((s < LSP - 1) ? sl[32] : 0.0) : ((nf > 1) ? sl[32] : 0.0);
        nx.x[2] = ((FUSED && DIM == 3) || nf > 2) ? sl[64] : 0.0;
        fields_of(nx, fn);
      }
      vc = sl[96];
    }

    Face F = {0.0, 0.0, 0.0, 0.0};
    double ha2j0 = 0.0, ha2j1 = 0.0;
    if (j >= 1) {
      double v;
      if (!FUSED) {
        v = vc;
      } else {
        v = 0.5 * (vprev + vc);
        vprev = vc;
      }
      const double dxc = __ldg(L.dx + j);
      if (UNIT) {
        F = make_face(v, 1.0, 1.0, dxc, dt);
        ha2j0 = ha2j1 = 1.0;
      } else if constexpr (SMETA) {
        const double* m = &sh_m[j & 3][0][threadIdx.x];
        F = make_face(v, m[0], m[32], dxc, dt);
        ha2j0 = m[64];
        ha2j1 = m[96];
      } else {
        const long long fk = fmet(j);
        F = make_face(v, __ldg(FT.hc + fk), __ldg(FT.yhc + fk), dxc, dt);
        ha2j0 = __ldg(FT.ha2i0 + fk);
        ha2j1 = __ldg(FT.ha2i1 + fk);
      }
    } else if (FUSED) {
      vprev = vc;
    }
    double ha1_0 = 1.0, yha1_0 = 1.0, ha1_1 = 1.0, yha1_1 = 1.0, dxi = 0.0, ydxi = 0.0;
    if (j >= 2) {
      dxi = __ldg(L.dxi + j - 2);
      ydxi = __ldg(L.ydxi + j - 2);
      if constexpr (SMETA) {
        const double* m = &sh_m[j & 3][4][threadIdx.x];
        ha1_0 = m[0];
        yha1_0 = m[32];
        if (frank[0] == 1 || frank[1] == 1) {
          ha1_1 = m[64];
          yha1_1 = m[96];
        }
      } else {
        const long long ck = cmet(j - 1);
        cell_metric<UNIT>(G, ck, 0, ha1_0, yha1_0);
        if (frank[0] == 1 || frank[1] == 1) cell_metric<UNIT>(G, ck, 1, ha1_1, yha1_1);
      }
    }
    double outv[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      if (f < nf) {
        FieldRun& r = run[f];
        double rs;
        const double sl = mc_slope(r.fp, r.fc, fn[f], r.ls, L, j, rs);
        r.ls = rs;
        if (j >= 1) {
          const double ph = mc_phi(r.fp, r.fc, r.slp, sl, F);
          const bool fr = frank[f] == 1;
          if (j >= 2)
            outv[f] = mc_update(r.fp, (fr ? ha2j1 : ha2j0) * ph, (fr ? ha2prev1 : ha2prev0) * r.php, dt, dxi, ydxi,
                                fr ? ha1_1 : ha1_0, fr ? yha1_1 : yha1_0);
          r.php = ph;
        }
        r.slp = sl;
        r.fp = r.fc;
        r.fc = fn[f];
      }
    }
    ha2prev0 = ha2j0;
    ha2prev1 = ha2j1;
    if constexpr (SMETA) {
      if (j < 2) {
        cp_async_wait<2>();
        __syncthreads();
      }
    }
    if (j < 2) continue;
    const int c = j - 1;  // finished cell
    const long long kc = cell(c);
    if constexpr (!(FUSED && DIM == 2)) {
      if (valid) {
#pragma unroll
        for (int f = 0; f < 3; ++f)
          if (f < nf) fld[f][kc] = outv[f];
        if (FUSED && DIM == 3 && s == LSP - 1)  // unswept electron momentum density
          B.rv(s)[kc] = conv_rv(B.ns(s)[kc], B.vs1(s)[kc], s);
      }
    } else {
      // ---- fused x2 epilogue: rhov12v1 (multifluid.f90:218-233), clean_param(1),
      // clean_param(2) null fill, rhoe2T (179-189), clean_param(3) for cell (a, c, b)
      __shared__ double sh_n[2][LSP - 1][32];
      __shared__ double sh_t[2][LSP - 1][32];
      const int buf = j & 1;
      const int lane = threadIdx.x;
      const bool nul = valid && is_null(G, aa, c, b);
      if (s < LSP - 1) {
        const double n = outv[0], r = outv[1], e = outv[2];
        const double v = r / (c_ms[s] * fmax_f(n, MINDENSDIV));
        sh_n[buf][s][lane] = n;
        sh_t[buf][s][lane] = n * c_qs[s] * v;
        double nc = fmax_f(n, MINDENS);
        if (nul) nc = (s == 0) ? MINDENSNULL * 1e-2 : MINDENSNULL;
        if constexpr (KEEPRE) {
          if (valid) {
            B.ns(s)[kc] = nc;
            B.rv(s)[kc] = r;
            B.vs1(s)[kc] = nul ? 0.0 : v;
            B.re(s)[kc] = e;
          }
        } else {
          double T = fmax_f(c_gm1kb[s] * e / fmax_f(nc, MINDENSDIV), 100.0);
          if (nul) T = 100;
          if (valid) {
            B.ns(s)[kc] = nc;
            B.rv(s)[kc] = r;
            B.vs1(s)[kc] = nul ? 0.0 : v;
            B.Ts(s)[kc] = T;
          }
        }
      }
      if constexpr (SMETA) cp_async_wait<2>();
      __syncthreads();
      if (s == LSP - 1) {
        double npre = 0.0, chrg = 0.0, npost = 0.0;
#pragma unroll
        for (int q = 0; q < LSP - 1; ++q) {
          const double nq = sh_n[buf][q][lane];
          npre = npre + nq;
          chrg = chrg + sh_t[buf][q][lane];
          npost = npost + fmax_f(nq, MINDENS);
        }
        const double ve = mdiv(-1 / fmax_f(npre, MINDENSDIV), QE, YQE) * chrg;
        const double ne = nul ? MINDENSNULL : npost;
        if constexpr (KEEPRE) {
          if (valid) {
            B.ns(s)[kc] = ne;
            B.vs1(s)[kc] = nul ? 0.0 : ve;
            B.re(s)[kc] = outv[0];
          }
        } else {
          double T = fmax_f(c_gm1kb[s] * outv[0] / fmax_f(ne, MINDENSDIV), 100.0);
          if (nul) T = 100;
          if (valid) {
            B.ns(s)[kc] = ne;
            B.vs1(s)[kc] = nul ? 0.0 : ve;
            B.Ts(s)[kc] = T;
          }
        }
      }
    }
  }
  // nothing in flight when the next work item (batched path) restages
  cp_async_wait<0>();
  __syncwarp();
}

#ifndef GEM_MARCH_MINB
#define GEM_MARCH_MINB 2
#endif
#ifndef GEM_X1_MINB
#define GEM_X1_MINB 3
#endif
template <int DIM, bool UNIT, bool FUSED, int PERM = 2, bool KEEPRE = false>
__global__ void __launch_bounds__(224, GEM_MARCH_MINB) k_sweep_march(SweepArgs P) {
  b_sweep_march<DIM, UNIT, FUSED, PERM, KEEPRE>(P, VB{(int)blockIdx.x, (int)blockIdx.y, (int)gridDim.x});
}


// ---- x1 sweep: lanes along the column ------------------------------------------------------
// Lane l of chunk c handles position p = 32c + l - 1... the chunk covers p = 32c .. 32c+31 over
// p = 0 .. lx1+1: the slope at cell p, the flux P(p) = ha2i(p)*phi(p) at face p, and the update
// of cell p-1 (which needs P(p) and P(p-1)).  Values crossing the chunk edge (slope(p-1),
// P(p-1)) are carried from lane 31 of the previous chunk.
template <bool UNIT, bool FUSED>
__device__ __forceinline__ void b_sweep_x1(const SweepArgs& P, const VB vb) {
  const GridDev& G = P.G;
  const Dims d = G.d;
  const Blocks& B = P.B;
  const double dt = *P.dtp;
  const int s = threadIdx.y;
  const int lane = threadIdx.x;
  const int i2 = vb.bx + 1, i3 = vb.by + 1;
  const int n = d.lx1;
  const Line1D& L = G.L[0];
  const FaceTab& FT = G.F[0];
  const long long col = gi(d, 0, i2, i3);  // cell i at col + i
  int nf;
  double* fld[3];
  if (FUSED) {
    if (s < LSP - 1) {
      nf = 3;
      fld[0] = B.ns(s); fld[1] = B.rv(s); fld[2] = B.re(s);
    } else {
      nf = 1;
      fld[0] = B.re(s); fld[1] = fld[0]; fld[2] = fld[0];
    }
  } else {
    nf = 1;
    fld[0] = (P.which == 0) ? B.ns(s) : (P.which == 1) ? B.rv(s) : B.re(s);
    fld[1] = fld[0]; fld[2] = fld[0];
  }
  const double* V1 = B.vs1(s) + col;
  // fused: velocities of the two boundary faces (advec.f90:170-196)
  double vface1 = 0.0, vfaceN = 0.0;
  if (FUSED) {
    const double v1 = V1[1], v2 = V1[2], vn1 = V1[n - 1], vn = V1[n];
    vface1 = (G.gridflag == 1) ? fmin_f(0.5 * (v1 + v2), 0.0) : v1;
    vfaceN = (G.gridflag == 0 || G.gridflag == 1) ? vn : fmax_f(0.5 * (vn1 + vn), 0.0);
    if (lane == 0) {
      P.vs1i[(long long)s * nf1(d) + f1i(d, 1, i2, i3)] = vface1;
      P.vs1i[(long long)s * nf1(d) + f1i(d, n + 1, i2, i3)] = vfaceN;
    }
  }
  double carry_sl[3] = {0.0, 0.0, 0.0}, carry_P[3] = {0.0, 0.0, 0.0};
  const int nchunk = (n + 2 + 31) / 32;
  // Each warp stages its next chunk while it computes this one, by cp.async into a two-slot
  // ring of its own in shared memory -- the fields' values at x1 indices 32c-1 .. 32c+32
  // (clamped to the ghost n+2), the velocities (fused: the cells' there, indices outside
  // 1..n reading cell 1 as the unstaged loads do; unfused: face p of each lane) and, on
  // non-unit grids, the chunk's face (hc, yhc, ha2i0) and cell (ha1, yha1) metrics.  Only
  // the warp reads its slots: it waits for its own copies and __syncwarp orders them; the
  // __syncwarp ending a chunk frees the slot that the next chunk's staging overwrites.
  constexpr int XW = 34;
  __shared__ double xs_f[LSP][2][4][XW];
  __shared__ double xs_m[UNIT ? 1 : LSP][2][5][32];
  auto x1_issue = [&](int cc) {
    {
      if (cc < nchunk) {
        const int slot = cc & 1;
        for (int t = lane; t < XW; t += 32) {
          const int e = 32 * cc - 1 + t;
          const int ef = (e <= n + 2) ? e : n + 2;
#pragma unroll
          for (int f = 0; f < 3; ++f)
            if (f < nf) cp_async8(&xs_f[s][slot][f][t], fld[f] + col + ef);
          if constexpr (FUSED) cp_async8(&xs_f[s][slot][3][t], V1 + ((e >= 1 && e <= n) ? e : 1));
        }
        if constexpr (!FUSED) {
          const int pp = 32 * cc + lane;
          const int ppc = (pp <= n + 1) ? pp : n + 1;
          cp_async8(&xs_f[s][slot][3][lane], P.vsi + (long long)s * nf1(d) + f1i(d, (ppc >= 1) ? ppc : 1, i2, i3));
        }
        if constexpr (!UNIT) {
          const int pp = 32 * cc + lane;
          const int ppc = (pp <= n + 1) ? pp : n + 1;
          const long long fk = fmi(FT, (ppc >= 1) ? ppc : 1, i2, i3);
          cp_async8(&xs_m[s][slot][0][lane], FT.hc + fk);
          cp_async8(&xs_m[s][slot][1][lane], FT.yhc + fk);
          cp_async8(&xs_m[s][slot][2][lane], FT.ha2i0 + fk);
          const int qq = (ppc - 1 >= 1 && ppc - 1 <= n) ? ppc - 1 : 1;
          const long long ck = cmi(G, qq, i2, i3);
          cp_async8(&xs_m[s][slot][3][lane], G.ha1_0 + ck);
          cp_async8(&xs_m[s][slot][4][lane], G.yha1_0 + ck);
        }
      }
      cp_async_commit();
    }
  };
  x1_issue(0);
  for (int c = 0; c < nchunk; ++c) {
    const int p = 32 * c + lane;  // 0 .. n+1 when active
    const bool act = p <= n + 1;
    const int pc = act ? p : n + 1;  // clamped for loads
    x1_issue(c + 1);
    cp_async_wait<1>();
    __syncwarp();
    const double* sf = &xs_f[s][c & 1][0][0];
    const double* sm = &xs_m[UNIT ? 0 : s][c & 1][0][0];
    // face p velocity (p >= 1)
    double v = 0.0;
    if (FUSED) {
      const double vcur = sf[3 * XW + lane + 1];
      const double vleft = sf[3 * XW + lane];
      if (pc == 1) v = vface1;
      else if (pc == n + 1) v = vfaceN;
      else v = 0.5 * (vleft + vcur);
    } else {
      v = sf[3 * XW + lane];
    }
    Face F = {0.0, 0.0, 0.0, 0.0};
    double ha2 = 1.0;
    const double dxc = __ldg(L.dx + pc), ydxc = __ldg(L.ydx + pc);
    const double dxn = __ldg(L.dx + pc + 1), ydxn = __ldg(L.ydx + pc + 1);
    const double dxs = __ldg(L.dxs + pc), ydxs = __ldg(L.ydxs + pc);
    {
      if (UNIT) {
        F = make_face(v, 1.0, 1.0, dxc, dt);
      } else {
        F = make_face(v, sm[lane], sm[32 + lane], dxc, dt);
        ha2 = sm[64 + lane];
      }
    }
    // cell p-1 metrics for the update
    const int q = pc - 1;  // updated cell
    double ha1 = 1.0, yha1 = 1.0, dxi = 1.0, ydxi = 1.0;
    if (q >= 1 && q <= n) {
      dxi = __ldg(L.dxi + q - 1);
      ydxi = __ldg(L.ydxi + q - 1);
      if constexpr (!UNIT) {
        ha1 = sm[96 + lane];
        yha1 = sm[128 + lane];
      }
    }
    double outv[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      if (f < nf) {
        const double fm = sf[f * XW + lane];
        const double f0 = sf[f * XW + lane + 1];
        const double fpl = sf[f * XW + lane + 2];
        // slope(p) (advec.f90:407-414) with lslope = rslope(p-1) from the lane below
        const double rs = mdiv(fpl - f0, dxn, ydxn);
        double ls = __shfl_up_sync(0xffffffffu, rs, 1);
        if (lane == 0) ls = mdiv(f0 - fm, dxc, ydxc);
        const double cs = mdiv(fpl - fm, dxs, ydxs);
        const double sl = minmod(cs, minmod(2 * ls, 2 * rs));
        double slm = __shfl_up_sync(0xffffffffu, sl, 1);
        if (lane == 0) slm = carry_sl[f];
        const double ph = mc_phi(fm, f0, slm, sl, F);
        const double Pp = ha2 * ph;
        double Pm = __shfl_up_sync(0xffffffffu, Pp, 1);
        if (lane == 0) Pm = carry_P[f];
        outv[f] = mc_update(fm, Pp, Pm, dt, dxi, ydxi, ha1, yha1);
        carry_sl[f] = __shfl_sync(0xffffffffu, sl, 31);
        carry_P[f] = __shfl_sync(0xffffffffu, Pp, 31);
      }
    }
    if (act && q >= 1 && q <= n) {
      const long long kq = col + q;
#pragma unroll
      for (int f = 0; f < 3; ++f)
        if (f < nf) fld[f][kq] = outv[f];
      if (FUSED && G.flagper) {
        // halo_allparams self-wrap of the updated column (mpihalo.f90:147-151)
        if (i3 >= d.lx3 - 1) {
          const long long kw = gi(d, q, i2, i3 - d.lx3);
#pragma unroll
          for (int f = 0; f < 3; ++f)
            if (f < nf) fld[f][kw] = outv[f];
        }
        if (i3 <= 2) {
          const long long kw = gi(d, q, i2, i3 + d.lx3);
#pragma unroll
          for (int f = 0; f < 3; ++f)
            if (f < nf) fld[f][kw] = outv[f];
        }
      }
    }
    __syncwarp();
  }
  cp_async_wait<0>();  // nothing in flight when the next work item (batched path) restages
}

template <bool UNIT, bool FUSED>
__global__ void __launch_bounds__(224, GEM_X1_MINB) k_sweep_x1(SweepArgs P) {
  b_sweep_x1<UNIT, FUSED>(P, VB{(int)blockIdx.x, (int)blockIdx.y, (int)gridDim.x});
}


// Fused step: the same epilogue for every ghost cell (rhov12v1 on the ghost values, then
// clean_param(1) sets density ghosts to mindensdiv and clean_param(3) temperature ghosts to
// 100; T2rhoe of those constants gives the final energy-density ghosts).
// KEEPRE: the ghost shell's part of rhov12v1 and clean_param(1), (2) only (the fused x2
// sweep's KEEPRE epilogue); Ts and rhoes stay for the compression sub-step.
template <bool KEEPRE = false>
__device__ __forceinline__ void b_ghost_epilogue(const GridDev& G, const Blocks& B, const VB vb) {
  const Dims d = G.d;
  const long long ngh = nghost(d);
  for (long long q = vb.bx * (long long)blockDim.x + threadIdx.x; q < ngh; q += (long long)vb.gx * blockDim.x) {
    int i1, i2, i3;
    ghost_cell(d, q, i1, i2, i3);
    const long long k = gi(d, i1, i2, i3);
    double chrg = 0.0, nsum = 0.0;
    for (int s = 0; s < LSP - 1; ++s) {
      const double n = B.ns(s)[k];
      const double v = B.rv(s)[k] / (c_ms[s] * fmax_f(n, MINDENSDIV));
      B.vs1(s)[k] = v;
      chrg = chrg + n * c_qs[s] * v;
      nsum = nsum + n;
    }
    B.vs1(LSP - 1)[k] = mdiv(-1 / fmax_f(nsum, MINDENSDIV), QE, YQE) * chrg;
    for (int s = 0; s < LSP; ++s) {
      B.ns(s)[k] = MINDENSDIV;
      if (!KEEPRE) {
        B.Ts(s)[k] = 100.0;
        B.re(s)[k] = conv_re(MINDENSDIV, 100.0, s);
      }
    }
  }
}

template <bool KEEPRE = false>
__global__ void k_ghost_epilogue(GridDev G, Blocks B) {
  b_ghost_epilogue<KEEPRE>(G, B, VB{(int)blockIdx.x, (int)blockIdx.y, (int)gridDim.x});
}

// clean_param(3) and T2rhoe on the ghost shell after a fused diffusion store (which covers
// the interior cells): every ghost temperature 100, rhoes from the cell's density.
__global__ void k_ghost_T100(GridDev G, Blocks B) {
  const Dims d = G.d;
  const long long ngh = nghost(d);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ngh; q += (long long)gridDim.x * blockDim.x) {
    int i1, i2, i3;
    ghost_cell(d, q, i1, i2, i3);
    const long long k = gi(d, i1, i2, i3);
    for (int s = 0; s < LSP; ++s) {
      B.Ts(s)[k] = 100.0;
      B.re(s)[k] = conv_re(B.ns(s)[k], 100.0, s);
    }
  }
}


// ======================================================================================
// 7. Field-aligned heat diffusion (multifluid.f90:309-342; collisions.f90:162-199;
//    diffusion.f90:24-152; PDEparabolic.f90:19-346).  The forward solve is k_diffusion_lu
//    (7a, gem_diffusion_lu.cuh): the reference's band systems factored in LAPACK dgbsv's
//    order.  This section also holds the warp-parallel tridiagonal solver (lane blocks,
//    interface reduction, cyclic reduction) that the adjoint (7b) uses to solve the
//    transposed stage systems; the adjoint needs no LAPACK-order rounding.
// ======================================================================================
struct DiffArgs {
  GridDev G;
  Blocks B;
  const double* J1;  // electrovars(:,:,:,4), ghosted
  const double* nn;  // (lx1,lx2,lx3,3)
  const double* Tn;  // (lx1,lx2,lx3)
  const double* dtp;
  double Teinf;
  const double* Ttop;  // optional per-column (i2 fastest) exospheric temperature, else Teinf
  int solver;  // 1 backward Euler, 2 TRBDF2
  int fused;   // 1: clean_param(3) + T2rhoe folded into the store
  double* lu;          // band-solve scratch of k_diffusion_lu (one slot per resident warp)
  long long lu_slot;   // doubles per slot (>= lx1 * LU_ROW * 32)
  int x3fast;          // column order of k_diffusion_lu: x3 fastest (x3-invariant metrics)
};

// 1/b to about one ulp for the solver's pivots and elimination multipliers (not for the
// discretisation coefficients, which stay IEEE): two Newton-Raphson steps y <- y + y(1-by)
// from the PTX hardware approximation rcp.approx.ftz.f64.  Zero, infinite and
// out-of-range pivots take the IEEE reciprocal.
__device__ __forceinline__ double rcp_nr(double b) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
  double e = __fma_rn(-b, y, 1.0);
  y = __fma_rn(y, e, y);
  e = __fma_rn(-b, y, 1.0);
  y = __fma_rn(y, e, y);
  const unsigned hb = (unsigned)__double2hiint(b) & 0x7fffffffu;
  if (hb - (123u << 20) < (1800u << 20)) return y;  // 2^-900 < |b| < 2^900
  return 1.0 / b;
}

// Lane-blocked tridiagonal solver.  Row k of this lane's block (global row 32-lane block
// order: lane l owns rows l*M .. l*M+M-1) couples x_{k-1}, x_k, x_{k+1}.
//
// Factorisation (matrix only, once per stage):
//   1. block elimination: rows 1..M-1 eliminated downward with row 1 as pivot start, which
//      leaves fill-in SS in the column of the block's first unknown x0; then rows M-3..1
//      upward, leaving fill-in TT in the column of the block's last unknown xl.  Row 0
//      then eliminates x1 (multiplier g0).  What remains per lane is two interface rows,
//      lo (row 0: prev xl, x0, xl) and hi (row M-1: x0, xl, next x0).
//   2. odd-even reduction: hi loses x0 (own lo, multiplier e1) and the next lane's x0
//      (next lo, e2), leaving a 32-row tridiagonal system in the xl of the lanes.
//   3. parallel cyclic reduction of that system over 5 shuffle levels (multipliers k1, k2).
// Every multiplier stays in shared memory (IB, SS, TT per row) or registers (IfaceLU), so
// a solve for a new right-hand side replays only the vector updates.
struct IfaceLU {
  double loA, loB, loC, g0;
  double e1, e2;
  double k1[5], k2[5];
  double iloB, ihiB;  // reciprocal pivots of the lo row and of the reduced hi row
};

template <class WM, class RowM>
__device__ __forceinline__ void band_factor(const WM& W, int M, int lane, RowM rowm, IfaceLU& F) {
  double a, b, c;
  rowm(1, a, b, c);
  double s_prev = a, c_prev = c, bp = b, ib_prev = rcp_nr(b);
  W.ss(1) = s_prev;
  W.ib(1) = ib_prev;
  W.tt(1) = c;
  for (int k = 2; k < M; ++k) {
    rowm(k, a, b, c);
    const double f = a * ib_prev;
    const double sk = -f * s_prev;
    const double bk = b - f * c_prev;
    const double ibk = rcp_nr(bk);
    W.ss(k) = sk;
    W.ib(k) = ibk;
    W.tt(k) = c;
    s_prev = sk;
    c_prev = c;
    bp = bk;
    ib_prev = ibk;
  }
  const double hiA = s_prev, hiC = c_prev;
  double hiB = bp;
  for (int k = M - 3; k >= 1; --k) {
    const double g = W.tt(k) * W.ib(k + 1);
    W.ss(k) = W.ss(k) - g * W.ss(k + 1);
    W.tt(k) = -g * W.tt(k + 1);
  }
  rowm(0, a, b, c);
  if (M >= 3) {
    F.g0 = c * W.ib(1);
    F.loA = a;
    F.loB = b - F.g0 * W.ss(1);
    F.loC = -F.g0 * W.tt(1);
  } else {
    F.g0 = 0.0;
    F.loA = a;
    F.loB = b;
    F.loC = c;
  }
  // odd-even reduction onto the hi rows; the row below lane 31 is an identity row
  double nA = __shfl_down_sync(0xffffffffu, F.loA, 1);
  double nB = __shfl_down_sync(0xffffffffu, F.loB, 1);
  double nC = __shfl_down_sync(0xffffffffu, F.loC, 1);
  if (lane == 31) {
    nA = 0.0;
    nB = 1.0;
    nC = 0.0;
  }
  F.iloB = rcp_nr(F.loB);
  F.e1 = hiA * F.iloB;
  double A = -F.e1 * F.loA, B = hiB - F.e1 * F.loC, C = hiC;
  F.e2 = C * rcp_nr(nB);
  B = B - F.e2 * nA;
  C = -F.e2 * nC;
#pragma unroll
  for (int lv = 0; lv < 5; ++lv) {
    const int sh = 1 << lv;
    double pA = __shfl_up_sync(0xffffffffu, A, sh), pB = __shfl_up_sync(0xffffffffu, B, sh),
           pC = __shfl_up_sync(0xffffffffu, C, sh);
    double qA = __shfl_down_sync(0xffffffffu, A, sh), qB = __shfl_down_sync(0xffffffffu, B, sh),
           qC = __shfl_down_sync(0xffffffffu, C, sh);
    if (lane < sh) {
      pA = 0.0;
      pB = 1.0;
      pC = 0.0;
    }
    if (lane + sh > 31) {
      qA = 0.0;
      qB = 1.0;
      qC = 0.0;
    }
    const double k1 = A * rcp_nr(pB), k2 = C * rcp_nr(qB);
    F.k1[lv] = k1;
    F.k2[lv] = k2;
    const double nA2 = -k1 * pA, nC2 = -k2 * qC;
    B = B - k1 * pC - k2 * qA;
    A = nA2;
    C = nC2;
  }
  F.ihiB = rcp_nr(B);
}

// Solve for the right-hand side in array ARR (in place: the solution replaces it).
template <class WM, class RowM>
__device__ __forceinline__ void band_solve(const WM& W, int M, int lane, RowM rowm, const IfaceLU& F,
                                           int ARR) {
  double a, b, c;
  double rp = W.at(ARR, 1);
  for (int k = 2; k < M; ++k) {
    rowm(k, a, b, c);
    rp = W.at(ARR, k) - a * W.ib(k - 1) * rp;
    W.at(ARR, k) = rp;
  }
  const double hiR = rp;
  double rn = (M >= 3) ? W.at(ARR, M - 2) : 0.0;
  for (int k = M - 3; k >= 1; --k) {
    rowm(k, a, b, c);
    rn = W.at(ARR, k) - c * W.ib(k + 1) * rn;
    W.at(ARR, k) = rn;
  }
  const double loR = (M >= 3) ? W.at(ARR, 0) - F.g0 * W.at(ARR, 1) : W.at(ARR, 0);
  double nR = __shfl_down_sync(0xffffffffu, loR, 1);
  if (lane == 31) nR = 0.0;
  double R = hiR - F.e1 * loR;
  R = R - F.e2 * nR;
#pragma unroll
  for (int lv = 0; lv < 5; ++lv) {
    const int sh = 1 << lv;
    double pR = __shfl_up_sync(0xffffffffu, R, sh), qR = __shfl_down_sync(0xffffffffu, R, sh);
    if (lane < sh) pR = 0.0;
    if (lane + sh > 31) qR = 0.0;
    R = R - F.k1[lv] * pR - F.k2[lv] * qR;
  }
  const double xl = R * F.ihiB;
  double xlp = __shfl_up_sync(0xffffffffu, xl, 1);
  if (lane == 0) xlp = 0.0;
  const double x0 = (loR - F.loA * xlp - F.loC * xl) * F.iloB;
  for (int k = 1; k <= M - 2; ++k)
    W.at(ARR, k) =
        (W.at(ARR, k) - W.ss(k) * x0 - W.tt(k) * xl) * W.ib(k);
  W.at(ARR, 0) = x0;
  W.at(ARR, M - 1) = xl;
}

// Solve with the transposed matrix, A^T y = g (g in ARR, replaced by y), reusing A's
// factorisation: band_solve is a fixed sequence of linear operations r -> A^-1 r (lane-block
// eliminations, the interface reduction, the cyclic-reduction levels, back substitution), so
// A^-T g is that sequence transposed and applied in reverse order -- every axpy y_j += m y_i
// becomes y_i += m y_j and every shuffle up becomes a shuffle down.  rowm gives A's rows.
template <class WM, class RowM>
__device__ __forceinline__ void band_solve_T(const WM& W, int M, int lane, RowM rowm, const IfaceLU& F,
                                             int ARR) {
  double a, b, c;
  // back substitution: x(k) = (r(k) - SS x0 - TT xl) IB (k = 1..M-2), x(0) = x0, x(M-1) = xl
  double x0b = W.at(ARR, 0), xlb = W.at(ARR, M - 1);
  for (int k = 1; k <= M - 2; ++k) {
    const double gk = W.at(ARR, k) * W.ib(k);
    x0b -= W.ss(k) * gk;
    xlb -= W.tt(k) * gk;
    W.at(ARR, k) = gk;
  }
  // x0 = (loR - loA xl(lane-1) - loC xl) iloB, xl = R ihiB
  double loRb = x0b * F.iloB;
  double t = __shfl_down_sync(0xffffffffu, -F.loA * F.iloB * x0b, 1);
  if (lane == 31) t = 0.0;
  xlb += -F.loC * F.iloB * x0b + t;
  double Rb = xlb * F.ihiB;
  // cyclic-reduction levels, last first: R = R - k1 R(lane-sh) - k2 R(lane+sh)
#pragma unroll
  for (int lv = 4; lv >= 0; --lv) {
    const int sh = 1 << lv;
    double t1 = __shfl_down_sync(0xffffffffu, F.k1[lv] * Rb, sh);
    double t2 = __shfl_up_sync(0xffffffffu, F.k2[lv] * Rb, sh);
    if (lane + sh > 31) t1 = 0.0;
    if (lane < sh) t2 = 0.0;
    Rb = Rb - t1 - t2;
  }
  // R = hiR - e1 loR - e2 loR(lane+1)
  loRb += -F.e1 * Rb;
  double u = __shfl_up_sync(0xffffffffu, -F.e2 * Rb, 1);
  if (lane == 0) u = 0.0;
  loRb += u;
  // loR = r(0) - g0 r(1); hiR = r(M-1) after the downward elimination
  if (M >= 3) W.at(ARR, 1) += -F.g0 * loRb;
  W.at(ARR, 0) = loRb;
  W.at(ARR, M - 1) = Rb;
  // upward elimination r(k) -= c(k) IB(k+1) r(k+1) (k = M-3 .. 1), transposed and reversed
  for (int k = 1; k <= M - 3; ++k) {
    rowm(k, a, b, c);
    W.at(ARR, k + 1) += -c * W.ib(k + 1) * W.at(ARR, k);
  }
  // downward elimination r(k) -= a(k) IB(k-1) r(k-1) (k = 2 .. M-1), transposed and reversed
  for (int k = M - 1; k >= 2; --k) {
    rowm(k, a, b, c);
    W.at(ARR, k - 1) += -a * W.ib(k - 1) * W.at(ARR, k);
  }
}

// ======================================================================================
// 7a. The diffusion with the reference's band solve (gem_diffusion_lu.cuh): one thread per
//     (x1 column, species), a warp = 32 columns of one species.  Columns are enumerated x3
//     fastest when the metric tables do not vary along x3 (the warp's metric loads are then
//     one broadcast address), else x2 fastest.  Warp tasks run electrons first (their rows
//     cost more).  Each resident warp owns a scratch slot of lx1 rows x LU_ROW doubles x 32
//     lanes.
// ======================================================================================
constexpr int LU_WPB = 4;  // warps per block
#ifndef GEM_LU_MINB
#define GEM_LU_MINB 4  // resident blocks per SM the register budget is sized for
#endif
constexpr int LU_MINB_DEFAULT = GEM_LU_MINB;

// column accessor of one thread (gemd::lu_column): four column offsets; the table base
// addresses stay in the launch parameters (DiffArgs), so they cost no registers
template <bool UNIT>
struct LuAccDev {
  const DiffArgs& P;
  long long tofs;  // Ts(s) + tofs: cell 0 of the column (ghosted block); ns(s) at nofs
  long long nofs;
  long long mofs;  // cell 0 in the metric tables
  long long qofs;  // interior offset of cell 1, minus 1 (neutral densities)
  long long jofs;  // cell 0 in J1 (ghosted)
  double* sc;      // this lane's scratch: row i, slot k at sc[((i-1)*LU_ROW + k)*32]
  __device__ __forceinline__ double T(int i) const { return P.B.F[tofs + i]; }
  __device__ __forceinline__ double n(int i) const { return __ldg(P.B.F + nofs + i); }
  __device__ __forceinline__ void metrics(int i, double& a1, double& a2, double& a3, double& y1, double& ha,
                                          double& yha) const {
    const long long k = mofs + i;
    a1 = __ldg(P.G.h1 + k);
    a2 = __ldg(P.G.h2 + k);
    a3 = __ldg(P.G.h3 + k);
    y1 = __ldg(P.G.yh1 + k);
    ha = __ldg(P.G.ha1_0 + k);
    yha = __ldg(P.G.yha1_0 + k);
  }
  __device__ __forceinline__ void neutrals(int i, double& a, double& b, double& c, double& j) const {
    const long long nc = nci(P.G.d);
    a = __ldg(P.nn + qofs + i);
    b = __ldg(P.nn + nc + qofs + i);
    c = __ldg(P.nn + 2 * nc + qofs + i);
    j = __ldg(P.J1 + jofs + i);
  }
  __device__ __forceinline__ double dx(int i) const { return __ldg(P.G.L[0].dx + i); }
  __device__ __forceinline__ double ydx(int i) const { return __ldg(P.G.L[0].ydx + i); }
  __device__ __forceinline__ double dxi(int i) const { return __ldg(P.G.L[0].dxi + i - 1); }
  __device__ __forceinline__ double ydxi(int i) const { return __ldg(P.G.L[0].ydxi + i - 1); }
  __device__ __forceinline__ double dxs(int i) const { return __ldg(P.G.L[0].dxs + i); }
  __device__ __forceinline__ double ydxs(int i) const { return __ldg(P.G.L[0].ydxs + i); }
  // the scratch streams through L2 only (ld/st.global.cg), keeping L1 for the column inputs
  // and the grid tables the warp re-reads
  __device__ __forceinline__ double sld(int i, int k) const { return __ldcg(sc + ((i - 1) * gemd::LU_ROW + k) * 32); }
  __device__ __forceinline__ void sst(int i, int k, double v) const {
    __stcg(sc + ((i - 1) * gemd::LU_ROW + k) * 32, v);
  }
};

// The solution's destination: max(T,100) (multifluid.f90:340) into Ts; fused with
// clean_param(3) (null cells 100) and T2rhoe (rhoes from ns), whose inputs are loaded ahead.
struct LuPre {
  double nv;
  bool nul;
};
struct LuStoreDev {
  double* Tout;
  double* re;                 // rhoes of the column (fused), else null
  const double* nc;           // ns of the column
  const unsigned char* nul;   // null-point flags of the column (interior offset - 1), or null
  int s;
  __device__ __forceinline__ LuPre pre(int i) const {
    LuPre p;
    p.nv = re ? __ldg(nc + i) : 0.0;
    p.nul = nul ? nul[i] != 0 : false;
    return p;
  }
  __device__ __forceinline__ void operator()(int i, double x, const LuPre& p) const {
    double T = fmax_f(x, 100.0);
    if (p.nul) T = 100;
    Tout[i] = T;
    if (re) re[i] = p.nv * KB * T / (c_gammas[s] - 1);  // T2rhoe (multifluid.f90:193-202)
  }
};

// One warp task: 32 columns of one species.  slot = this warp's scratch slot (lane 0).
template <bool UNIT>
__device__ __forceinline__ void b_diffusion_lu(const DiffArgs& P, int task, double* slot) {
  const GridDev& G = P.G;
  const Dims d = G.d;
  const int n = d.lx1;
  const int lane = threadIdx.x & 31;
  const int ncol = d.lx2 * d.lx3;
  const int tps = (ncol + 31) / 32;
  const int s = LSP - 1 - task / tps;
  const int col = (task % tps) * 32 + lane;
  if (col >= ncol) return;
  int i2, i3;
  if (P.x3fast) {
    i3 = col % d.lx3 + 1;
    i2 = col / d.lx3 + 1;
  } else {
    i2 = col % d.lx2 + 1;
    i3 = col / d.lx2 + 1;
  }
  const long long m0 = gi(d, 0, i2, i3);
  const long long mm0 = cmi(G, 0, i2, i3);
  const long long q0 = ci(d, 1, i2, i3) - 1;

  LuAccDev<UNIT> a{P, (long long)(4 * LSP + s) * d.ng + m0, (long long)s * d.ng + m0, mm0, q0, m0, slot + lane};
  // Dirichlet values (diffusion.f90:54-79): the exospheric side takes Teinf or the column's value
  const double tn1 = __ldg(P.Tn + ci(d, 1, i2, i3)), tnl = __ldg(P.Tn + ci(d, n, i2, i3));
  const double tinf = P.Ttop ? __ldg(P.Ttop + (i2 - 1) + (long long)d.lx2 * (i3 - 1)) : P.Teinf;
  gemd::LuK k;
  k.n = n;
  k.s = s;
  k.dt = *P.dtp;
  if (G.gridflag == 0) {
    k.tmin = tn1;
    k.tmax = tnl;
  } else if (G.gridflag == 1) {
    k.tmin = tinf;
    k.tmax = tnl;
  } else {
    k.tmin = tn1;
    k.tmax = tinf;
  }
  k.c0 = (c_gammas[s] - 1.0) / KB;
  k.tcoef = (s < LSP - 1) ? c_tcoef[s] : 0.0;
  LuStoreDev st;
  st.Tout = P.B.Ts(s) + m0;
  st.re = P.fused ? P.B.re(s) + m0 : nullptr;
  st.nc = P.B.ns(s) + m0;
  st.nul = (P.fused && G.has_null) ? G.nullpts + (ci(d, 1, i2, i3) - 1) : nullptr;
  st.s = s;
  if (s == LSP - 1)
    gemd::lu_column<UNIT, true>(a, k, P.solver, st);
  else
    gemd::lu_column<UNIT, false>(a, k, P.solver, st);
  double* Tout = st.Tout;
  if (!P.fused) {
    Tout[0] = fmax_f(k.tmin, 100.0);
    Tout[n + 1] = fmax_f(k.tmax, 100.0);
  }
}

// plain launch: persistent warps over the warp tasks; scratch slot = the global warp index
template <bool UNIT>
__global__ void __launch_bounds__(32 * LU_WPB, GEM_LU_MINB) k_diffusion_lu(DiffArgs P) {
  const int warp = threadIdx.x >> 5;
  const int gw = blockIdx.x * LU_WPB + warp;
  const int nw = gridDim.x * LU_WPB;
  const int ncol = P.G.d.lx2 * P.G.d.lx3;
  const int ntask = ((ncol + 31) / 32) * LSP;
  double* slot = P.lu + (long long)gw * P.lu_slot;
  for (int t = gw; t < ntask; t += nw) b_diffusion_lu<UNIT>(P, t, slot);
}


// standalone energy_diffusion: max(T,100) on the ghost cells other than the x1 BC layers
__global__ void k_diffusion_ghost_floor(GridDev G, Blocks B) {
  const Dims d = G.d;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < d.ng;
       k += (long long)gridDim.x * blockDim.x) {
    int i1, i2, i3;
    decode_cell(d, k, i1, i2, i3);
    if (!is_ghost(d, i1, i2, i3)) continue;
    const bool bc = (i1 == 0 || i1 == d.lx1 + 1) && i2 >= 1 && i2 <= d.lx2 && i3 >= 1 && i3 <= d.lx3;
    if (bc) continue;
    for (int s = 0; s < LSP; ++s) B.Ts(s)[k] = fmax_f(B.Ts(s)[k], 100.0);
  }
}

// ======================================================================================
// 7b. Adjoint (vector-Jacobian product) of the energy diffusion, for the differentiable
//     path.  One warp per (x1 column, species), lanes owning blocks of M consecutive rows,
//     as in the forward solver: the kernel recomputes the per-row conduction factors
//     q-, q+, bq, both TRBDF2 stage solutions X and Y, then solves the transposed stage
//     systems by the transpose of the lane-blocked band solve (reusing each stage's
//     factorisation) and chains the cotangents of the band entries and
//     right-hand sides back through q+-, Dh, C, B and lambda to T, n and the column's
//     exospheric boundary value.  Every per-row array lives in shared memory; T, n, Ybar,
//     Tbar and nbar move along x1 (coalesced).  Cotangent inputs/outputs are ghosted
//     7-species blocks; only interior rows are written (the caller zero-initialises Tbar
//     and nbar).
// ======================================================================================
struct DiffAdjArgs {
  GridDev G;
  const double* T;     // diffusion input temperature (ghosted, 7 species)
  const double* ns;    // densities (ghosted, 7 species)
  const double* J1;    // electrovars(:,:,:,4)
  const double* nn;    // (lx1,lx2,lx3,3)
  const double* Tn;    // (lx1,lx2,lx3)
  const double* Ttop;  // optional per-column exospheric temperature
  double Teinf;
  const double* dtp;
  int solver;
  int M;               // rows per lane
  const double* Ybar;  // cotangent of the diffusion output (after max(T,100))
  double* Tbar;
  double* nbar;
  double* Ttop_bar;    // optional: (lx2*lx3) per species, species slowest
};

// per-row shared-memory arrays of the adjoint, row-interleaved: the VNA arrays of row k of
// every lane sit together (warp base + (k*VNA + arr)*32 + lane).  Slots are
// reused once their first content is dead: D becomes the stage-1 solution X, Y becomes the
// temperature cotangent TB, R carries Ybar -> lambda2 -> xbar -> lambda1, and after the
// first-stage pass QMB / QPB / BQB hold EM / EP / the C cotangent.
constexpr int VA_T = 0, VA_C = 1, VA_BQ = 2, VA_QM = 3, VA_QP = 4, VA_X = 5, VA_SS = 6, VA_IB = 7, VA_TT = 8,
              VA_Y = 9, VA_R = 10, VA_QMB = 11, VA_QPB = 12, VA_BQB = 13;
constexpr int VNA = 14;
constexpr int VA_D = VA_X, VA_TB = VA_Y;

struct WarpMemA {
  double* wb;
  double* b;
  __device__ __forceinline__ double& at(int arr, int k) const { return b[(k * VNA + arr) * 32]; }
  __device__ __forceinline__ double& at_lane(int arr, int k, int l) const { return wb[(k * VNA + arr) * 32 + l]; }
  __device__ __forceinline__ double& ss(int k) const { return at(VA_SS, k); }
  __device__ __forceinline__ double& ib(int k) const { return at(VA_IB, k); }
  __device__ __forceinline__ double& tt(int k) const { return at(VA_TT, k); }
};

// thermal conductivity lambda(T, n) (collisions.f90:162-199) and its partial derivatives;
// n1, n2, n3: the neutral densities of the cell (electrons)
__device__ __forceinline__ void lam_deriv(int s, double T, double nv, double n1, double n2, double n3, double& lam,
                                          double& dl_dT, double& dl_dn) {
  // the adjoint needs no exact quotients or correctly rounded powers: each reciprocal is
  // formed once and multiplied, and T^2.5 = T^2 sqrt(T) in plain arithmetic
  const double sq = sqrt(T);
  const double T25 = T * T * sq;
  const double yT = 1.0 / T;
  if (s < LSP - 1) {
    lam = c_tcoef[s] * T25;
    dl_dT = 2.5 * lam * yT;
    dl_dn = 0.0;
    return;
  }
  const double hy = 0.5 * yT * sq;  // 1 / (2 sqrt(T))
  const double ynv = 1.0 / nv;
  const double X = n1 * 1.1e-16 * (1 + 5.7e-4 * T) + n2 * 2.82e-17 * sq * (1 - 1.21e-4 * T) +
                   n3 * 2.2e-16 * (1 + 3.6e-2 * sq);
  const double Xp = n1 * 1.1e-16 * 5.7e-4 + n2 * 2.82e-17 * (hy * (1 - 1.21e-4 * T) - 1.21e-4 * sq) +
                    n3 * 2.2e-16 * 3.6e-2 * hy;
  const double den = 1 + 3.22e4 * (T * T) * ynv * X;
  const double yden = 1.0 / den;
  lam = ELCHRG * 100 * 7.7e5 * T25 * yden;
  const double dden_dT = 3.22e4 * (2 * T * X + T * T * Xp) * ynv;
  dl_dT = lam * (2.5 * yT - dden_dT * yden);
  dl_dn = lam * (3.22e4 * T * T * X * ynv * ynv) * yden;
}

template <bool UNIT>
__global__ void __launch_bounds__(128) k_diffusion_vjp(DiffAdjArgs P) {
  extern __shared__ double smem[];
  const GridDev& G = P.G;
  const Dims d = G.d;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  const int M = P.M;
  const WarpMemA W{smem + warp * VNA * M * 32, smem + warp * VNA * M * 32 + lane};
  const int n = d.lx1;
  const double dt = *P.dtp;
  const long long ncol = (long long)d.lx2 * d.lx3;
  const long long ncs = ncol * LSP;
  const long long nc = nci(d);
  const Line1D& L1 = G.L[0];
  const bool trbdf = P.solver == 2;
  const double dA = trbdf ? 1 / (dt / 2) : 1 / dt;  // first-stage diagonal term
  const double d2 = 1 / (dt / 3);                   // BDF2 diagonal term
  // coalesced passes: row idx = 32c + lane lives in the slot (lane idx/M, row idx%M)
  const int lp0 = lane / M, kp0 = lane - lp0 * M, q32 = 32 / M, r32 = 32 - q32 * M;
  for (long long cs = (long long)blockIdx.x * wpb + warp; cs < ncs; cs += (long long)gridDim.x * wpb) {
    const int s = (int)(cs % LSP);
    const int col = (int)(cs / LSP);
    const int i2 = col % d.lx2 + 1, i3 = col / d.lx2 + 1;
    const long long m0 = gi(d, 0, i2, i3);
    const long long mm0 = cmi(G, 0, i2, i3);
    const long long q0 = ci(d, 1, i2, i3) - 1;
    const double* Tc = P.T + (long long)s * d.ng + m0;
    const double* nsc = P.ns + (long long)s * d.ng + m0;
    const double c0 = c_gm1kb[s];
    const bool el = s == LSP - 1;
    // ---- the column's inputs, global -> shared by cp.async with every chunk in flight (zero
    //      fill past n): T into T; ns, J1 and the neutral densities into the q-, q+ and
    //      factorisation rows, the metrics into the cotangent rows (all written later), and
    //      Ybar into R, where the backward starts
    {
      const double* Yb = P.Ybar + (long long)s * d.ng + m0;
      int lp = lp0, kp = kp0;
      for (int c = 0; c < M; ++c) {
        const int i = 1 + 32 * c + lane;
        const bool in = i <= n;
        const int ii = in ? i : 1;
        const long long q = q0 + ii, mk = mm0 + ii;
        cp_async8z(&W.at_lane(VA_T, kp, lp), Tc + ii, in);
        cp_async8z(&W.at_lane(VA_QM, kp, lp), nsc + ii, in);
        cp_async8z(&W.at_lane(VA_R, kp, lp), Yb + ii, in);
        if (el) {
          cp_async8z(&W.at_lane(VA_QP, kp, lp), P.J1 + m0 + ii, in);
          cp_async8z(&W.at_lane(VA_SS, kp, lp), P.nn + q, in);
          cp_async8z(&W.at_lane(VA_IB, kp, lp), P.nn + nc + q, in);
          cp_async8z(&W.at_lane(VA_TT, kp, lp), P.nn + 2 * nc + q, in);
        }
        if (!UNIT) {
          cp_async8z(&W.at_lane(VA_Y, kp, lp), G.yh1 + mk, in);
          cp_async8z(&W.at_lane(VA_QMB, kp, lp), G.h2 + mk, in);
          cp_async8z(&W.at_lane(VA_QPB, kp, lp), G.h3 + mk, in);
          cp_async8z(&W.at_lane(VA_BQB, kp, lp), G.yha1_0 + mk, in);
        }
        kp += r32;
        lp += q32;
        if (kp >= M) {
          kp -= M;
          ++lp;
        }
      }
      cp_async_commit();
      cp_async_wait<0>();
      __syncwarp();
    }
    // ---- pass 1 (along x1): T, D = lambda h2 h3 / h1, C, bq
    {
      int lp = lp0, kp = kp0;
      for (int c = 0; c < M; ++c) {
        const int i = 1 + 32 * c + lane;
        double T = 0, D = 0, C = 0, bq = 0;
        if (i <= n) {
          T = W.at_lane(VA_T, kp, lp);
          const double nv = W.at_lane(VA_QM, kp, lp);
          const double yh1 = UNIT ? 1.0 : W.at_lane(VA_Y, kp, lp);
          const double h23 = UNIT ? 1.0 : W.at_lane(VA_QMB, kp, lp) * W.at_lane(VA_QPB, kp, lp);
          const double yha1 = UNIT ? 1.0 : W.at_lane(VA_BQB, kp, lp);
          double lam, dl_dT, dl_dn;
          if (el)
            lam_deriv(s, T, nv, W.at_lane(VA_SS, kp, lp), W.at_lane(VA_IB, kp, lp), W.at_lane(VA_TT, kp, lp), lam,
                      dl_dT, dl_dn);
          else
            lam_deriv(s, T, nv, 0.0, 0.0, 0.0, lam, dl_dT, dl_dn);
          D = lam * h23 * yh1;
          C = c0 / fmax_f(nv, MINDENSDIV) * yha1;
          if (el && i >= 2 && i <= n - 1) {
            const double beta = 5.0 / 2 * KB / ELCHRG * W.at_lane(VA_QP, kp, lp);  // collisions.f90:197
            bq = C * beta * yh1 * __ldg(L1.ydxs + i);  // 1/(dx1(i) + dx1(i+1))
          }
        }
        W.at_lane(VA_T, kp, lp) = T;
        W.at_lane(VA_D, kp, lp) = D;
        W.at_lane(VA_C, kp, lp) = C;
        W.at_lane(VA_BQ, kp, lp) = bq;
        kp += r32;
        lp += q32;
        if (kp >= M) {
          kp -= M;
          ++lp;
        }
      }
    }
    __syncwarp();
    // value of array arr at the row delta (-1, 0, +1) away from slot k, across lanes; 0 past
    // the ends of the lane blocks
    auto nb = [&](int arr, int k, int delta) -> double {
      int kk = k + delta, ll = lane;
      if (kk < 0) { kk = M - 1; --ll; }
      if (kk >= M) { kk = 0; ++ll; }
      return (ll < 0 || ll > 31) ? 0.0 : W.at_lane(arr, kk, ll);
    };
    // ---- q-, q+ per slot (rows 2..n-1): Dh(i) = (D(i-1) + D(i))/2
    for (int k = 0; k < M; ++k) {
      const int i = 1 + lane * M + k;
      double qm = 0.0, qp = 0.0;
      if (i >= 2 && i <= n - 1) {
        const double Dm = nb(VA_D, k, -1), Dc = W.at(VA_D, k), Dp = nb(VA_D, k, 1);
        const double Cy = W.at(VA_C, k) * __ldg(L1.ydxi + i - 1);
        qm = Cy * (0.5 * (Dm + Dc)) * __ldg(L1.ydx + i);
        qp = Cy * (0.5 * (Dc + Dp)) * __ldg(L1.ydx + i + 1);
      }
      W.at(VA_QM, k) = qm;
      W.at(VA_QP, k) = qp;
    }
    __syncwarp();
    // Dirichlet values (diffusion.f90:54-79)
    double tmin, tmax;
    {
      const double tn1 = __ldg(P.Tn + ci(d, 1, i2, i3)), tnl = __ldg(P.Tn + ci(d, n, i2, i3));
      const double tinf = P.Ttop ? __ldg(P.Ttop + col) : P.Teinf;
      if (G.gridflag == 0) { tmin = tn1; tmax = tnl; }
      else if (G.gridflag == 1) { tmin = tinf; tmax = tnl; }
      else { tmin = tn1; tmax = tinf; }
    }
    // stage matrix rows: stage 0 = the first stage (TR half step, or backward Euler), 1 = BDF2;
    // the row in slot kk of lane ll; rows 1, n, the padding past n and rows outside the
    // warp are identity rows
    auto row_at = [&](int stage, int kk, int ll, double& a, double& b, double& c) {
      const int i = 1 + ll * M + kk;
      if (ll < 0 || ll > 31 || i == 1 || i >= n) { a = 0; b = 1; c = 0; return; }
      const double qm = W.at_lane(VA_QM, kk, ll), qp = W.at_lane(VA_QP, kk, ll), bq = W.at_lane(VA_BQ, kk, ll);
      if (stage == 0 && trbdf) {
        a = -(qm / 2) + bq / 2;
        b = dA + qp / 2 + qm / 2;
        c = -(qp / 2) - bq / 2;
      } else {
        a = -qm + bq;
        b = ((stage == 0) ? dA : d2) + qp + qm;
        c = -qp - bq;
      }
    };
    // one row function for both stages (the band solver is instantiated once)
    int stage = 0;
    auto rowf = [&](int k, double& a, double& b, double& c) { row_at(stage, k, lane, a, b, c); };
    IfaceLU F;
    // ---- forward replay: first stage into X (the slot of D, now dead)
    for (int k = 0; k < M; ++k) {
      const int i = 1 + lane * M + k;
      double r;
      if (i == 1) r = tmin;
      else if (i == n) r = tmax;
      else if (i > n) r = 0.0;
      else if (trbdf) {
        double a, b, c;
        row_at(0, k, lane, a, b, c);
        const double qm = W.at(VA_QM, k), qp = W.at(VA_QP, k);
        const double Tv = W.at(VA_T, k);
        r = Tv * dA - a * nb(VA_T, k, -1) - (qp / 2 + qm / 2) * Tv - c * nb(VA_T, k, 1);
      } else {
        r = W.at(VA_T, k) * dA;
      }
      W.at(VA_X, k) = r;
    }
    stage = 0;
    band_factor(W, M, lane, rowf, F);
    band_solve(W, M, lane, rowf, F, VA_X);
    __syncwarp();
    int YOUT = VA_X;
    if (trbdf) {
      for (int k = 0; k < M; ++k) {
        const int i = 1 + lane * M + k;
        double r;
        if (i == 1) r = tmin;
        else if (i == n) r = tmax;
        else if (i > n) r = 0.0;
        else r = -(1 / 3.0 * W.at(VA_T, k) * d2) + 4 / 3.0 * W.at(VA_X, k) * d2;
        W.at(VA_Y, k) = r;
      }
      stage = 1;
      band_factor(W, M, lane, rowf, F);
      band_solve(W, M, lane, rowf, F, VA_Y);
      YOUT = VA_Y;
    }
    __syncwarp();
    // ---- Ybar (staged into R with the inputs), masked by max(T,100) of the output
    for (int k = 0; k < M; ++k)
      if (!(W.at(YOUT, k) >= 100.0)) W.at(VA_R, k) = 0.0;
    double tminb = 0.0, tmaxb = 0.0;  // on the lanes that own rows 1 and n
    const int lane_n = (n - 1) / M, k_n = (n - 1) - lane_n * M;
    if (trbdf) {
      // lambda2 = A2^-T g (A2's factorisation is still in place); then the BDF2 cotangents
      // of q-, q+, bq and T, and xbar
      band_solve_T(W, M, lane, rowf, F, VA_R);
      __syncwarp();
      if (lane == 0) tminb += W.at(VA_R, 0);
      if (lane == lane_n) tmaxb += W.at(VA_R, k_n);
      // Y(k-1) is read after slot k-1 of Y became TB: keep a sliding window
      double ym = nb(VA_Y, 0, -1), yc = W.at(VA_Y, 0);
      const double ynext = nb(VA_Y, M - 1, 1);
      __syncwarp();
      for (int k = 0; k < M; ++k) {
        const int i = 1 + lane * M + k;
        const double yp = (k < M - 1) ? W.at(VA_Y, k + 1) : ynext;
        double qmb = 0.0, qpb = 0.0, bqb = 0.0, tb = 0.0, xb = 0.0;
        if (i >= 2 && i <= n - 1) {
          const double l2 = W.at(VA_R, k);
          const double ab = -l2 * ym, bb = -l2 * yc, cb = -l2 * yp;
          qmb = -ab + bb;
          qpb = bb - cb;
          bqb = ab - cb;
          tb = l2 * (-(1 / 3.0) * d2);
          xb = l2 * ((4 / 3.0) * d2);
        }
        W.at(VA_QMB, k) = qmb;
        W.at(VA_QPB, k) = qpb;
        W.at(VA_BQB, k) = bqb;
        W.at(VA_TB, k) = tb;  // the slot of Y (read above)
        W.at(VA_R, k) = xb;
        ym = yc;
        yc = yp;
      }
    } else {
      for (int k = 0; k < M; ++k) {
        W.at(VA_QMB, k) = 0.0;
        W.at(VA_QPB, k) = 0.0;
        W.at(VA_BQB, k) = 0.0;
        W.at(VA_TB, k) = 0.0;
      }
    }
    __syncwarp();
    // lambda1 = A1^-T xbar (or A^-T g for backward Euler, whose factorisation is in place)
    stage = 0;
    if (trbdf) band_factor(W, M, lane, rowf, F);
    band_solve_T(W, M, lane, rowf, F, VA_R);
    __syncwarp();
    if (lane == 0) tminb += W.at(VA_R, 0);
    if (lane == lane_n) tmaxb += W.at(VA_R, k_n);
    // first-stage cotangents, then EM / EP (the Dh cotangent parts) and the C cotangent
    for (int k = 0; k < M; ++k) {
      const int i = 1 + lane * M + k;
      if (i > n) continue;
      double tb = W.at(VA_TB, k);
      // T(i) in the right-hand sides of rows i-1 and i+1 (TR only)
      if (trbdf) {
        if (i + 1 >= 2 && i + 1 <= n - 1) {
          double a, b, c;
          int kk = k + 1, ll = lane;
          if (kk >= M) { kk = 0; ++ll; }
          row_at(0, kk, ll, a, b, c);
          tb += -nb(VA_R, k, 1) * a;
        }
        if (i - 1 >= 2 && i - 1 <= n - 1) {
          double a, b, c;
          int kk = k - 1, ll = lane;
          if (kk < 0) { kk = M - 1; --ll; }
          row_at(0, kk, ll, a, b, c);
          tb += -nb(VA_R, k, -1) * c;
        }
      }
      double em = 0.0, ep = 0.0, cb = 0.0;
      if (i >= 2 && i <= n - 1) {
        const double l1 = W.at(VA_R, k);
        const double qm = W.at(VA_QM, k), qp = W.at(VA_QP, k), bq = W.at(VA_BQ, k);
        const double xm = nb(VA_X, k, -1), xc = W.at(VA_X, k), xp = nb(VA_X, k, 1);
        double qmb = W.at(VA_QMB, k), qpb = W.at(VA_QPB, k), bqb = W.at(VA_BQB, k);
        if (trbdf) {
          const double Tm = nb(VA_T, k, -1), Tv = W.at(VA_T, k), Tp = nb(VA_T, k, 1);
          const double ab = -l1 * (xm + Tm), cbv = -l1 * (xp + Tp), bb = -l1 * xc, pb = -l1 * Tv;
          qmb += -ab / 2 + bb / 2 + pb / 2;
          qpb += -cbv / 2 + bb / 2 + pb / 2;
          bqb += ab / 2 - cbv / 2;
          tb += l1 * (dA - (qp / 2 + qm / 2));
        } else {
          const double ab = -l1 * xm, cbv = -l1 * xp, bb = -l1 * xc;
          qmb += -ab + bb;
          qpb += bb - cbv;
          bqb += ab - cbv;
          tb += l1 * dA;
        }
        // q- = C Dh(i) / (dxi dx(i)), q+ = C Dh(i+1) / (dxi dx(i+1)), bq = C beta/h1/(dx(i)+dx(i+1))
        const double C = W.at(VA_C, k);
        const double Cy = C * __ldg(L1.ydxi + i - 1);
        em = qmb * Cy * __ldg(L1.ydx + i);      // -> Dh(i)
        ep = qpb * Cy * __ldg(L1.ydx + i + 1);  // -> Dh(i+1)
        cb = (qmb * qm + qpb * qp + bqb * bq) / C;
      }
      W.at(VA_TB, k) = tb;
      W.at(VA_QMB, k) = em;
      W.at(VA_QPB, k) = ep;
      W.at(VA_BQB, k) = cb;
    }
    __syncwarp();
    // ---- ns, the neutral densities and the metrics again, staged by cp.async into rows
    //      that are dead now (factorisation, R, X, q-, q+)
    {
      int lp = lp0, kp = kp0;
      for (int c = 0; c < M; ++c) {
        const int i = 1 + 32 * c + lane;
        const bool in = i <= n;
        const int ii = in ? i : 1;
        const long long q = q0 + ii, mk = mm0 + ii;
        cp_async8z(&W.at_lane(VA_SS, kp, lp), nsc + ii, in);
        if (el) {
          cp_async8z(&W.at_lane(VA_IB, kp, lp), P.nn + q, in);
          cp_async8z(&W.at_lane(VA_TT, kp, lp), P.nn + nc + q, in);
          cp_async8z(&W.at_lane(VA_R, kp, lp), P.nn + 2 * nc + q, in);
        }
        if (!UNIT) {
          cp_async8z(&W.at_lane(VA_X, kp, lp), G.h2 + mk, in);
          cp_async8z(&W.at_lane(VA_QM, kp, lp), G.h3 + mk, in);
          cp_async8z(&W.at_lane(VA_QP, kp, lp), G.yh1 + mk, in);
        }
        kp += r32;
        lp += q32;
        if (kp >= M) {
          kp -= M;
          ++lp;
        }
      }
      cp_async_commit();
      cp_async_wait<0>();
      __syncwarp();
    }
    // ---- along x1: D(i) feeds Dh(i) (i >= 2) and Dh(i+1) (i < n), Dh(j) collects EM(j) and
    // EP(j-1); then through lambda(T, n) and C(n) to Tbar, nbar
    {
      double* Tbo = P.Tbar + (long long)s * d.ng + m0;
      double* nbo = P.nbar + (long long)s * d.ng + m0;
      int lp = lp0, kp = kp0;
      for (int c = 0; c < M; ++c) {
        const int i = 1 + 32 * c + lane;
        if (i <= n) {
          int km = kp - 1, lm = lp, kq = kp + 1, lq = lp;
          if (km < 0) { km = M - 1; --lm; }
          if (kq >= M) { kq = 0; ++lq; }
          const double dh_i = (i >= 2) ? W.at_lane(VA_QMB, kp, lp) + W.at_lane(VA_QPB, km, lm) : 0.0;
          const double dh_ip1 = (i < n) ? W.at_lane(VA_QMB, kq, lq) + W.at_lane(VA_QPB, kp, lp) : 0.0;
          const double Db = 0.5 * (dh_i + dh_ip1);
          const double T = W.at_lane(VA_T, kp, lp), nv = W.at_lane(VA_SS, kp, lp);
          const double g =
              UNIT ? 1.0 : W.at_lane(VA_X, kp, lp) * W.at_lane(VA_QM, kp, lp) * W.at_lane(VA_QP, kp, lp);
          double lam, dl_dT, dl_dn;
          if (el)
            lam_deriv(s, T, nv, W.at_lane(VA_IB, kp, lp), W.at_lane(VA_TT, kp, lp), W.at_lane(VA_R, kp, lp), lam,
                      dl_dT, dl_dn);
          else
            lam_deriv(s, T, nv, 0.0, 0.0, 0.0, lam, dl_dT, dl_dn);
          const double dcn = (nv > MINDENSDIV) ? -W.at_lane(VA_C, kp, lp) / nv : 0.0;
          Tbo[i] = W.at_lane(VA_TB, kp, lp) + Db * dl_dT * g;
          nbo[i] = W.at_lane(VA_BQB, kp, lp) * dcn + Db * dl_dn * g;
        }
        kp += r32;
        lp += q32;
        if (kp >= M) {
          kp -= M;
          ++lp;
        }
      }
    }
    if (P.Ttop_bar) {
      double tb = (G.gridflag == 1) ? tminb : (G.gridflag == 2) ? tmaxb : 0.0;
      for (int o = 16; o > 0; o >>= 1) tb += __shfl_xor_sync(0xffffffffu, tb, o);
      if (lane == 0) P.Ttop_bar[(long long)s * ncol + col] = tb;
    }
    __syncwarp();
  }
}

// ======================================================================================
// 7c. Adjoint (vector-Jacobian product) of one field sweep (advec.f90:384-435 along x1, x2
//     or x3, species 0..nsp-1), for the differentiable path.  With the limiter and upwind
//     branches of the forward sweep replayed, the line update is linear in f, and its
//     transpose is a local stencil: the cotangent of face i's flux reaches the upwind cell
//     directly and, through the selected slope (zero, centred, or twice the left or right
//     difference), the cells around it -- cells i-2 .. i+1 in all.  Each slope branch and
//     each face's cotangent parts are computed once: x2 / x3 lines by threads marching along
//     the line (lanes along i1), x1 lines by warps with lanes along the contiguous x1 and
//     neighbours exchanged by shuffles.  Every cell is written by one thread, as obar plus
//     its flux parts; vbar (optional) gets the face-velocity cotangent.
// ======================================================================================
struct SweepVjpArgs {
  GridDev G;
  const double* f;  // the sweep's input field (ghosted, nsp species blocks)
  const double* v;  // face velocities (reference face layout, species blocks)
  const double* dtp;
  const double* obar;  // cotangent of the output field
  double* fbar;        // out: the cotangent of f.  The kernels write obar + the flux parts
                       // to every cell of the swept lines; the other cells (ghost frame of
                       // the other directions, species past nsp) must hold obar already
  double* vbar;        // optional: cotangent of v (same layout as v)
  int frank, nsp;
  int vacc;            // 1: vbar += the face cotangents (several sweeps share v), 0: vbar =
};

// minmod(a,b) branch: 0 zero, 1 a, 2 b (advec.f90:438-447)
__device__ __forceinline__ int minmod_branch(double a, double b) {
  if (a * b <= 0.0) return 0;
  return (fabs(a) < fabs(b)) ? 1 : 2;
}

// x2 / x3 sweep adjoints by marching (several fields in one launch).  One thread per (line,
// segment, species, field), lanes along i1 (coalesced): the thread walks the faces
// j0-1 .. jend+2 of its segment once, keeping the slopes of the two candidate upwind cells,
// the flux-cotangent inputs of the previous cell and the pending cotangents of cells i-2 ..
// i+1 in registers; cell i-2 is final after face i and is added to fbar.
constexpr int SVM_TJ = 32;  // cells per segment
constexpr int SVM_MAXF = 3;

struct SweepVjpFields {
  const double* f[SVM_MAXF];
  const double* obar[SVM_MAXF];
  double* fbar[SVM_MAXF];
  double* vbar[SVM_MAXF];  // x1: per-field face-velocity cotangent (written), or null
  int nsp[SVM_MAXF];
  int frank[SVM_MAXF];
  int nfld;
  int nfs;  // sum of nsp
};

// (field, species) of the flattened index fs; selects instead of indexing keep the parameter
// block out of local memory
__device__ __forceinline__ void field_of(const SweepVjpFields& FS, int fs, int& fld, int& s) {
  fld = 0;
  if (FS.nfld > 1 && fs >= FS.nsp[0]) { fs -= FS.nsp[0]; fld = 1; }
  if (FS.nfld > 2 && fld == 1 && fs >= FS.nsp[1]) { fs -= FS.nsp[1]; fld = 2; }
  s = fs;
}
template <class T>
__device__ __forceinline__ T pick3(int i, T a, T b, T c) { return (i == 0) ? a : (i == 1) ? b : c; }

struct SlopeBr {
  double val;
  int code;  // 0 zero, 1 centred, 2 twice left, 3 twice right
};

// slope(k) of advec.f90:438-447 with its branch, from f(k-1), f(k), f(k+1) (correctly rounded
// quotients, as the forward)
__device__ __forceinline__ SlopeBr slope_br(const Line1D& L, int k, double fm, double f0, double fp) {
  const double Ls = mdiv(f0 - fm, __ldg(L.dx + k), __ldg(L.ydx + k));
  const double Rs = mdiv(fp - f0, __ldg(L.dx + k + 1), __ldg(L.ydx + k + 1));
  const double Cs = mdiv(fp - fm, __ldg(L.dxs + k), __ldg(L.ydxs + k));
  const int inner = minmod_branch(2 * Ls, 2 * Rs);
  const double m1 = (inner == 0) ? 0.0 : (inner == 1) ? 2 * Ls : 2 * Rs;
  const int outer = minmod_branch(Cs, m1);
  SlopeBr r;
  r.code = (outer == 0) ? 0 : (outer == 1) ? 1 : (inner == 0) ? 0 : (inner == 1) ? 2 : 3;
  r.val = (r.code == 0) ? 0.0 : (r.code == 1) ? Cs : (r.code == 2) ? 2 * Ls : 2 * Rs;
  return r;
}

template <int DIM, bool UNIT>
__global__ void __launch_bounds__(256, 3) k_sweep_vjp_march(SweepVjpArgs P, SweepVjpFields FS, int nseg) {
  const GridDev& G = P.G;
  const Dims d = G.d;
  const int lx = (DIM == 2) ? d.lx2 : d.lx3;
  if (lx <= 1) return;
  const double dt = *P.dtp;
  const int na = d.lx1;
  const int nb = (DIM == 2) ? d.lx3 : d.lx2;
  const long long nl = (long long)na * nb;
  const long long total = nl * nseg * FS.nfs;
  const Line1D& L = G.L[DIM - 1];
  const FaceTab& FT = G.F[DIM - 1];
  const long long nfaces = (DIM == 2) ? nf2(d) : nf3(d);
  const long long stride = (DIM == 2) ? d.s2 : d.s3;                        // cells along the line
  const long long fstride = (DIM == 2) ? (long long)d.lx1 : (long long)d.lx1 * d.lx2;  // faces
  const long long mstride = (DIM == 2) ? d.s2 : G.c3;                       // cell metrics
  const long long tstride = (DIM == 2) ? FT.t2 : FT.t3;                     // face metrics
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long ln = t % nl;
    const long long r = t / nl;
    const int g = (int)(r % nseg);
    // (field, species); selects instead of indexing keep the parameter block out of local memory
    int fs = (int)(r / nseg);
    int fld = 0;
    if (FS.nfld > 1 && fs >= FS.nsp[0]) { fs -= FS.nsp[0]; fld = 1; }
    if (FS.nfld > 2 && fld == 1 && fs >= FS.nsp[1]) { fs -= FS.nsp[1]; fld = 2; }
    const int s = fs;
    const int frank = (fld == 0) ? FS.frank[0] : (fld == 1) ? FS.frank[1] : FS.frank[2];
    const int a = (int)(ln % na) + 1, b = (int)(ln / na) + 1;
    const long long c0 = (long long)s * d.ng + ((DIM == 2) ? gi(d, a, 0, b) : gi(d, a, b, 0));  // cell 0
    const long long v0 = (long long)s * nfaces + ((DIM == 2) ? f2i(d, a, 1, b) : f3i(d, a, b, 1)) - fstride;
    const long long m0 = (DIM == 2) ? cmi(G, a, 0, b) : cmi(G, a, b, 0);
    const long long t0 = ((DIM == 2) ? fmi(FT, a, 1, b) : fmi(FT, a, b, 1)) - tstride;
    const double* f = (fld == 0) ? FS.f[0] : (fld == 1) ? FS.f[1] : FS.f[2];
    const double* ob = (fld == 0) ? FS.obar[0] : (fld == 1) ? FS.obar[1] : FS.obar[2];
    double* fb = (fld == 0) ? FS.fbar[0] : (fld == 1) ? FS.fbar[1] : FS.fbar[2];
    const double* yha1 = (frank == 1) ? G.yha1_1 : G.yha1_0;
    const double* ha2t = (frank == 1) ? FT.ha2i1 : FT.ha2i0;
    auto F = [&](int j) { return __ldg(f + c0 + j * stride); };
    auto kob = [&](int j) -> double {  // d out(j)/d P(j) * obar(j), 0 outside 1..lx
      if (j < 1 || j > lx) return 0.0;
      const double y = UNIT ? 1.0 : __ldg(yha1 + m0 + j * mstride);
      return dt * __ldg(L.ydxi + j - 1) * y * __ldg(ob + c0 + j * stride);
    };
    // the global inputs of face i: f(i+1), obar(i), v(i) and the metrics
    struct In {
      double fn, ob, v, y, h, yc;
    };
    auto load = [&](int i) {
      In q;
      q.fn = F(i + 1);
      q.ob = (i >= 1 && i <= lx) ? __ldg(ob + c0 + i * stride) : 0.0;
      q.v = __ldg(P.v + v0 + i * fstride);
      q.y = q.h = q.yc = 1.0;
      if (!UNIT) {
        if (i >= 1 && i <= lx) q.y = __ldg(yha1 + m0 + i * mstride);
        q.h = __ldg(ha2t + t0 + i * tstride);
        q.yc = __ldg(FT.yhc + t0 + i * tstride);
      }
      return q;
    };
    const int j0 = -1 + g * SVM_TJ;
    const int jend = min(j0 + SVM_TJ - 1, lx + 2);
    const int i0 = max(1, j0 - 1), i1e = min(lx + 1, jend + 2);
    double fc = F(i0 - 1), fp = F(i0);                              // f(i-1), f(i)
    SlopeBr sprev = slope_br(L, i0 - 1, F(i0 - 2), fc, fp);         // slope(i-1)
    double kprev = kob(i0 - 1);
    double A0 = 0, A1 = 0, A2 = 0, A3 = 0;                          // pending cells i-2 .. i+1
    for (int i = i0; i <= i1e; ++i) {
      const In qa = load(i);
      const double fn = qa.fn;
      const SlopeBr scur = slope_br(L, i, fc, fp, fn);  // slope(i)
      const double kc = (i >= 1 && i <= lx) ? dt * __ldg(L.ydxi + i - 1) * qa.y * qa.ob : 0.0;
      const double v = qa.v;
      const double ha2 = qa.h, yhc = qa.yc;
      const double phib = ha2 * (kc - kprev);
      const double dxf = __ldg(L.dx + i);
      const double vq = v * yhc * dt;
      const bool neg = v < 0;
      const SlopeBr sk = neg ? scur : sprev;  // slope of the upwind cell k
      const int k = neg ? i : i - 1;
      const double sbar = neg ? -0.5 * v * (dxf + vq) * phib : 0.5 * v * (dxf - vq) * phib;
      const double w = (sk.code == 1) ? sbar * __ldg(L.ydxs + k) : (sk.code == 2) ? 2 * sbar * __ldg(L.ydx + k)
                       : (sk.code == 3) ? 2 * sbar * __ldg(L.ydx + k + 1) : 0.0;
      // contributions to cells k-1, k, k+1 (k = i-1: A0 A1 A2; k = i: A1 A2 A3)
      const double cm = (sk.code == 1 || sk.code == 2) ? -w : 0.0;
      const double cc = v * phib + ((sk.code == 2) ? w : (sk.code == 3) ? -w : 0.0);
      const double cp = (sk.code == 1 || sk.code == 3) ? w : 0.0;
      if (neg) { A1 += cm; A2 += cc; A3 += cp; }
      else { A0 += cm; A1 += cc; A2 += cp; }
      if (P.vbar && i >= j0 && i <= jend) {
        const double f0 = neg ? fp : fc;  // f(k)
        const double vb = neg ? phib * (f0 - 0.5 * (dxf + vq) * sk.val - 0.5 * v * (dt * yhc) * sk.val)
                              : phib * (f0 + 0.5 * (dxf - vq) * sk.val - 0.5 * v * (dt * yhc) * sk.val);
        const long long fc_ = v0 + i * fstride;
        if (P.vacc) P.vbar[fc_] += vb; else P.vbar[fc_] = vb;
      }
      // cell i-2 is final: its cotangent is obar plus the flux parts
      if (i - 2 >= j0 && i - 2 <= jend) {
        const long long q = c0 + (i - 2) * stride;
        fb[q] = __ldg(ob + q) + A0;
      }
      A0 = A1;
      A1 = A2;
      A2 = A3;
      A3 = 0.0;
      fc = fp;
      fp = fn;
      sprev = scur;
      kprev = kc;
    }
    // cells i1e-1 .. i1e+1 are final after the last face
    const double Af[3] = {A0, A1, A2};
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const int j = i1e - 1 + m;
      if (j >= j0 && j <= jend) {
        const long long q = c0 + j * stride;
        fb[q] = __ldg(ob + q) + Af[m];
      }
    }
  }
}

// x1 sweep adjoints (several fields in one launch).  One warp per (x1 line, species, field),
// lanes along the contiguous x1, the line walked in chunks of 32 positions p = -1 + 32c +
// lane.  Each lane computes the slope branch of cell p and the cotangent parts of face p
// (the upwind slope of face p is its own or lane p-1's, by shuffle, carried across chunks);
// cell p-2 then gathers from faces p-3 .. p (the four that reach it) by shuffles from this
// chunk and the previous one.  Face-velocity cotangents go to the field's own vbar slice.
template <bool UNIT>
__global__ void __launch_bounds__(256, 3) k_sweep_vjp_x1(SweepVjpArgs P, SweepVjpFields FS) {
  const GridDev& G = P.G;
  const Dims d = G.d;
  const int lx = d.lx1;
  if (lx <= 1) return;
  const double dt = *P.dtp;
  const int lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  const long long ncol = (long long)d.lx2 * d.lx3;
  const long long nwarp = ncol * FS.nfs;
  const Line1D& L = G.L[0];
  const FaceTab& FT = G.F[0];
  const long long nfaces = nf1(d);
  const int nch = (lx + 4 + 31) / 32 + 1;  // one chunk past the line flushes its last cells
  for (long long w = (long long)blockIdx.x * wpb + (threadIdx.x >> 5); w < nwarp; w += (long long)gridDim.x * wpb) {
    const long long col = w % ncol;
    int fld, s;
    field_of(FS, (int)(w / ncol), fld, s);
    const int frank = pick3(fld, FS.frank[0], FS.frank[1], FS.frank[2]);
    (void)frank;  // x1 sweeps use the frank-0 metrics
    const double* f = pick3(fld, FS.f[0], FS.f[1], FS.f[2]);
    const double* ob = pick3(fld, FS.obar[0], FS.obar[1], FS.obar[2]);
    double* fb = pick3(fld, FS.fbar[0], FS.fbar[1], FS.fbar[2]);
    double* vbar = pick3(fld, FS.vbar[0], FS.vbar[1], FS.vbar[2]);
    const int i2 = (int)(col % d.lx2) + 1, i3 = (int)(col / d.lx2) + 1;
    const long long c0 = (long long)s * d.ng + gi(d, 0, i2, i3);        // cell 0 of the line
    const long long v0 = (long long)s * nfaces + f1i(d, 1, i2, i3) - 1;  // face p at v0 + p
    const long long m0 = cmi(G, 0, i2, i3);
    const long long t0 = fmi(FT, 1, i2, i3) - FT.t1;                     // face metrics at t0 + p*t1
    // carried from the previous chunk: slope and kappa*obar of position p-1 for lane 0, and
    // the face contributions of lanes 29..31
    int ccode = 0;
    double cval = 0.0, ckob = 0.0;
    double h1p = 0.0, h2p = 0.0, h3p = 0.0;
    // f(p), obar(p), v(p) of the next chunk are loaded one chunk ahead
    auto ldf = [&](int p) { return (p >= -1 && p <= lx + 2) ? __ldg(f + c0 + p) : 0.0; };
    auto ldo = [&](int p) { return (p >= 1 && p <= lx) ? __ldg(ob + c0 + p) : 0.0; };
    auto ldv = [&](int p) { return (p >= 1 && p <= lx + 1) ? __ldg(P.v + v0 + p) : 0.0; };
    double f0n = ldf(lane - 1), obn = ldo(lane - 1), vn = ldv(lane - 1);
    for (int c = 0; c < nch; ++c) {
      const int p = -1 + 32 * c + lane;
      const double f0 = f0n, obp = obn, vp = vn;
      f0n = ldf(p + 32);
      obn = ldo(p + 32);
      vn = ldv(p + 32);
      // slope of cell p (0 .. lx+1), from f(p-1), f(p), f(p+1)
      double fm = __shfl_up_sync(0xffffffffu, f0, 1);
      double fp = __shfl_down_sync(0xffffffffu, f0, 1);
      if (lane == 0 && p - 1 >= -1) fm = __ldg(f + c0 + p - 1);
      if (lane == 31 && p + 1 <= lx + 2) fp = __ldg(f + c0 + p + 1);
      SlopeBr sc;
      sc.code = 0;
      sc.val = 0.0;
      if (p >= 0 && p <= lx + 1) sc = slope_br(L, p, fm, f0, fp);
      // kappa*obar of cell p (0 outside 1..lx)
      double kc = 0.0;
      if (p >= 1 && p <= lx) {
        const double y = UNIT ? 1.0 : __ldg(G.yha1_0 + m0 + p);
        kc = dt * __ldg(L.ydxi + p - 1) * y * obp;
      }
      // the same of position p-1
      int pcode = __shfl_up_sync(0xffffffffu, sc.code, 1);
      double pval = __shfl_up_sync(0xffffffffu, sc.val, 1);
      double pkob = __shfl_up_sync(0xffffffffu, kc, 1);
      if (lane == 0) { pcode = ccode; pval = cval; pkob = ckob; }
      // face p (1 .. lx+1): contributions to cells k-1, k, k+1 of its upwind cell k, as the
      // parts cell p-2 collects from the faces 3, 2, 1, 0 lanes up the line (g3 .. g0)
      double g0 = 0.0, g1 = 0.0, g2 = 0.0, g3 = 0.0;
      if (p >= 1 && p <= lx + 1) {
        const double v = vp;
        double ha2 = 1.0, yhc = 1.0;
        if (!UNIT) {
          ha2 = __ldg(FT.ha2i0 + t0 + p * FT.t1);
          yhc = __ldg(FT.yhc + t0 + p * FT.t1);
        }
        const double phib = ha2 * (kc - pkob);
        const double dxf = __ldg(L.dx + p);
        const double vq = v * yhc * dt;
        const bool neg = v < 0;
        const int code = neg ? sc.code : pcode;
        const double sl = neg ? sc.val : pval;
        const int k = neg ? p : p - 1;
        const double sbar = neg ? -0.5 * v * (dxf + vq) * phib : 0.5 * v * (dxf - vq) * phib;
        const double wt = (code == 1) ? sbar * __ldg(L.ydxs + k) : (code == 2) ? 2 * sbar * __ldg(L.ydx + k)
                          : (code == 3) ? 2 * sbar * __ldg(L.ydx + k + 1) : 0.0;
        const double cm = (code == 1 || code == 2) ? -wt : 0.0;
        const double cc = v * phib + ((code == 2) ? wt : (code == 3) ? -wt : 0.0);
        const double cp = (code == 1 || code == 3) ? wt : 0.0;
        // g_m: the part for cell p-2+m (gathered by the lane m up the line)
        if (neg) { g3 = cp; g2 = cc; g1 = cm; g0 = 0.0; }
        else { g3 = 0.0; g2 = cp; g1 = cc; g0 = cm; }
        if (vbar) {
          const double fk = neg ? f0 : fm;  // f(k)
          const double vb = neg ? phib * (fk - 0.5 * (dxf + vq) * sl - 0.5 * v * (dt * yhc) * sl)
                                : phib * (fk + 0.5 * (dxf - vq) * sl - 0.5 * v * (dt * yhc) * sl);
          if (P.vacc) vbar[v0 + p] += vb; else vbar[v0 + p] = vb;
        }
      }
      // cell p-2 gathers g3 of face p-3, g2 of face p-2, g1 of face p-1 and its own g0 of face p
      double acc = g0;
      {
        const int src1 = (lane - 1) & 31, src2 = (lane - 2) & 31, src3 = (lane - 3) & 31;
        const double a1 = __shfl_sync(0xffffffffu, g1, src1), b1 = __shfl_sync(0xffffffffu, h1p, src1);
        const double a2 = __shfl_sync(0xffffffffu, g2, src2), b2 = __shfl_sync(0xffffffffu, h2p, src2);
        const double a3 = __shfl_sync(0xffffffffu, g3, src3), b3 = __shfl_sync(0xffffffffu, h3p, src3);
        acc += (lane >= 1) ? a1 : b1;
        acc += (lane >= 2) ? a2 : b2;
        acc += (lane >= 3) ? a3 : b3;
      }
      const int pc = p - 2;
      if (pc >= -1 && pc <= lx + 2) fb[c0 + pc] = __ldg(ob + c0 + pc) + acc;
      // carry to the next chunk
      ccode = __shfl_sync(0xffffffffu, sc.code, 31);
      cval = __shfl_sync(0xffffffffu, sc.val, 31);
      ckob = __shfl_sync(0xffffffffu, kc, 31);
      h1p = g1;
      h2p = g2;
      h3p = g3;
    }
  }
}

// ======================================================================================
// 8. CFL time step (temporal_mpi.f90:86-167), max CFL (temporal.f90:12-49), finiteness
// ======================================================================================
#ifndef GEM_DT_UNROLL
#define GEM_DT_UNROLL 2
#endif
#ifndef GEM_DT_MINB
#define GEM_DT_MINB 4
#endif
constexpr int kDtUnroll = GEM_DT_UNROLL;  // x1 cells per thread in flight
// Rates are >= 0, so their IEEE bit patterns order like unsigned integers and the block
// maxima combine with 64-bit atomicMax; max is exact, so the result is independent of the
// reduction order and equals the reference's sequential loop.
// Block (32, LSP): threadIdx.y is the species, lanes run along x1, blocks stride over the
// x1 rows (i2, i3).  Each thread keeps the three running maxima of its species.
// The CFL rates of one interior cell and species (temporal_mpi.f90:127-150): dl = dxi*h
// (multifluid.f90:764-770), tabulated per cell with its reciprocal; vsnd from T and Te for
// the ions; every quotient exact (mdiv_try, else the IEEE division).  MODE 0 keeps the
// per-direction maxima g1, g2, g3; MODE 1 (maxcfl) the largest dtv*rate in g1.
template <bool UNIT, int MODE>
__device__ __forceinline__ void dt_cell(const GridDev& G, long long mk, int i1, double dx2i, double ydx2i, double dx3i,
                                        double ydx3i, int s, double T, double Te, double v1, double v2, double v3,
                                        double dtv, double& g1, double& g2, double& g3) {
  const double ms = c_ms[s], yms = c_yms[s];
  double dl1, y1, dl2, y2, dl3, y3;
  if (UNIT) {
    dl1 = __ldg(G.L[0].dxi + i1 - 1);
    y1 = __ldg(G.L[0].ydxi + i1 - 1);
    dl2 = dx2i;
    y2 = ydx2i;
    dl3 = dx3i;
    y3 = ydx3i;
  } else {
    dl1 = __ldg(G.dl[0] + mk);
    y1 = __ldg(G.ydl[0] + mk);
    dl2 = __ldg(G.dl[1] + mk);
    y2 = __ldg(G.ydl[1] + mk);
    if (G.dl3_tab) {
      dl3 = __ldg(G.dl[2] + mk);
      y3 = __ldg(G.ydl[2] + mk);
    } else {
      dl3 = dx3i * __ldg(G.h3 + mk);
      y3 = 1.0 / dl3;
    }
  }
  bool ok = true;
  double vsnd = 0.0;
  if (s < LSP - 1) vsnd = sqrt(mdiv_try(KB * T, ms, yms, ok) + mdiv_try(5.0 / 3.0 * KB * Te, ms, yms, ok));
  double r1, r2, r3;
  if (MODE == 0) {
    r1 = mdiv_try(vsnd + fabs(v1), dl1, y1, ok);
    r2 = mdiv_try(fabs(v2), dl2, y2, ok);
    r3 = mdiv_try(fabs(v3), dl3, y3, ok);
  } else {
    r1 = mdiv_try(dtv * (vsnd + fabs(v1)), dl1, y1, ok);
    r2 = mdiv_try(dtv * fabs(v2), dl2, y2, ok);
    r3 = mdiv_try(dtv * fabs(v3), dl3, y3, ok);
  }
  if (!ok) {  // rare: a quotient outside the exact fast range
    vsnd = 0.0;
    if (s < LSP - 1) vsnd = sqrt(slow_div(KB * T, ms) + slow_div(5.0 / 3.0 * KB * Te, ms));
    const double a1 = (MODE == 0) ? vsnd + fabs(v1) : dtv * (vsnd + fabs(v1));
    const double a2 = (MODE == 0) ? fabs(v2) : dtv * fabs(v2);
    const double a3 = (MODE == 0) ? fabs(v3) : dtv * fabs(v3);
    r1 = slow_div(a1, dl1);
    r2 = slow_div(a2, dl2);
    r3 = slow_div(a3, dl3);
  }
  if (MODE == 0) {
    g1 = fmax_f(r1, g1);
    g2 = fmax_f(r2, g2);
    g3 = fmax_f(r3, g3);
  } else {
    g1 = fmax_f(r1, g1);
    g1 = fmax_f(r2, g1);
    g1 = fmax_f(r3, g1);
  }
}

template <bool UNIT, int MODE /*0 gridrates, 1 maxcfl*/>
__device__ __forceinline__ void b_dt_reduce(const GridDev& G, const Blocks& B, unsigned long long* acc /*3*LSP*/,
                                                        const double* dtp, const VB vb) {
  const Dims d = G.d;
  const int s = threadIdx.y;
  const int lane = threadIdx.x;
  double g1 = 0.0, g2 = 0.0, g3 = 0.0;
  const double dtv = (MODE == 1) ? *dtp : 0.0;
  const int nrow = d.lx2 * d.lx3;
  const double* Tsp = B.Ts(s);
  const double* Tep = B.Ts(LSP - 1);
  const double* v1p = B.vs1(s);
  const double* v2p = B.vs2(s);
  const double* v3p = B.vs3(s);
  for (int row = vb.bx; row < nrow; row += vb.gx) {
    const int i2 = row % d.lx2 + 1, i3 = row / d.lx2 + 1;
    const long long k0 = gi(d, 0, i2, i3);
    const long long m0 = cmi(G, 0, i2, i3);
    const double dx2i = __ldg(G.L[1].dxi + i2 - 1), ydx2i = __ldg(G.L[1].ydxi + i2 - 1);
    const double dx3i = __ldg(G.L[2].dxi + i3 - 1), ydx3i = __ldg(G.L[2].ydxi + i3 - 1);
#pragma unroll kDtUnroll
    for (int i1 = lane + 1; i1 <= d.lx1; i1 += 32) {
      const long long k = k0 + i1;
      dt_cell<UNIT, MODE>(G, m0 + i1, i1, dx2i, ydx2i, dx3i, ydx3i, s, Tsp[k], Tep[k], v1p[k], v2p[k], v3p[k], dtv, g1,
                          g2, g3);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    g1 = fmax_f(g1, __shfl_down_sync(0xffffffffu, g1, o));
    if (MODE == 0) {
      g2 = fmax_f(g2, __shfl_down_sync(0xffffffffu, g2, o));
      g3 = fmax_f(g3, __shfl_down_sync(0xffffffffu, g3, o));
    }
  }
  if (lane == 0) {
    if (MODE == 0) {
      atomicMax(acc + s, (unsigned long long)__double_as_longlong(g1));
      atomicMax(acc + LSP + s, (unsigned long long)__double_as_longlong(g2));
      atomicMax(acc + 2 * LSP + s, (unsigned long long)__double_as_longlong(g3));
    } else {
      atomicMax(acc, (unsigned long long)__double_as_longlong(g1));
    }
  }
}

template <bool UNIT, int MODE /*0 gridrates, 1 maxcfl*/>
__global__ void __launch_bounds__(32 * LSP, GEM_DT_MINB) k_dt_reduce(GridDev G, Blocks B, unsigned long long* acc /*3*LSP*/,
                                                        const double* dtp) {
  b_dt_reduce<UNIT, MODE>(G, B, acc, dtp, VB{(int)blockIdx.x, (int)blockIdx.y, (int)gridDim.x});
}


// Per-x3-plane partial maxima of the dt rates (block i3 covers the plane's x1 rows):
// part[(i3-1)*3*LSP + slot], slot as in k_dt_reduce.  Every slot of every plane is written.
template <bool UNIT>
__global__ void __launch_bounds__(32 * LSP) k_dt_reduce_planes(GridDev G, Blocks B, double* part) {
  const Dims d = G.d;
  const int s = threadIdx.y;
  const int lane = threadIdx.x;
  const int i3 = blockIdx.x + 1;
  double g1 = 0.0, g2 = 0.0, g3 = 0.0;
  const double ms = c_ms[s];
  const double dx3i = __ldg(G.L[2].dxi + i3 - 1);
  for (int i2 = 1; i2 <= d.lx2; ++i2) {
    const long long k0 = gi(d, 0, i2, i3);
    const long long m0 = cmi(G, 0, i2, i3);
    const double dx2i = __ldg(G.L[1].dxi + i2 - 1);
    for (int i1 = lane + 1; i1 <= d.lx1; i1 += 32) {
      const long long k = k0 + i1;
      const double dl1 = __ldg(G.L[0].dxi + i1 - 1) * ldm<UNIT>(G.h1, m0 + i1);
      const double dl2 = dx2i * ldm<UNIT>(G.h2, m0 + i1);
      const double dl3 = dx3i * ldm<UNIT>(G.h3, m0 + i1);
      double vsnd = 0.0;
      if (s < LSP - 1) vsnd = sqrt(KB * B.Ts(s)[k] / ms + 5.0 / 3.0 * KB * B.Ts(LSP - 1)[k] / ms);
      g1 = fmax_f((vsnd + fabs(B.vs1(s)[k])) / dl1, g1);
      g2 = fmax_f(fabs(B.vs2(s)[k]) / dl2, g2);
      g3 = fmax_f(fabs(B.vs3(s)[k]) / dl3, g3);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    g1 = fmax_f(g1, __shfl_down_sync(0xffffffffu, g1, o));
    g2 = fmax_f(g2, __shfl_down_sync(0xffffffffu, g2, o));
    g3 = fmax_f(g3, __shfl_down_sync(0xffffffffu, g3, o));
  }
  if (lane == 0) {
    double* p = part + (long long)(i3 - 1) * 3 * LSP;
    p[s] = g1;
    p[LSP + s] = g2;
    p[2 * LSP + s] = g3;
  }
}

// max over the planes per slot, then the k_dt_finalize formula (one warp)
__global__ void k_dt_finalize_planes(const double* part, int nplane, double tcfl, double* dt_out) {
  const int lane = threadIdx.x;
  double m = 0.0;
  for (int q = 0; q < 3 * LSP; ++q) {
    double g = 0.0;
    for (int p = lane; p < nplane; p += 32) g = fmax_f(part[(long long)p * 3 * LSP + q], g);
    for (int o = 16; o > 0; o >>= 1) g = fmax_f(g, __shfl_xor_sync(0xffffffffu, g, o));
    const double inv = 1.0 / fmax_f(g, 1e-10);
    if (q == 0 || inv < m) m = inv;
  }
  if (lane == 0) *dt_out = fmax_f(tcfl * m, 1e-6);
}

__global__ void k_dt_finalize(const unsigned long long* acc, double tcfl, double* dt_out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double m = 0.0;
  for (int q = 0; q < 3 * LSP; ++q) {
    const double gr = fmax_f(__longlong_as_double((long long)acc[q]), 1e-10);
    const double inv = 1.0 / gr;
    if (q == 0 || inv < m) m = inv;
  }
  *dt_out = fmax_f(tcfl * m, 1e-6);
}

__global__ void k_maxcfl_finalize(const unsigned long long* acc, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *out = __longlong_as_double((long long)acc[0]);
}

__global__ void k_count_nonfinite(GridDev G, Blocks B, unsigned long long* cnt) {
  const Dims d = G.d;
  const long long nc = nci(d);
  unsigned long long local = 0;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nc;
       q += (long long)gridDim.x * blockDim.x) {
    const int i1 = (int)(q % d.lx1) + 1;
    const long long r = q / d.lx1;
    const int i2 = (int)(r % d.lx2) + 1, i3 = (int)(r / d.lx2) + 1;
    const long long k = gi(d, i1, i2, i3);
    for (int s = 0; s < LSP; ++s) {
      local += !isfinite(B.ns(s)[k]);
      local += !isfinite(B.vs1(s)[k]);
      local += !isfinite(B.Ts(s)[k]);
    }
  }
  for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(cnt, local);
}

}  // namespace gemk
