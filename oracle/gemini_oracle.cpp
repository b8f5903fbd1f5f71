// TEST INFRASTRUCTURE -- NOT PART OF THE PRODUCT.
//
// CPU restatement ("oracle") of the GEMINI3D multifluid fluid-advance hot path:
// the MC-limited advection sweeps, the global-boundary ghost fill, the interface
// velocities, the state conversions, clean_param, thermal conductivity, the
// TRBDF2 / backward-Euler field-aligned diffusion (with LAPACK's partial-pivoting
// band LU restated from its published algorithm) and the CFL time step; and, ahead of
// its device version, the compression sub-step (artificial viscosity, the RK2
// zero-order-hold ghosts, div3D_curv_23 and the two-stage energy update) and the
// source/loss ETD solves, with the continuity, momentum and energy equations'
// production/loss rates and the collision frequencies they use.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
// library, as the checker.  The product (gemini_b200/) never links or calls it.
//
// Every function follows the Fortran it cites line by line: same operation order
// (Fortran evaluates a*b/c*d left to right), same slice semantics, no FMA
// contraction (build with -ffp-contract=off, as gfortran emits for x86-64 without
// -march), x**2 -> x*x, x**(5.0_wp/2) -> pow(x,2.5).  Array layouts are the
// reference's Fortran layouts (column-major, x1 fastest, 2 ghost cells per side,
// species/variable slowest).  Citations are paths inside gemini3d/gemini.
//
// Parity pins: the 1-D TRBDF2 / backward-Euler drivers reproduce the golden values
// of test/diffusion/test_diffusion1D.py:32-36, and the band solver is checked
// against LAPACK dgbsv from scipy's bundled OpenBLAS (tests/).  The advection
// sweeps have no reference test; they are pinned only by this restatement.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---- constants: src/numerical/constants/phys_consts.in.f90:20-84 ------------------
constexpr int LSP = 7;
const double kB = 1.38064852e-23;
const double elchrg = 1.60217662e-19;
const double amu = 1.660539040e-27;
const double mindens = 1.0e-100;
const double mindensnull = 1.0e-20;
const double mindensdiv = 1.0e-5;

struct Consts {
  double ms[LSP], qs[LSP], gammas[LSP], thermal_coeff[LSP - 1];
  Consts() {
    // phys_consts.in.f90:43  ms=[real(wp) :: 16,30,28,32,14,1,5.485799090e-4_wp]*amu
    const double m[LSP] = {16.0, 30.0, 28.0, 32.0, 14.0, 1.0, 5.485799090e-4};
    for (int i = 0; i < LSP; ++i) ms[i] = m[i] * amu;
    // phys_consts.in.f90:45
    for (int i = 0; i < LSP - 1; ++i) qs[i] = 1.0 * elchrg;
    qs[LSP - 1] = -1.0 * elchrg;
    // phys_consts.in.f90:47-53
    const double g53 = 5.0 / 3, g75 = 7.0 / 5;
    const double g[LSP] = {g53, g75, g75, g75, g53, g53, g53};
    for (int i = 0; i < LSP; ++i) gammas[i] = g[i];
    // collisions.f90:51-53: default-REAL literals widened to real(wp)
    const float tc[LSP - 1] = {0.1019e-12f, 0.0747e-12f, 0.0754e-12f,
                               0.0701e-12f, 0.1068e-12f, 0.3986e-12f};
    for (int i = 0; i < LSP - 1; ++i) thermal_coeff[i] = (double)tc[i];
  }
};
const Consts K;

inline double fmax_f(double a, double b) { return (a > b) ? a : b; }
inline double fmin_f(double a, double b) { return (a < b) ? a : b; }

}  // namespace

extern "C" {

// Grid description: the curvmesh fields the hot path reads (meshobj.f90:49-154).
struct ora_grid {
  int lx1, lx2, lx3;
  int gridflag;  // 0 closed dipole, 1 open inverted, 2 non-inverted (meshobj.f90:549-570)
  int flagper;   // x3 periodic (meshobj.f90:324-335)
  const double *dx1, *dx1i, *dx2, *dx2i, *dx3, *dx3i;  // dx: 0..l+2, dxi: 1..l
  const double *h1, *h2, *h3;                           // (-1:lx1+2,-1:lx2+2,-1:lx3+2)
  const double *h1x1i, *h2x1i, *h3x1i;                  // (1:lx1+1,1:lx2,1:lx3)
  const double *h1x2i, *h2x2i, *h3x2i;                  // (1:lx1,1:lx2+1,1:lx3)
  const double *h1x3i, *h2x3i, *h3x3i;                  // (1:lx1,1:lx2,1:lx3+1)
  const unsigned char* nullpts;                         // (1:lx1,1:lx2,1:lx3) or NULL
};

}  // extern "C"

namespace {

struct Ix {
  int lx1, lx2, lx3;
  long long s2, s3, ng;  // strides of a ghosted array
  explicit Ix(const ora_grid* g) : lx1(g->lx1), lx2(g->lx2), lx3(g->lx3) {
    s2 = lx1 + 4;
    s3 = (long long)(lx1 + 4) * (lx2 + 4);
    ng = s3 * (lx3 + 4);
  }
  // ghosted (-1:lx1+2,-1:lx2+2,-1:lx3+2)
  long long g(int i1, int i2, int i3) const { return (i1 + 1) + s2 * (i2 + 1) + s3 * (i3 + 1); }
  // interior-only (1:lx1,1:lx2,1:lx3)
  long long c(int i1, int i2, int i3) const {
    return (i1 - 1) + (long long)lx1 * ((i2 - 1) + (long long)lx2 * (i3 - 1));
  }
  long long nc() const { return (long long)lx1 * lx2 * lx3; }
  // x1 faces (1:lx1+1,1:lx2,1:lx3)
  long long f1(int i1, int i2, int i3) const {
    return (i1 - 1) + (long long)(lx1 + 1) * ((i2 - 1) + (long long)lx2 * (i3 - 1));
  }
  long long nf1() const { return (long long)(lx1 + 1) * lx2 * lx3; }
  // x2 faces (1:lx1,1:lx2+1,1:lx3)
  long long f2(int i1, int i2, int i3) const {
    return (i1 - 1) + (long long)lx1 * ((i2 - 1) + (long long)(lx2 + 1) * (i3 - 1));
  }
  long long nf2() const { return (long long)lx1 * (lx2 + 1) * lx3; }
  // x3 faces (1:lx1,1:lx2,1:lx3+1)
  long long f3(int i1, int i2, int i3) const {
    return (i1 - 1) + (long long)lx1 * ((i2 - 1) + (long long)lx2 * (i3 - 1));
  }
  long long nf3() const { return (long long)lx1 * lx2 * (lx3 + 1); }
};

// ---- advec.f90:438-447 -------------------------------------------------------------
inline double minmod(double a, double b) {
  if (a * b <= 0.0) return 0.0;
  if (std::fabs(a) < std::fabs(b)) return a;
  return b;
}

// ---- advec.f90:384-435 advec1D_MC_curv ---------------------------------------------
// f,ha1,out: index -1..lx+2 stored at [i+1]; v1i,ha2i,h1i: 1..lx+1 at [i-1];
// dx: 0..lx+2 at [i]; dxi: 1..lx at [i-1].  phi/slope: scratch of lx+2.
void advec1D_MC_curv(const double* f, const double* v1i, double dt, const double* dx,
                     const double* dxi, const double* ha1, const double* ha2i,
                     const double* h1i, int lx, double* out, double* phi, double* slope) {
#define F_(i) f[(i) + 1]
  if (lx > 1) {
    double lslope = (F_(0) - F_(-1)) / dx[0];
    for (int i = 0; i <= lx + 1; ++i) {
      double rslope = (F_(i + 1) - F_(i)) / dx[i + 1];
      double cslope = (F_(i + 1) - F_(i - 1)) / (dx[i] + dx[i + 1]);
      slope[i] = minmod(cslope, minmod(2 * lslope, 2 * rslope));
      lslope = rslope;
    }
    for (int i = 1; i <= lx + 1; ++i) {
      const double v = v1i[i - 1];
      if (v < 0) {
        phi[i] = F_(i) * v - 0.5 * v * (dx[i] + v / h1i[i - 1] * dt) * slope[i];
      } else {
        phi[i] = F_(i - 1) * v + 0.5 * v * (dx[i] - v / h1i[i - 1] * dt) * slope[i - 1];
      }
    }
    for (int i = 1; i <= lx; ++i) {
      out[i + 1] = F_(i) - dt * (ha2i[i] * phi[i + 1] - ha2i[i - 1] * phi[i]) / dxi[i - 1] / ha1[i + 1];
    }
    out[0] = F_(-1);
    out[1] = F_(0);
    out[lx + 2] = F_(lx + 1);
    out[lx + 3] = F_(lx + 2);
  } else {
    for (int i = -1; i <= lx + 2; ++i) out[i + 1] = F_(i);
  }
#undef F_
}

// ---- advec.f90:283-309 sweep1 ----------------------------------------------------
void sweep1(const ora_grid* G, double* f, const double* v1i, double dt) {
  Ix X(G);
  const int lx1 = G->lx1;
#pragma omp parallel
  {
    std::vector<double> fl(lx1 + 4), out(lx1 + 4), ha1(lx1 + 4), ha2i(lx1 + 1), h1i(lx1 + 1),
        v(lx1 + 1), phi(lx1 + 2), slope(lx1 + 2);
#pragma omp for collapse(2) schedule(static)
    for (int i3 = 1; i3 <= G->lx3; ++i3) {
      for (int i2 = 1; i2 <= G->lx2; ++i2) {
        for (int i1 = -1; i1 <= lx1 + 2; ++i1) {
          const long long k = X.g(i1, i2, i3);
          fl[i1 + 1] = f[k];
          ha1[i1 + 1] = G->h1[k] * G->h2[k] * G->h3[k];
        }
        for (int i1 = 1; i1 <= lx1 + 1; ++i1) {
          const long long k = X.f1(i1, i2, i3);
          v[i1 - 1] = v1i[k];
          ha2i[i1 - 1] = G->h2x1i[k] * G->h3x1i[k];
          h1i[i1 - 1] = G->h1x1i[k];
        }
        advec1D_MC_curv(fl.data(), v.data(), dt, G->dx1, G->dx1i, ha1.data(), ha2i.data(),
                        h1i.data(), lx1, out.data(), phi.data(), slope.data());
        for (int i1 = -1; i1 <= lx1 + 2; ++i1) f[X.g(i1, i2, i3)] = out[i1 + 1];
      }
    }
  }
}

// ---- advec.f90:313-345 sweep2 ----------------------------------------------------
void sweep2(const ora_grid* G, double* f, const double* v2i, double dt, int frank) {
  Ix X(G);
  const int lx2 = G->lx2;
#pragma omp parallel
  {
    std::vector<double> fl(lx2 + 4), out(lx2 + 4), ha1(lx2 + 4), ha2i(lx2 + 1), h1i(lx2 + 1),
        v(lx2 + 1), phi(lx2 + 2), slope(lx2 + 2);
#pragma omp for collapse(2) schedule(static)
    for (int i3 = 1; i3 <= G->lx3; ++i3) {
      for (int i1 = 1; i1 <= G->lx1; ++i1) {
        for (int i2 = -1; i2 <= lx2 + 2; ++i2) {
          const long long k = X.g(i1, i2, i3);
          fl[i2 + 1] = f[k];
          if (frank == 0)
            ha1[i2 + 1] = G->h1[k] * G->h2[k] * G->h3[k];
          else
            ha1[i2 + 1] = G->h1[k] * G->h1[k] * G->h2[k] * G->h3[k];
        }
        for (int i2 = 1; i2 <= lx2 + 1; ++i2) {
          const long long k = X.f2(i1, i2, i3);
          v[i2 - 1] = v2i[k];
          if (frank == 0)
            ha2i[i2 - 1] = G->h1x2i[k] * G->h3x2i[k];
          else
            ha2i[i2 - 1] = G->h1x2i[k] * G->h1x2i[k] * G->h3x2i[k];
          h1i[i2 - 1] = G->h2x2i[k];
        }
        advec1D_MC_curv(fl.data(), v.data(), dt, G->dx2, G->dx2i, ha1.data(), ha2i.data(),
                        h1i.data(), lx2, out.data(), phi.data(), slope.data());
        for (int i2 = -1; i2 <= lx2 + 2; ++i2) f[X.g(i1, i2, i3)] = out[i2 + 1];
      }
    }
  }
}

// ---- advec.f90:349-381 sweep3 ----------------------------------------------------
void sweep3(const ora_grid* G, double* f, const double* v3i, double dt, int frank) {
  Ix X(G);
  const int lx3 = G->lx3;
#pragma omp parallel
  {
    std::vector<double> fl(lx3 + 4), out(lx3 + 4), ha1(lx3 + 4), ha2i(lx3 + 1), h1i(lx3 + 1),
        v(lx3 + 1), phi(lx3 + 2), slope(lx3 + 2);
#pragma omp for collapse(2) schedule(static)
    for (int i2 = 1; i2 <= G->lx2; ++i2) {
      for (int i1 = 1; i1 <= G->lx1; ++i1) {
        for (int i3 = -1; i3 <= lx3 + 2; ++i3) {
          const long long k = X.g(i1, i2, i3);
          fl[i3 + 1] = f[k];
          if (frank == 0)
            ha1[i3 + 1] = G->h1[k] * G->h2[k] * G->h3[k];
          else
            ha1[i3 + 1] = G->h1[k] * G->h1[k] * G->h2[k] * G->h3[k];
        }
        for (int i3 = 1; i3 <= lx3 + 1; ++i3) {
          const long long k = X.f3(i1, i2, i3);
          v[i3 - 1] = v3i[k];
          if (frank == 0)
            ha2i[i3 - 1] = G->h1x3i[k] * G->h2x3i[k];
          else
            ha2i[i3 - 1] = G->h1x3i[k] * G->h1x3i[k] * G->h2x3i[k];
          h1i[i3 - 1] = G->h3x3i[k];
        }
        advec1D_MC_curv(fl.data(), v.data(), dt, G->dx3, G->dx3i, ha1.data(), ha2i.data(),
                        h1i.data(), lx3, out.data(), phi.data(), slope.data());
        for (int i3 = -1; i3 <= lx3 + 2; ++i3) f[X.g(i1, i2, i3)] = out[i3 + 1];
      }
    }
  }
}

// ---- mpihalo.f90:147-151: single-rank x3 periodic self-wrap, lhalo=2 --------------
// Rows 1:lx2 only, all x1 including ghosts.  Fortran array-assignment semantics: the
// right-hand side is read completely before the left-hand side is written.
void halo_periodic(const ora_grid* G, double* p) {
  if (!G->flagper) return;
  Ix X(G);
  const int lx3 = G->lx3;
  std::vector<double> tmp((size_t)(G->lx1 + 4) * G->lx2 * 2);
  auto copy_slab = [&](int dst0, int src0) {
    size_t t = 0;
    for (int j = 0; j < 2; ++j)
      for (int i2 = 1; i2 <= G->lx2; ++i2)
        for (int i1 = -1; i1 <= G->lx1 + 2; ++i1) tmp[t++] = p[X.g(i1, i2, src0 + j)];
    t = 0;
    for (int j = 0; j < 2; ++j)
      for (int i2 = 1; i2 <= G->lx2; ++i2)
        for (int i1 = -1; i1 <= G->lx1 + 2; ++i1) p[X.g(i1, i2, dst0 + j)] = tmp[t++];
  };
  copy_slab(-1, lx3 - 1);  // param(:,1:lx2,-1:0) = param(:,1:lx2,lx3-1:lx3)
  copy_slab(lx3 + 1, 1);   // param(:,1:lx2,lx3+1:lx3+2) = param(:,1:lx2,1:2)
}

}  // namespace

extern "C" {

// Layout helpers for callers.
long long ora_ghosted_size(int lx1, int lx2, int lx3) {
  return (long long)(lx1 + 4) * (lx2 + 4) * (lx3 + 4);
}

void ora_constants(double* ms, double* qs, double* gammas, double* thermal_coeff) {
  for (int i = 0; i < LSP; ++i) {
    ms[i] = K.ms[i];
    qs[i] = K.qs[i];
    gammas[i] = K.gammas[i];
  }
  for (int i = 0; i < LSP - 1; ++i) thermal_coeff[i] = K.thermal_coeff[i];
}

// advec.f90:384-435 on one line (test hook).
void ora_advec1D_MC_curv(const double* f, const double* v1i, double dt, const double* dx,
                         const double* dxi, const double* ha1, const double* ha2i,
                         const double* h1i, int lx, double* out) {
  std::vector<double> phi(lx + 2), slope(lx + 2);
  advec1D_MC_curv(f, v1i, dt, dx, dxi, ha1, ha2i, h1i, lx, out, phi.data(), slope.data());
}

// advec.f90:233-279 sweep{1,2,3}_allspec: first `lsp` species of a 4-D ghosted array.
// multifluid.f90:49-126 fixes (frank, lsp): mass (0,6), momentum (1,6), energy (0,7).
void ora_sweep_allspec(const ora_grid* G, int dim, double* fs, const double* vsi, double dt,
                       int frank, int lsp) {
  Ix X(G);
  for (int s = 0; s < lsp; ++s) {
    double* f = fs + s * X.ng;
    if (dim == 1) sweep1(G, f, vsi + s * X.nf1(), dt);
    if (dim == 2) sweep2(G, f, vsi + s * X.nf2(), dt, frank);
    if (dim == 3) sweep3(G, f, vsi + s * X.nf3(), dt, frank);
  }
}

// ---- advec.f90:21-149 set_global_boundaries(_allspec), single rank (all isglobal*) --
// ns, rhovs1, vs1, vs2, vs3, rhoes: ghosted (.,lsp); vs1i: (lx1+1,lx2,lx3,lsp).
void ora_set_global_boundaries_allspec(const ora_grid* G, double* ns, double* rhovs1,
                                       const double* vs1, double* vs2, double* vs3,
                                       double* rhoes, const double* vs1i, int lsp) {
  Ix X(G);
  const int lx1 = G->lx1, lx2 = G->lx2, lx3 = G->lx3;
  for (int s = 0; s < lsp; ++s) {
    double* n = ns + s * X.ng;
    double* rv = rhovs1 + s * X.ng;
    const double* v1 = vs1 + s * X.ng;
    double* v2 = vs2 + s * X.ng;
    double* v3 = vs3 + s * X.ng;
    double* re = rhoes + s * X.ng;
    const double* v1i = vs1i + s * X.nf1();
    const double msp = K.ms[s];
    // x1 minimum (advec.f90:42-60)
    for (int i3 = 1; i3 <= lx3; ++i3)
      for (int i2 = 1; i2 <= lx2; ++i2) {
        const double coeff = n[X.g(2, i2, i3)] / n[X.g(3, i2, i3)];
        n[X.g(0, i2, i3)] = fmin_f(coeff * n[X.g(1, i2, i3)], n[X.g(1, i2, i3)]);
        n[X.g(-1, i2, i3)] = fmin_f(coeff * n[X.g(0, i2, i3)], n[X.g(0, i2, i3)]);
      }
    for (int i3 = 1; i3 <= lx3; ++i3)
      for (int i2 = 1; i2 <= lx2; ++i2)
        rv[X.g(0, i2, i3)] = 2 * v1i[X.f1(1, i2, i3)] - v1[X.g(1, i2, i3)];
    for (int i3 = -1; i3 <= lx3 + 2; ++i3)
      for (int i2 = -1; i2 <= lx2 + 2; ++i2)
        rv[X.g(-1, i2, i3)] = rv[X.g(0, i2, i3)] + rv[X.g(0, i2, i3)] - v1[X.g(1, i2, i3)];
    for (int i3 = -1; i3 <= lx3 + 2; ++i3)
      for (int i2 = -1; i2 <= lx2 + 2; ++i2)
        for (int i1 = -1; i1 <= 0; ++i1) {
          const long long k = X.g(i1, i2, i3);
          rv[k] = rv[k] * n[k] * msp;
        }
    for (int i3 = -1; i3 <= lx3 + 2; ++i3)
      for (int i2 = -1; i2 <= lx2 + 2; ++i2) {
        const double Tb = re[X.g(1, i2, i3)] / n[X.g(1, i2, i3)];
        re[X.g(0, i2, i3)] = Tb * n[X.g(0, i2, i3)];
        re[X.g(-1, i2, i3)] = Tb * n[X.g(-1, i2, i3)];
      }
    // x1 maximum (advec.f90:61-79)
    for (int i3 = 1; i3 <= lx3; ++i3)
      for (int i2 = 1; i2 <= lx2; ++i2) {
        const double coeff = n[X.g(lx1 - 1, i2, i3)] / n[X.g(lx1 - 2, i2, i3)];
        n[X.g(lx1 + 1, i2, i3)] = fmin_f(coeff * n[X.g(lx1, i2, i3)], n[X.g(lx1, i2, i3)]);
        n[X.g(lx1 + 2, i2, i3)] =
            fmin_f(coeff * n[X.g(lx1 + 1, i2, i3)], n[X.g(lx1 + 1, i2, i3)]);
      }
    for (int i3 = 1; i3 <= lx3; ++i3)
      for (int i2 = 1; i2 <= lx2; ++i2)
        rv[X.g(lx1 + 1, i2, i3)] = 2 * v1i[X.f1(lx1 + 1, i2, i3)] - v1[X.g(lx1, i2, i3)];
    for (int i3 = -1; i3 <= lx3 + 2; ++i3)
      for (int i2 = -1; i2 <= lx2 + 2; ++i2)
        rv[X.g(lx1 + 2, i2, i3)] =
            rv[X.g(lx1 + 1, i2, i3)] + rv[X.g(lx1 + 1, i2, i3)] - v1[X.g(lx1, i2, i3)];
    for (int i3 = -1; i3 <= lx3 + 2; ++i3)
      for (int i2 = -1; i2 <= lx2 + 2; ++i2)
        for (int i1 = lx1 + 1; i1 <= lx1 + 2; ++i1) {
          const long long k = X.g(i1, i2, i3);
          rv[k] = rv[k] * n[k] * msp;
        }
    for (int i3 = -1; i3 <= lx3 + 2; ++i3)
      for (int i2 = -1; i2 <= lx2 + 2; ++i2) {
        const double Tb = re[X.g(lx1, i2, i3)] / n[X.g(lx1, i2, i3)];
        re[X.g(lx1 + 1, i2, i3)] = Tb * n[X.g(lx1 + 1, i2, i3)];
        re[X.g(lx1 + 2, i2, i3)] = Tb * n[X.g(lx1 + 2, i2, i3)];
      }
    // x2 (advec.f90:83-104): never periodic
    double* arrs2[4] = {v2, n, rv, re};
    for (double* a : arrs2)
      for (int i3 = -1; i3 <= lx3 + 2; ++i3)
        for (int i1 = -1; i1 <= lx1 + 2; ++i1) {
          a[X.g(i1, 0, i3)] = a[X.g(i1, 1, i3)];
          a[X.g(i1, -1, i3)] = a[X.g(i1, 1, i3)];
        }
    for (double* a : arrs2)
      for (int i3 = -1; i3 <= lx3 + 2; ++i3)
        for (int i1 = -1; i1 <= lx1 + 2; ++i1) {
          a[X.g(i1, lx2 + 1, i3)] = a[X.g(i1, lx2, i3)];
          a[X.g(i1, lx2 + 2, i3)] = a[X.g(i1, lx2, i3)];
        }
    // x3 (advec.f90:107-132)
    if (!G->flagper) {
      double* arrs3[4] = {v3, n, rv, re};
      for (double* a : arrs3)
        for (int i2 = -1; i2 <= lx2 + 2; ++i2)
          for (int i1 = -1; i1 <= lx1 + 2; ++i1) {
            a[X.g(i1, i2, 0)] = a[X.g(i1, i2, 1)];
            a[X.g(i1, i2, -1)] = a[X.g(i1, i2, 1)];
          }
      for (double* a : arrs3)
        for (int i2 = -1; i2 <= lx2 + 2; ++i2)
          for (int i1 = -1; i1 <= lx1 + 2; ++i1) {
            a[X.g(i1, i2, lx3 + 1)] = a[X.g(i1, i2, lx3)];
            a[X.g(i1, i2, lx3 + 2)] = a[X.g(i1, i2, lx3)];
          }
    }
  }
}

// multifluid_mpi.f90:12-19 halo_allparams (single rank: periodic wrap only).
void ora_halo_allparams(const ora_grid* G, double* ns, double* rhovs1, double* rhoes) {
  Ix X(G);
  for (int s = 0; s < LSP; ++s) {
    halo_periodic(G, ns + s * X.ng);
    halo_periodic(G, rhovs1 + s * X.ng);
    halo_periodic(G, rhoes + s * X.ng);
  }
}

// multifluid_mpi.f90:23-41 halo_fluidvars (single rank).
void ora_halo_fluidvars(const ora_grid* G, double* ns, double* rhovs1, double* rhoes,
                        double* vs2, double* vs3) {
  Ix X(G);
  ora_halo_allparams(G, ns, rhovs1, rhoes);
  for (int s = 0; s < LSP; ++s) halo_periodic(G, vs2 + s * X.ng);
  for (int s = 0; s < LSP; ++s) halo_periodic(G, vs3 + s * X.ng);
}

// ---- advec.f90:155-229 interface_vels(_allspec), single rank -----------------------
void ora_interface_vels_allspec(const ora_grid* G, const double* vs1, const double* vs2,
                                const double* vs3, double* vs1i, double* vs2i, double* vs3i,
                                int lsp) {
  Ix X(G);
  const int lx1 = G->lx1, lx2 = G->lx2, lx3 = G->lx3;
  for (int s = 0; s < lsp; ++s) {
    const double* v1 = vs1 + s * X.ng;
    const double* v2 = vs2 + s * X.ng;
    const double* v3 = vs3 + s * X.ng;
    double* a = vs1i + s * X.nf1();
    double* b = vs2i + s * X.nf2();
    double* c = vs3i + s * X.nf3();
    for (int i3 = 1; i3 <= lx3; ++i3)
      for (int i2 = 1; i2 <= lx2; ++i2) {
        for (int i1 = 2; i1 <= lx1; ++i1)
          a[X.f1(i1, i2, i3)] = 0.5 * (v1[X.g(i1 - 1, i2, i3)] + v1[X.g(i1, i2, i3)]);
        if (G->gridflag == 0)
          a[X.f1(1, i2, i3)] = v1[X.g(1, i2, i3)];
        else if (G->gridflag == 1)
          a[X.f1(1, i2, i3)] = fmin_f(a[X.f1(2, i2, i3)], 0.0);
        else
          a[X.f1(1, i2, i3)] = v1[X.g(1, i2, i3)];
        if (G->gridflag == 0)
          a[X.f1(lx1 + 1, i2, i3)] = v1[X.g(lx1, i2, i3)];
        else if (G->gridflag == 1)
          a[X.f1(lx1 + 1, i2, i3)] = v1[X.g(lx1, i2, i3)];
        else
          a[X.f1(lx1 + 1, i2, i3)] = fmax_f(a[X.f1(lx1, i2, i3)], 0.0);
      }
    for (int i3 = 1; i3 <= lx3; ++i3)
      for (int i2 = 1; i2 <= lx2 + 1; ++i2)
        for (int i1 = 1; i1 <= lx1; ++i1)
          b[X.f2(i1, i2, i3)] = 0.5 * (v2[X.g(i1, i2 - 1, i3)] + v2[X.g(i1, i2, i3)]);
    for (int i3 = 1; i3 <= lx3 + 1; ++i3)
      for (int i2 = 1; i2 <= lx2; ++i2)
        for (int i1 = 1; i1 <= lx1; ++i1)
          c[X.f3(i1, i2, i3)] = 0.5 * (v3[X.g(i1, i2, i3 - 1)] + v3[X.g(i1, i2, i3)]);
  }
}

// ---- multifluid.f90:179-233 conversions (full ghosted arrays, all species) ---------
void ora_rhoe2T(const ora_grid* G, const double* ns, const double* rhoes, double* Ts) {
  Ix X(G);
  for (int s = 0; s < LSP; ++s)
    for (long long k = 0; k < X.ng; ++k) {
      const long long q = s * X.ng + k;
      const double T = (K.gammas[s] - 1) / kB * rhoes[q] / fmax_f(ns[q], mindensdiv);
      Ts[q] = fmax_f(T, 100.0);
    }
}

void ora_T2rhoe(const ora_grid* G, const double* ns, const double* Ts, double* rhoes) {
  Ix X(G);
  for (int s = 0; s < LSP; ++s)
    for (long long k = 0; k < X.ng; ++k) {
      const long long q = s * X.ng + k;
      rhoes[q] = ns[q] * kB * Ts[q] / (K.gammas[s] - 1);
    }
}

void ora_v12rhov1(const ora_grid* G, const double* ns, const double* vs1, double* rhovs1) {
  Ix X(G);
  for (int s = 0; s < LSP; ++s)
    for (long long k = 0; k < X.ng; ++k) {
      const long long q = s * X.ng + k;
      rhovs1[q] = ns[q] * K.ms[s] * vs1[q];
    }
}

void ora_rhov12v1(const ora_grid* G, double* ns, const double* rhovs1, double* vs1) {
  Ix X(G);
  std::vector<double> chrg(X.ng, 0.0);
  for (int s = 0; s < LSP - 1; ++s)
    for (long long k = 0; k < X.ng; ++k) {
      const long long q = s * X.ng + k;
      vs1[q] = rhovs1[q] / (K.ms[s] * fmax_f(ns[q], mindensdiv));
      chrg[k] = chrg[k] + ns[q] * K.qs[s] * vs1[q];
    }
  const long long e = (LSP - 1) * X.ng;
  for (long long k = 0; k < X.ng; ++k) {
    double acc = 0.0;
    for (int s = 0; s < LSP - 1; ++s) acc = acc + ns[s * X.ng + k];
    ns[e + k] = acc;
  }
  for (long long k = 0; k < X.ng; ++k)
    vs1[e + k] = -1 / fmax_f(ns[e + k], mindensdiv) / K.qs[LSP - 1] * chrg[k];
}

// ---- multifluid.f90:553-688 clean_param --------------------------------------------
// param: ghosted 4-D (lsp species) block of ns (1), vs1 (2) or Ts (3).
void ora_clean_param(const ora_grid* G, int paramflag, double* param) {
  Ix X(G);
  const int lx1 = G->lx1, lx2 = G->lx2, lx3 = G->lx3;
  auto isnull = [&](int i1, int i2, int i3) -> bool {
    return G->nullpts && G->nullpts[X.c(i1, i2, i3)];
  };
  auto set_ghosts = [&](double val) {
    for (int s = 0; s < LSP; ++s) {
      double* p = param + s * X.ng;
      for (int i3 = -1; i3 <= lx3 + 2; ++i3)
        for (int i2 = -1; i2 <= lx2 + 2; ++i2)
          for (int i1 = -1; i1 <= lx1 + 2; ++i1) {
            const bool ghost = i1 < 1 || i1 > lx1 || i2 < 1 || i2 > lx2 || i3 < 1 || i3 > lx3;
            if (ghost) p[X.g(i1, i2, i3)] = val;
          }
    }
  };
  if (paramflag == 1) {
    for (int s = 0; s < LSP - 1; ++s)
      for (long long k = 0; k < X.ng; ++k) param[s * X.ng + k] = fmax_f(param[s * X.ng + k], mindens);
    for (long long k = 0; k < X.ng; ++k) {
      double acc = 0.0;
      for (int s = 0; s < LSP - 1; ++s) acc = acc + param[s * X.ng + k];
      param[(LSP - 1) * X.ng + k] = acc;
    }
    for (int s = 0; s < LSP; ++s)
      for (int i3 = 1; i3 <= lx3; ++i3)
        for (int i2 = 1; i2 <= lx2; ++i2)
          for (int i1 = 1; i1 <= lx1; ++i1)
            if (isnull(i1, i2, i3))
              param[s * X.ng + X.g(i1, i2, i3)] = (s == 0) ? mindensnull * 1e-2 : mindensnull;
    set_ghosts(mindensdiv);
  } else if (paramflag == 2) {
    for (int s = 0; s < LSP; ++s)
      for (int i3 = 1; i3 <= lx3; ++i3)
        for (int i2 = 1; i2 <= lx2; ++i2)
          for (int i1 = 1; i1 <= lx1; ++i1)
            if (isnull(i1, i2, i3)) param[s * X.ng + X.g(i1, i2, i3)] = 0;
    if (G->gridflag == 0) {
      for (int s = 0; s < LSP; ++s) {
        double* p = param + s * X.ng;
        for (int i3 = 1; i3 <= lx3; ++i3)
          for (int i2 = 1; i2 <= lx2; ++i2) {
            int beg = 1;
            while (!isnull(beg, i2, i3) && beg < lx1) beg = beg + 1;
            int end = beg;
            while (isnull(end, i2, i3) && end < lx1) end = end + 1;
            if (beg != lx1) p[X.g(beg, i2, i3)] = p[X.g(beg + 1, i2, i3)];
            if (end != lx1) p[X.g(end, i2, i3)] = p[X.g(end - 1, i2, i3)];
          }
      }
    } else if (G->gridflag == 1) {
      for (int s = 0; s < LSP; ++s) {
        double* p = param + s * X.ng;
        for (int i3 = 1; i3 <= lx3; ++i3)
          for (int i2 = 1; i2 <= lx2; ++i2) {
            int end = 1;
            while (!isnull(end, i2, i3) && end < lx1) end = end + 1;
            if (end != lx1) p[X.g(end, i2, i3)] = p[X.g(end - 1, i2, i3)];
          }
      }
    }
  } else if (paramflag == 3) {
    for (long long k = 0; k < LSP * X.ng; ++k) param[k] = fmax_f(param[k], 100.0);
    for (int s = 0; s < LSP; ++s)
      for (int i3 = 1; i3 <= lx3; ++i3)
        for (int i2 = 1; i2 <= lx2; ++i2)
          for (int i1 = 1; i1 <= lx1; ++i1)
            if (isnull(i1, i2, i3)) param[s * X.ng + X.g(i1, i2, i3)] = 100;
    set_ghosts(100.0);
  }
}

// ---- LAPACK dgbsv restated (dgbtrf -> dgbtf2 for kl < block size, dgbtrs), with the
// reference BLAS semantics for idamax/dswap/dscal/dger/dtbsv.  Column-major band
// storage ab(ldab, n), 1-based in the comments, 0-based in code.  info is returned
// (gbsv.in.f90:93 drops it).
int ora_dgbsv(int n, int kl, int ku, double* ab, int ldab, int* ipiv, double* b) {
#define AB(i, j) ab[((i)-1) + (long long)((j)-1) * ldab]
  int info = 0;
  const int kv = ku + kl;
  // dgbtf2: zero the fill-in elements in columns KU+2..KV.
  for (int j = ku + 2; j <= std::min(kv, n); ++j)
    for (int i = kv - j + 2; i <= kl; ++i) AB(i, j) = 0.0;
  int ju = 1;
  for (int j = 1; j <= n; ++j) {
    if (j + kv <= n)
      for (int i = 1; i <= kl; ++i) AB(i, j + kv) = 0.0;
    const int km = std::min(kl, n - j);
    // idamax over AB(kv+1 .. kv+1+km, j): first index of the largest |.|
    int jp = 1;
    double amax = std::fabs(AB(kv + 1, j));
    for (int i = 2; i <= km + 1; ++i) {
      const double t = std::fabs(AB(kv + i, j));
      if (t > amax) {
        amax = t;
        jp = i;
      }
    }
    ipiv[j - 1] = jp + j - 1;
    if (AB(kv + jp, j) != 0.0) {
      ju = std::max(ju, std::min(j + ku + jp - 1, n));
      if (jp != 1) {
        // dswap(ju-j+1, AB(kv+jp,j), ldab-1, AB(kv+1,j), ldab-1)
        for (int t = 0; t <= ju - j; ++t) {
          double& x = ab[(kv + jp - 1) + (long long)(j - 1) * ldab + (long long)t * (ldab - 1)];
          double& y = ab[(kv) + (long long)(j - 1) * ldab + (long long)t * (ldab - 1)];
          std::swap(x, y);
        }
      }
      if (km > 0) {
        const double r = 1.0 / AB(kv + 1, j);  // dscal(km, one/pivot, ...)
        for (int i = 1; i <= km; ++i) AB(kv + 1 + i, j) = r * AB(kv + 1 + i, j);
        if (ju > j) {
          // dger(km, ju-j, -one, x=AB(kv+2,j), y=AB(kv,j+1) stride ldab-1, A=AB(kv+1,j+1) lda ldab-1)
          for (int c = 1; c <= ju - j; ++c) {
            const double y = ab[(kv - 1) + (long long)j * ldab + (long long)(c - 1) * (ldab - 1)];
            if (y != 0.0) {
              const double temp = -1.0 * y;
              for (int i = 1; i <= km; ++i) {
                double& a = ab[(kv) + (long long)(j)*ldab + (long long)(c - 1) * (ldab - 1) + (i - 1)];
                a = a + AB(kv + 1 + i, j) * temp;
              }
            }
          }
        }
      }
    } else if (info == 0) {
      info = j;
    }
  }
  if (info != 0) return info;
  // dgbtrs, no transpose, nrhs = 1: L solve with the row interchanges ...
  const int kd = ku + kl + 1;
  if (kl > 0) {
    for (int j = 1; j <= n - 1; ++j) {
      const int lm = std::min(kl, n - j);
      const int l = ipiv[j - 1];
      if (l != j) std::swap(b[l - 1], b[j - 1]);
      const double y = b[j - 1];
      if (y != 0.0) {  // dger(lm, 1, -one, AB(kd+1,j), 1, b(j), ldb, b(j+1), ldb)
        const double temp = -1.0 * y;
        for (int i = 1; i <= lm; ++i) b[j + i - 1] = b[j + i - 1] + AB(kd + i, j) * temp;
      }
    }
  }
  // ... then dtbsv('Upper','No transpose','Non-unit', n, kl+ku, ab, ldab, b, 1).
  const int k = kl + ku;
  for (int j = n; j >= 1; --j) {
    if (b[j - 1] != 0.0) {
      const int l = k + 1 - j;
      b[j - 1] = b[j - 1] / AB(k + 1, j);
      const double temp = b[j - 1];
      for (int i = j - 1; i >= std::max(1, j - k); --i) b[i - 1] = b[i - 1] - temp * AB(l + i, j);
    }
  }
  return 0;
#undef AB
}

}  // extern "C"

namespace {

// Diffusion band-solver mode.  0: LAPACK dgbsv restated (the reference's arithmetic,
// default).  1: the same banded system, eliminated without pivoting in x87 extended
// precision (64-bit significand) and rounded once to double -- an accurate solution of the
// reference's discrete equations, used to check solvers whose rounding differs from a
// particular LAPACK build (partial pivoting on the Dirichlet identity rows leaves rounding
// errors of up to ~1e-9 relative in stiff columns, and OpenBLAS and netlib-BLAS builds of
// the reference disagree by that much).
int g_diff_solver = 0;

// T**(5/2) (collisions.f90:187,189).  Mode 0: the C library pow, as the Fortran calls it
// (glibc's pow is not correctly rounded everywhere: ~1 in 1200 arguments in 1e2..4e4 differ
// by 1 ulp from the correctly rounded value).  Mode 1: x^2 * sqrt(x) evaluated in
// double-double with fma and rounded once -- the correctly rounded value except in
// vanishingly rare near-halfway cases; the GPU kernels evaluate the same expression.
int g_pow_mode = 0;

double pow25_dd(double x) {
  if (!(x > 0.0)) return std::pow(x, 2.5);
  const double s = std::sqrt(x);
  const double es = std::fma(-s, s, x);   // x - s*s exactly
  const double sl = es / (2.0 * s);       // sqrt(x) ~ s + sl
  const double x2 = x * x;
  const double x2l = std::fma(x, x, -x2); // x*x = x2 + x2l exactly
  const double p = x2 * s;
  const double pl = std::fma(x2, s, -p);  // x2*s = p + pl exactly
  return p + (pl + (x2 * sl + x2l * s));
}

inline double pow25(double x) { return g_pow_mode == 1 ? pow25_dd(x) : std::pow(x, 2.5); }

// Tridiagonal band matrix in dgbsv storage (ldab 7, kl=ku=2; only the diagonal and the
// first sub/super diagonals are non-zero), solved by Thomas in long double.
void band_solve_extended(int n, const double* M, double* b) {
#define MB(r, j) M[((r)-1) + 7LL * ((j)-1)]
  std::vector<long double> cp(n + 1), dp(n + 1);
  for (int i = 1; i <= n; ++i) {
    const long double a = (i > 1) ? (long double)MB(6, i - 1) : 0.0L;  // A(i,i-1)
    const long double d = (long double)MB(5, i);                        // A(i,i)
    const long double c = (i < n) ? (long double)MB(4, i + 1) : 0.0L;   // A(i,i+1)
    const long double m = (i > 1) ? d - a * cp[i - 1] : d;
    cp[i] = c / m;
    dp[i] = ((long double)b[i - 1] - ((i > 1) ? a * dp[i - 1] : 0.0L)) / m;
  }
  long double x = dp[n];
  b[n - 1] = (double)x;
  for (int i = n - 1; i >= 1; --i) {
    x = dp[i] - cp[i] * x;
    b[i - 1] = (double)x;
  }
#undef MB
}

int band_solve(int n, double* M, int* ipiv, double* b) {
  if (g_diff_solver == 1) {
    band_solve_extended(n, M, b);
    return 0;
  }
  return ora_dgbsv(n, 2, 2, M, 7, ipiv, b);
}

struct Col {
  // 1-based accessors for the 1-D arrays of one column.
  const double *Ts, *A, *B, *C, *D, *E, *dx1, *dx1i;
  double T(int i) const { return Ts[i - 1]; }
  double a(int i) const { return A[i - 1]; }
  double b(int i) const { return B[i - 1]; }
  double c(int i) const { return C[i - 1]; }
  double e(int i) const { return E[i - 1]; }
  double dx(int i) const { return dx1[i]; }
  double dxi(int i) const { return dx1i[i - 1]; }
};

// PDEparabolic.f90:19-218.  Returns the LAPACK info of the second solve (ignored by
// the reference, gbsv.in.f90:93).
int trbdf21d(int lx1, const Col& c, double Tsminx1, double Tsmaxx1, double dt, double* out,
             std::vector<double>& Mv, std::vector<int>& ipiv, std::vector<double>& Dhv,
             std::vector<double>& TRv) {
  const int ll = 2;
  double* M = Mv.data();
#define M_(r, j) M[((r)-1) + 7LL * ((j)-1)]
  auto Dh = [&](int i) -> double& { return Dhv[i - 1]; };
  auto TR = [&](int i) -> double& { return TRv[i - 1]; };
  auto OUT = [&](int i) -> double& { return out[i - 1]; };

  Dh(1) = 0;
  for (int i = 2; i <= lx1; ++i) Dh(i) = 0.5 * (c.D[i - 2] + c.D[i - 1]);

  // ---- TR half step (59-137)
  int ix1 = 1;
  M_(ll + 3, ix1) = 1;
  M_(ll + 2, ix1 + 1) = 0;
  M_(ll + 1, ix1 + 2) = 0;
  TR(ix1) = Tsminx1;

  auto tr_row = [&](int i, bool first, bool last) {
    if (!first) M_(ll + 5, i - 2) = 0;
    M_(ll + 4, i - 1) = -c.c(i) * Dh(i) / c.dxi(i) / c.dx(i) / 2 + c.b(i) / (c.dx(i + 1) + c.dx(i)) / 2;
    M_(ll + 3, i) = 1 / (dt / 2) - c.a(i) / 2 + c.c(i) * Dh(i + 1) / c.dxi(i) / c.dx(i + 1) / 2 +
                    c.c(i) * Dh(i) / c.dxi(i) / c.dx(i) / 2;
    M_(ll + 2, i + 1) =
        -c.c(i) * Dh(i + 1) / c.dxi(i) / c.dx(i + 1) / 2 - c.b(i) / (c.dx(i + 1) + c.dx(i)) / 2;
    if (!last) M_(ll + 1, i + 2) = 0;
    double r = c.T(i) / (dt / 2) + c.e(i);
    if (!first) r = r - M_(ll + 5, i - 2) * c.T(i - 2);
    r = r - M_(ll + 4, i - 1) * c.T(i - 1);
    r = r - (-c.a(i) / 2 + c.c(i) * Dh(i + 1) / c.dxi(i) / c.dx(i + 1) / 2 +
             c.c(i) * Dh(i) / c.dxi(i) / c.dx(i) / 2) *
                c.T(i);
    r = r - M_(ll + 2, i + 1) * c.T(i + 1);
    if (!last) r = r - M_(ll + 1, i + 2) * c.T(i + 2);
    TR(i) = r;
  };
  tr_row(2, true, false);
  for (int i = 3; i <= lx1 - 2; ++i) tr_row(i, false, false);
  tr_row(lx1 - 1, false, true);
  ix1 = lx1;
  M_(ll + 5, ix1 - 2) = 0;
  M_(ll + 4, ix1 - 1) = 0;
  M_(ll + 3, ix1) = 1;
  TR(ix1) = Tsmaxx1;
  band_solve(lx1, M, ipiv.data(), TRv.data());

  // ---- BDF2 step (148-216)
  ix1 = 1;
  M_(ll + 3, ix1) = 1;
  M_(ll + 2, ix1 + 1) = 0;
  M_(ll + 1, ix1 + 2) = 0;
  OUT(ix1) = Tsminx1;
  auto bdf_row = [&](int i, bool first, bool last) {
    if (!first) M_(ll + 5, i - 2) = 0;
    M_(ll + 4, i - 1) = -c.c(i) * Dh(i) / c.dxi(i) / c.dx(i) + c.b(i) / (c.dx(i + 1) + c.dx(i));
    M_(ll + 3, i) = 1 / (dt / 3) - c.a(i) + c.c(i) * Dh(i + 1) / c.dxi(i) / c.dx(i + 1) +
                    c.c(i) * Dh(i) / c.dxi(i) / c.dx(i);
    M_(ll + 2, i + 1) = -c.c(i) * Dh(i + 1) / c.dxi(i) / c.dx(i + 1) - c.b(i) / (c.dx(i + 1) + c.dx(i));
    if (!last) M_(ll + 1, i + 2) = 0;
    OUT(i) = c.e(i) - 1 / 3.0 * c.T(i) / (dt / 3) + 4 / 3.0 * TR(i) / (dt / 3);
  };
  bdf_row(2, true, false);
  for (int i = 3; i <= lx1 - 2; ++i) bdf_row(i, false, false);
  bdf_row(lx1 - 1, false, true);
  ix1 = lx1;
  M_(ll + 5, ix1 - 2) = 0;
  M_(ll + 4, ix1 - 1) = 0;
  M_(ll + 3, ix1) = 1;
  OUT(ix1) = Tsmaxx1;
  return band_solve(lx1, M, ipiv.data(), out);
#undef M_
}

// PDEparabolic.f90:221-346 backEuler1D (without the optional outputs).
int backeuler1d(int lx1, const Col& c, double Tsminx1, double Tsmaxx1, double dt, double* out,
                std::vector<double>& Mv, std::vector<int>& ipiv, std::vector<double>& Dhv) {
  const int ll = 2;
  double* M = Mv.data();
#define M_(r, j) M[((r)-1) + 7LL * ((j)-1)]
  auto Dh = [&](int i) -> double& { return Dhv[i - 1]; };
  auto OUT = [&](int i) -> double& { return out[i - 1]; };
  Dh(1) = 0;
  for (int i = 2; i <= lx1; ++i) Dh(i) = 0.5 * (c.D[i - 2] + c.D[i - 1]);
  for (int i = 1; i <= lx1; ++i) OUT(i) = c.T(i) / dt + c.e(i);
  int ix1 = 1;
  M_(ll + 3, ix1) = 1;
  M_(ll + 2, ix1 + 1) = 0;
  M_(ll + 1, ix1 + 2) = 0;
  OUT(ix1) = Tsminx1;
  auto row = [&](int i, bool first, bool last) {
    if (!first) M_(ll + 5, i - 2) = 0;
    M_(ll + 4, i - 1) = -c.c(i) * Dh(i) / c.dxi(i) / c.dx(i) + c.b(i) / (c.dx(i + 1) + c.dx(i));
    M_(ll + 3, i) = 1 / dt - c.a(i) + c.c(i) * Dh(i + 1) / c.dxi(i) / c.dx(i + 1) +
                    c.c(i) * Dh(i) / c.dxi(i) / c.dx(i);
    M_(ll + 2, i + 1) = -c.c(i) * Dh(i + 1) / c.dxi(i) / c.dx(i + 1) - c.b(i) / (c.dx(i + 1) + c.dx(i));
    if (!last) M_(ll + 1, i + 2) = 0;
  };
  row(2, true, false);
  for (int i = 3; i <= lx1 - 2; ++i) row(i, false, false);
  row(lx1 - 1, false, true);
  ix1 = lx1;
  M_(ll + 5, ix1 - 2) = 0;
  M_(ll + 4, ix1 - 1) = 0;
  M_(ll + 3, ix1) = 1;
  OUT(ix1) = Tsmaxx1;
  return band_solve(lx1, M, ipiv.data(), out);
#undef M_
}

}  // namespace

extern "C" {

// 1-D drivers (test hooks, e.g. test/diffusion/test_diffusion1D.f90).
int ora_TRBDF21D(int lx1, const double* Ts, const double* A, const double* B, const double* C,
                 const double* D, const double* E, double Tsminx1, double Tsmaxx1, double dt,
                 const double* dx1, const double* dx1i, double* out) {
  if (lx1 < 4) return -1;
  Col c{Ts, A, B, C, D, E, dx1, dx1i};
  std::vector<double> M(7 * lx1), Dh(lx1), TR(lx1);
  std::vector<int> ipiv(lx1);
  return trbdf21d(lx1, c, Tsminx1, Tsmaxx1, dt, out, M, ipiv, Dh, TR);
}

int ora_backEuler1D(int lx1, const double* Ts, const double* A, const double* B, const double* C,
                    const double* D, const double* E, double Tsminx1, double Tsmaxx1, double dt,
                    const double* dx1, const double* dx1i, double* out) {
  if (lx1 < 4) return -1;
  Col c{Ts, A, B, C, D, E, dx1, dx1i};
  std::vector<double> M(7 * lx1), Dh(lx1);
  std::vector<int> ipiv(lx1);
  return backeuler1d(lx1, c, Tsminx1, Tsmaxx1, dt, out, M, ipiv, Dh);
}

// ---- multifluid.f90:309-342 energy_diffusion (+ collisions.f90:162-199 thermal_conduct,
// diffusion.f90:24-80 diffusion_prep, diffusion.f90:83-152 backEuler3D/TRBDF23D).
// Ts/ns/J1 ghosted; nn (lx1,lx2,lx3,3) = O, N2, O2; Tn (lx1,lx2,lx3).
// The reference leaves the ghost cells of the returned temperature undefined (the
// function results of TRBDF23D/backEuler3D assign 1:lx1 only); this restatement keeps
// the input ghosts except the x1 layers 0 and lx1+1, which receive the Dirichlet values
// loaded by diffusion_prep, and then applies max(T,100) everywhere (multifluid.f90:340).
int ora_energy_diffusion(const ora_grid* G, const double* ns, double* Ts, const double* J1,
                         const double* nn, const double* Tn, double dt, int flagdiffsolve,
                         double Teinf) {
  if (flagdiffsolve != 1 && flagdiffsolve != 2) return -2;
  if (G->lx1 < 4) return -1;
  Ix X(G);
  const int lx1 = G->lx1, lx2 = G->lx2, lx3 = G->lx3;
  const long long nc = X.nc();
  std::vector<double> lam(nc), beta(nc), Bc(nc), Cc(nc), Dc(nc);
  for (int s = 0; s < LSP; ++s) {
    double* T = Ts + s * X.ng;
    const double* n = ns + s * X.ng;
    // thermal_conduct
#pragma omp parallel for collapse(2) schedule(static)
    for (int i3 = 1; i3 <= lx3; ++i3)
      for (int i2 = 1; i2 <= lx2; ++i2)
        for (int i1 = 1; i1 <= lx1; ++i1) {
          const long long k = X.c(i1, i2, i3), q = X.g(i1, i2, i3);
          const double t = T[q];
          if (s < LSP - 1) {
            lam[k] = K.thermal_coeff[s] * pow25(t);
            beta[k] = 0.0;
          } else {
            const double n1 = nn[k], n2 = nn[nc + k], n3 = nn[2 * nc + k];
            const double X3 = n1 * 1.1e-16 * (1 + 5.7e-4 * t) +
                              n2 * 2.82e-17 * std::sqrt(t) * (1 - 1.21e-4 * t) +
                              n3 * 2.2e-16 * (1 + 3.6e-2 * std::sqrt(t));
            lam[k] = elchrg * 100 * 7.7e5 * pow25(t) / (1 + 3.22e4 * (t * t) / n[q] * X3);
            beta[k] = 5.0 / 2 * kB / elchrg * J1[q];
          }
          // diffusion_prep (A = E = 0)
          const double hp = G->h1[q] * G->h2[q] * G->h3[q];
          Cc[k] = (K.gammas[s] - 1.0) / kB / fmax_f(n[q], mindensdiv) / hp;
          Bc[k] = Cc[k] * beta[k] / G->h1[q];
          Dc[k] = lam[k] * G->h2[q] * G->h3[q] / G->h1[q];
        }
    // boundary conditions into the x1 ghosts (diffusion.f90:54-79)
    for (int i3 = 1; i3 <= lx3; ++i3)
      for (int i2 = 1; i2 <= lx2; ++i2) {
        const double tn1 = Tn[X.c(1, i2, i3)], tnl = Tn[X.c(lx1, i2, i3)];
        if (G->gridflag == 0) {
          T[X.g(0, i2, i3)] = tn1;
          T[X.g(lx1 + 1, i2, i3)] = tnl;
        } else if (G->gridflag == 1) {
          T[X.g(lx1 + 1, i2, i3)] = tnl;
          T[X.g(0, i2, i3)] = Teinf;
        } else {
          T[X.g(0, i2, i3)] = tn1;
          T[X.g(lx1 + 1, i2, i3)] = Teinf;
        }
      }
    // column solves
#pragma omp parallel
    {
      std::vector<double> M(7 * lx1), Dh(lx1), TR(lx1), Tc(lx1), out(lx1), zero(lx1, 0.0);
      std::vector<int> ipiv(lx1);
#pragma omp for collapse(2) schedule(static)
      for (int i3 = 1; i3 <= lx3; ++i3)
        for (int i2 = 1; i2 <= lx2; ++i2) {
          for (int i1 = 1; i1 <= lx1; ++i1) Tc[i1 - 1] = T[X.g(i1, i2, i3)];
          const long long k0 = X.c(1, i2, i3);
          Col c{Tc.data(), zero.data(), &Bc[k0], &Cc[k0], &Dc[k0], zero.data(), G->dx1, G->dx1i};
          const double tmin = T[X.g(0, i2, i3)], tmax = T[X.g(lx1 + 1, i2, i3)];
          if (flagdiffsolve == 2)
            trbdf21d(lx1, c, tmin, tmax, dt, out.data(), M, ipiv, Dh, TR);
          else
            backeuler1d(lx1, c, tmin, tmax, dt, out.data(), M, ipiv, Dh);
          for (int i1 = 1; i1 <= lx1; ++i1) T[X.g(i1, i2, i3)] = out[i1 - 1];
        }
    }
    for (long long k = 0; k < X.ng; ++k) T[k] = fmax_f(T[k], 100.0);
  }
  return 0;
}

// ---- temporal_mpi.f90:86-167 dt_calc, then the dt_comm floor (temporal_mpi.f90:64) --
// dl_k i = dx_k i * h_k (meshobj.f90:421-446).  Returns dt; gridrates (3*lsp) optional.
double ora_dt_calc(const ora_grid* G, double tcfl, const double* Ts, const double* vs1,
                   const double* vs2, const double* vs3, double* gridrates) {
  Ix X(G);
  double gr[3][LSP];
  for (int s = 0; s < LSP; ++s) gr[0][s] = gr[1][s] = gr[2][s] = 0.0;
  for (int s = 0; s < LSP; ++s) {
    double g1 = 0.0, g2 = 0.0, g3 = 0.0;
#pragma omp parallel for collapse(2) reduction(max : g1, g2, g3) schedule(static)
    for (int i3 = 1; i3 <= G->lx3; ++i3)
      for (int i2 = 1; i2 <= G->lx2; ++i2)
        for (int i1 = 1; i1 <= G->lx1; ++i1) {
          const long long q = X.g(i1, i2, i3);
          double vsnd = 0.0;
          if (s < LSP - 1)
            vsnd = std::sqrt(kB * Ts[s * X.ng + q] / K.ms[s] +
                             5.0 / 3.0 * kB * Ts[(LSP - 1) * X.ng + q] / K.ms[s]);
          const double dl1 = G->dx1i[i1 - 1] * G->h1[q];
          const double dl2 = G->dx2i[i2 - 1] * G->h2[q];
          const double dl3 = G->dx3i[i3 - 1] * G->h3[q];
          g1 = fmax_f((vsnd + std::fabs(vs1[s * X.ng + q])) / dl1, g1);
          g2 = fmax_f(std::fabs(vs2[s * X.ng + q]) / dl2, g2);
          g3 = fmax_f(std::fabs(vs3[s * X.ng + q]) / dl3, g3);
        }
    gr[0][s] = g1;
    gr[1][s] = g2;
    gr[2][s] = g3;
  }
  double m = 0.0;
  bool first = true;
  for (int d = 0; d < 3; ++d)
    for (int s = 0; s < LSP; ++s) {
      gr[d][s] = fmax_f(gr[d][s], 1e-10);
      const double inv = 1.0 / gr[d][s];
      if (first || inv < m) m = inv;
      first = false;
      if (gridrates) gridrates[d * LSP + s] = gr[d][s];
    }
  double dt = tcfl * m;
  return fmax_f(dt, 1e-6);
}

// ---- app/main.f90:280-355 fluid_adv, the advection + diffusion subset -------------
// (compression, ionization and source/loss excluded).  fluidvars: (.,35) =
// ns|vs1|vs2|vs3|Ts; fluidauxvars: at least (.,14) = rhovs1|rhoes; J1 ghosted;
// vs1i/vs2i/vs3i carried between steps (libgemini.f90:284-291).
int ora_fluid_adv(const ora_grid* G, double* fluidvars, double* fluidauxvars, const double* J1,
                  double* vs1i, double* vs2i, double* vs3i, const double* nn, const double* Tn,
                  double dt, double Teinf, int diffsolvetype) {
  Ix X(G);
  double* ns = fluidvars;
  double* vs1 = fluidvars + LSP * X.ng;
  double* vs2 = fluidvars + 2 * LSP * X.ng;
  double* vs3 = fluidvars + 3 * LSP * X.ng;
  double* Ts = fluidvars + 4 * LSP * X.ng;
  double* rhovs1 = fluidauxvars;
  double* rhoes = fluidauxvars + LSP * X.ng;
  ora_v12rhov1(G, ns, vs1, rhovs1);
  ora_T2rhoe(G, ns, Ts, rhoes);
  ora_set_global_boundaries_allspec(G, ns, rhovs1, vs1, vs2, vs3, rhoes, vs1i, LSP);
  ora_halo_fluidvars(G, ns, rhovs1, rhoes, vs2, vs3);
  ora_interface_vels_allspec(G, vs1, vs2, vs3, vs1i, vs2i, vs3i, LSP);
  ora_sweep_allspec(G, 3, ns, vs3i, dt, 0, 6);
  ora_sweep_allspec(G, 3, rhovs1, vs3i, dt, 1, 6);
  ora_sweep_allspec(G, 3, rhoes, vs3i, dt, 0, 7);
  ora_sweep_allspec(G, 1, ns, vs1i, dt, 0, 6);
  ora_sweep_allspec(G, 1, rhovs1, vs1i, dt, 0, 6);
  ora_sweep_allspec(G, 1, rhoes, vs1i, dt, 0, 7);
  ora_halo_allparams(G, ns, rhovs1, rhoes);
  ora_sweep_allspec(G, 2, ns, vs2i, dt, 0, 6);
  ora_sweep_allspec(G, 2, rhovs1, vs2i, dt, 1, 6);
  ora_sweep_allspec(G, 2, rhoes, vs2i, dt, 0, 7);
  ora_rhov12v1(G, ns, rhovs1, vs1);
  ora_clean_param(G, 1, ns);
  ora_clean_param(G, 2, vs1);
  ora_rhoe2T(G, ns, rhoes, Ts);
  ora_clean_param(G, 3, Ts);
  const int rc = ora_energy_diffusion(G, ns, Ts, J1, nn, Tn, dt, diffsolvetype, Teinf);
  if (rc != 0) return rc;
  ora_clean_param(G, 3, Ts);
  ora_T2rhoe(G, ns, Ts, rhoes);
  return 0;
}

// ---- the compression sub-step (app/main.f90:320-338) ------------------------------

// multifluid.f90:237-268 VNRicht_artvisc with xicon = 3 (multifluid.f90:43).  Q: interior
// (1:lx1,1:lx2,1:lx3,lsp), column-major.  Reads vs1 at x1 indices 0..lx1+1, ghosts as they
// stand after the advection (the reference notes this at multifluid.f90:255-256).
void ora_vnricht_artvisc(const ora_grid* G, const double* ns, const double* vs1, double* Q) {
  Ix X(G);
  const double xicon = 3.0;
  const double xicon2 = xicon * xicon;  // xicon**2
  const long long nc = X.nc();
  std::vector<double> v1i(G->lx1 + 1);
  for (int s = 0; s < LSP - 1; ++s) {
    const double* n = ns + s * X.ng;
    const double* v = vs1 + s * X.ng;
    for (int i3 = 1; i3 <= G->lx3; ++i3)
      for (int i2 = 1; i2 <= G->lx2; ++i2) {
        // v1iupdate(1:lx1+1) = 0.5*(vs1(0:lx1) + vs1(1:lx1+1))
        for (int i = 1; i <= G->lx1 + 1; ++i) v1i[i - 1] = 0.5 * (v[X.g(i - 1, i2, i3)] + v[X.g(i, i2, i3)]);
        for (int i1 = 1; i1 <= G->lx1; ++i1) {
          const double dv = v1i[i1] - v1i[i1 - 1];  // dv1iupdate
          const double m = fmin_f(dv, 0.0);
          Q[s * nc + X.c(i1, i2, i3)] = n[X.g(i1, i2, i3)] * K.ms[s] * 0.25 * xicon2 * (m * m);
        }
      }
  }
  for (long long q = 0; q < nc; ++q) Q[(LSP - 1) * nc + q] = 0.0;
}

// sources_mpi.f90:68-111 RK2_global_boundary(_allspec) on a single rank (every global
// boundary is local): zero-order hold of vs1 along x1, then of vs1, vs2, vs3 along x2 and,
// unless x3 is periodic, along x3 -- each over the full extent of the other indices.
void ora_rk2_global_boundary_allspec(const ora_grid* G, double* vs1, double* vs2, double* vs3) {
  Ix X(G);
  const int lx1 = G->lx1, lx2 = G->lx2, lx3 = G->lx3;
  for (int s = 0; s < LSP; ++s) {
    double* v[3] = {vs1 + s * X.ng, vs2 + s * X.ng, vs3 + s * X.ng};
    for (int i3 = -1; i3 <= lx3 + 2; ++i3)
      for (int i2 = -1; i2 <= lx2 + 2; ++i2) {
        v[0][X.g(0, i2, i3)] = v[0][X.g(1, i2, i3)];
        v[0][X.g(lx1 + 1, i2, i3)] = v[0][X.g(lx1, i2, i3)];
      }
    for (int c = 0; c < 3; ++c)
      for (int i3 = -1; i3 <= lx3 + 2; ++i3)
        for (int i1 = -1; i1 <= lx1 + 2; ++i1) v[c][X.g(i1, 0, i3)] = v[c][X.g(i1, 1, i3)];
    for (int c = 0; c < 3; ++c)
      for (int i3 = -1; i3 <= lx3 + 2; ++i3)
        for (int i1 = -1; i1 <= lx1 + 2; ++i1) v[c][X.g(i1, lx2 + 1, i3)] = v[c][X.g(i1, lx2, i3)];
    if (!G->flagper) {
      for (int c = 0; c < 3; ++c)
        for (int i2 = -1; i2 <= lx2 + 2; ++i2)
          for (int i1 = -1; i1 <= lx1 + 2; ++i1) v[c][X.g(i1, i2, 0)] = v[c][X.g(i1, i2, 1)];
      for (int c = 0; c < 3; ++c)
        for (int i2 = -1; i2 <= lx2 + 2; ++i2)
          for (int i1 = -1; i1 <= lx1 + 2; ++i1) v[c][X.g(i1, i2, lx3 + 1)] = v[c][X.g(i1, i2, lx3)];
    }
  }
}

// calculus/div.f90:110-200 div3D_curv_23 as compression calls it (multifluid.f90:289-291):
// the slab of grid indices 0..lx+1 in each direction.  f1, f2, f3: one species, ghosted;
// div: (lx1+2, lx2+2, lx3+2), column-major, slab index j <-> grid index j-1.  One-sided
// differences on the slab's faces, centred ones inside; dx arrays are backward differences.
void ora_div3D(const ora_grid* G, const double* f1, const double* f2, const double* f3, double* div) {
  Ix X(G);
  const int L1 = G->lx1 + 2, L2 = G->lx2 + 2, L3 = G->lx3 + 2;
  auto D = [&](int j1, int j2, int j3) -> double& {
    return div[(j1 - 1) + (long long)L1 * ((j2 - 1) + (long long)L2 * (j3 - 1))];
  };
  auto at = [&](const double* a, int j1, int j2, int j3) { return a[X.g(j1 - 1, j2 - 1, j3 - 1)]; };
  auto dx1 = [&](int j) { return G->dx1[j - 1]; };  // x%dx1(0:lx1+1) re-based at 1
  auto dx2 = [&](int j) { return G->dx2[j - 1]; };
  auto dx3 = [&](int j) { return G->dx3[j - 1]; };
  const double *h1 = G->h1, *h2 = G->h2, *h3 = G->h3;
  for (int j3 = 1; j3 <= L3; ++j3)
    for (int j2 = 1; j2 <= L2; ++j2) {
      auto t = [&](int j) { return at(h2, j, j2, j3) * at(h3, j, j2, j3) * at(f1, j, j2, j3); };
      D(1, j2, j3) = (t(2) - t(1)) / dx1(2);
      for (int j = 2; j <= L1 - 1; ++j) D(j, j2, j3) = (t(j + 1) - t(j - 1)) / (dx1(j + 1) + dx1(j));
      D(L1, j2, j3) = (t(L1) - t(L1 - 1)) / dx1(L1);
    }
  if (G->lx2 > 1)
    for (int j3 = 1; j3 <= L3; ++j3)
      for (int j1 = 1; j1 <= L1; ++j1) {
        auto t = [&](int j) { return at(h1, j1, j, j3) * at(h3, j1, j, j3) * at(f2, j1, j, j3); };
        D(j1, 1, j3) = D(j1, 1, j3) + (t(2) - t(1)) / dx2(2);
        for (int j = 2; j <= L2 - 1; ++j) D(j1, j, j3) = D(j1, j, j3) + (t(j + 1) - t(j - 1)) / (dx2(j + 1) + dx2(j));
        D(j1, L2, j3) = D(j1, L2, j3) + (t(L2) - t(L2 - 1)) / dx2(L2);
      }
  if (G->lx3 > 1)
    for (int j2 = 1; j2 <= L2; ++j2)
      for (int j1 = 1; j1 <= L1; ++j1) {
        auto t = [&](int j) { return at(h1, j1, j2, j) * at(h2, j1, j2, j) * at(f3, j1, j2, j); };
        D(j1, j2, 1) = D(j1, j2, 1) + (t(2) - t(1)) / dx3(2);
        for (int j = 2; j <= L3 - 1; ++j) D(j1, j2, j) = D(j1, j2, j) + (t(j + 1) - t(j - 1)) / (dx3(j + 1) + dx3(j));
        D(j1, j2, L3) = D(j1, j2, L3) + (t(L3) - t(L3 - 1)) / dx3(L3);
      }
  for (int j3 = 1; j3 <= L3; ++j3)
    for (int j2 = 1; j2 <= L2; ++j2)
      for (int j1 = 1; j1 <= L1; ++j1)
        D(j1, j2, j3) = D(j1, j2, j3) / (at(h1, j1, j2, j3) * at(h2, j1, j2, j3) * at(h3, j1, j2, j3));
}

// multifluid.f90:274-302 compression: the half-step and full-step energy updates with
// the slab divergence of each species' velocity.  Q: interior (lsp species); rhoes ghosted.
void ora_compression(const ora_grid* G, double dt, const double* vs1, const double* vs2, const double* vs3,
                     const double* Q, double* rhoes) {
  Ix X(G);
  const long long nc = X.nc();
  const int L1 = G->lx1 + 2, L2 = G->lx2 + 2;
  std::vector<double> div((size_t)(G->lx1 + 2) * (G->lx2 + 2) * (G->lx3 + 2));
  for (int s = 0; s < LSP; ++s) {
    ora_div3D(G, vs1 + s * X.ng, vs2 + s * X.ng, vs3 + s * X.ng, div.data());
    double* re = rhoes + s * X.ng;
    for (int i3 = 1; i3 <= G->lx3; ++i3)
      for (int i2 = 1; i2 <= G->lx2; ++i2)
        for (int i1 = 1; i1 <= G->lx1; ++i1) {
          const double dv = div[i1 + (long long)L1 * (i2 + (long long)L2 * i3)];  // slab (i+1)
          const double q = Q[s * nc + X.c(i1, i2, i3)];
          const double p = re[X.g(i1, i2, i3)];
          const double half = p - dt / 2 * (p * (K.gammas[s] - 1) + q) * dv;
          re[X.g(i1, i2, i3)] = p - dt * (half * (K.gammas[s] - 1) + q) * dv;
        }
  }
}

// app/main.f90:280-355 with the compression sub-step (main.f90:320-338) between the
// post-advection clean_param(2) and rhoe2T; otherwise ora_fluid_adv.
static int fluid_adv_compression_q(const ora_grid* G, double* fluidvars, double* fluidauxvars, const double* J1,
                                   double* vs1i, double* vs2i, double* vs3i, const double* nn, const double* Tn,
                                   double dt, double Teinf, int diffsolvetype, std::vector<double>& Q) {
  Ix X(G);
  double* ns = fluidvars;
  double* vs1 = fluidvars + LSP * X.ng;
  double* vs2 = fluidvars + 2 * LSP * X.ng;
  double* vs3 = fluidvars + 3 * LSP * X.ng;
  double* Ts = fluidvars + 4 * LSP * X.ng;
  double* rhovs1 = fluidauxvars;
  double* rhoes = fluidauxvars + LSP * X.ng;
  ora_v12rhov1(G, ns, vs1, rhovs1);
  ora_T2rhoe(G, ns, Ts, rhoes);
  ora_set_global_boundaries_allspec(G, ns, rhovs1, vs1, vs2, vs3, rhoes, vs1i, LSP);
  ora_halo_fluidvars(G, ns, rhovs1, rhoes, vs2, vs3);
  ora_interface_vels_allspec(G, vs1, vs2, vs3, vs1i, vs2i, vs3i, LSP);
  ora_sweep_allspec(G, 3, ns, vs3i, dt, 0, 6);
  ora_sweep_allspec(G, 3, rhovs1, vs3i, dt, 1, 6);
  ora_sweep_allspec(G, 3, rhoes, vs3i, dt, 0, 7);
  ora_sweep_allspec(G, 1, ns, vs1i, dt, 0, 6);
  ora_sweep_allspec(G, 1, rhovs1, vs1i, dt, 0, 6);
  ora_sweep_allspec(G, 1, rhoes, vs1i, dt, 0, 7);
  ora_halo_allparams(G, ns, rhovs1, rhoes);
  ora_sweep_allspec(G, 2, ns, vs2i, dt, 0, 6);
  ora_sweep_allspec(G, 2, rhovs1, vs2i, dt, 1, 6);
  ora_sweep_allspec(G, 2, rhoes, vs2i, dt, 0, 7);
  ora_rhov12v1(G, ns, rhovs1, vs1);
  ora_clean_param(G, 1, ns);
  ora_clean_param(G, 2, vs1);
  Q.assign((size_t)LSP * X.nc(), 0.0);
  ora_vnricht_artvisc(G, ns, vs1, Q.data());
  ora_halo_fluidvars(G, ns, rhovs1, rhoes, vs2, vs3);
  ora_rk2_global_boundary_allspec(G, vs1, vs2, vs3);
  ora_compression(G, dt, vs1, vs2, vs3, Q.data(), rhoes);
  ora_rhoe2T(G, ns, rhoes, Ts);
  ora_clean_param(G, 3, Ts);
  const int rc = ora_energy_diffusion(G, ns, Ts, J1, nn, Tn, dt, diffsolvetype, Teinf);
  if (rc != 0) return rc;
  ora_clean_param(G, 3, Ts);
  ora_T2rhoe(G, ns, Ts, rhoes);
  return 0;
}

// ---- the source/loss sub-step's solves, with given production/loss rates ----------
// (the rates themselves come from sources.f90, not restated here)

// sources.f90:18-276 srcsContinuity: production and loss rates of the continuity
// equations.  nn: interior (lx1,lx2,lx3,>=6) neutral densities (O, N2, O2, H, N, NO); vn1..3,
// Tn: interior; ns, vs1, vs2, vs3, Ts: ghosted; Pr, Lo: interior (lx1,lx2,lx3,lsp), zeroed
// first.  Integer powers as gfortran expands them (x**2 = x*x, x**3 = (x*x)*x, x**4 =
// (x*x)*(x*x)), real powers through pow; each rate expression in the reference's order.
void ora_srcs_continuity(const ora_grid* G, const double* nn, const double* vn1, const double* vn2,
                         const double* vn3, const double* Tn, const double* ns, const double* vs1,
                         const double* vs2, const double* vs3, const double* Ts, double* Pr, double* Lo) {
  Ix X(G);
  const long long nc = X.nc();
  auto p2 = [](double x) { return x * x; };
  auto p3 = [](double x) { return x * x * x; };
  auto p4 = [](double x) { const double t = x * x; return t * t; };
  for (long long q = 0; q < LSP * nc; ++q) Pr[q] = Lo[q] = 0.0;
  double kreac = 0.0;  // where-masked: keeps its last value where no branch applies
  for (int i3 = 1; i3 <= G->lx3; ++i3)
    for (int i2 = 1; i2 <= G->lx2; ++i2)
      for (int i1 = 1; i1 <= G->lx1; ++i1) {
        const long long c = X.c(i1, i2, i3), k = X.g(i1, i2, i3);
        auto N = [&](int j) { return nn[(j - 1) * nc + c]; };           // nn(:,:,:,j)
        auto NS = [&](int sp) { return ns[(sp - 1) * X.ng + k]; };      // ns(1:lx1,..,sp)
        auto TS = [&](int sp) { return Ts[(sp - 1) * X.ng + k]; };
        auto PR = [&](int sp) -> double& { return Pr[(sp - 1) * nc + c]; };
        auto LO = [&](int sp) -> double& { return Lo[(sp - 1) * nc + c]; };
        const double tn = Tn[c];
        const double Te = TS(LSP);
        const double dv2 = p2(vs1[k] - vn1[c]) + p2(vs2[k] - vn2[c]) + p2(vs3[k] - vn3[c]);  // species 1
        double Teff, betanow;
        // O+ + N2 --> NO+ + N
        Teff = 28 / (16 + 28.0) * (16 * amu / 3 / kB * (dv2) + TS(1) - tn) + tn;
        if (Teff <= 3725)
          kreac = 1.71676e-12 - 7.19934e-13 * (Teff / 300) + 1.33276e-13 * p2(Teff / 300) -
                  9.28213e-15 * p3(Teff / 300) + 6.39557e-16 * p4(Teff / 300);
        if (Teff > 3725 && Teff <= 30000)
          kreac = -1.52489e-11 + 7.67112e-13 * (Teff / 300) + 1.19064e-13 * p2(Teff / 300) -
                  1.30858e-15 * p3(Teff / 300) + 4.67756e-18 * p4(Teff / 300);
        if (Teff > 30000)
          kreac = -1.52489e-11 + 7.67112e-13 * (100) + 1.19064e-13 * (10000) - 1.30858e-15 * (1000000) +
                  4.67756e-18 * (100000000);
        betanow = kreac * N(2) * 1e-6;
        PR(2) = PR(2) + betanow * NS(1);
        LO(1) = LO(1) + betanow;
        // O+ + O2 --> O2+ + O
        Teff = 32 / (16 + 32.0) * (16 * amu / 3 / kB * (dv2) + TS(1) - tn) + tn;
        if (Teff <= 4800)
          kreac = 2.78932e-11 - 6.92612e-12 * (Teff / 300) + 8.67684e-13 * p2(Teff / 300) -
                  3.47251e-14 * p3(Teff / 300) + 5.07097e-16 * p4(Teff / 300);
        if (Teff > 4800 && Teff <= 30000)
          kreac = -1.74046e-11 + 3.02328e-12 * Teff / 300 - 2.39214e-15 * p2(Teff / 300) -
                  4.02394e-17 * p3(Teff / 300);
        if (Teff > 30000) kreac = -1.74046e-11 + 3.02328e-12 * 100 - 2.39214e-15 * 10000 - 4.02394e-17 * 1000000;
        betanow = kreac * N(3) * 1e-6;
        PR(4) = PR(4) + betanow * NS(1);
        LO(1) = LO(1) + betanow;
        // O+ + NO --> NO+ + O
        Teff = 30 / (16 + 30.0) * (16 * amu / 3 / kB * (dv2) + TS(1) - tn) + tn;
        if (Teff <= 3800)
          kreac = 6.40408e-13 - 1.33888e-13 * (Teff / 300) + 7.65103e-14 * p2(Teff / 300) -
                  3.11509e-15 * p3(Teff / 300) + 6.62374e-17 * p4(Teff / 300);
        if (Teff > 3800 && Teff <= 30000)
          kreac = -7.48312e-13 + 2.31502e-13 * (Teff / 300) + 3.07160e-14 * p2(Teff / 300) -
                  2.65436e-16 * p3(Teff / 300) + 7.76665e-19 * p4(Teff / 300);
        if (Teff > 30000)
          kreac = -7.48312e-13 + 2.31502e-13 * (100) + 3.07160e-14 * (10000) - 2.65436e-16 * (1000000) +
                  7.76665e-19 * (100000000);
        betanow = kreac * N(6) * 1e-6;
        PR(2) = PR(2) + betanow * NS(1);
        LO(1) = LO(1) + betanow;
        // O+ + e --> O + hv
        betanow = 3.7e-12 * std::pow(250 / TS(LSP), 0.7) * NS(LSP) * 1e-6;
        LO(1) = LO(1) + betanow;
        // N2+ + O --> O+ + N2
        Teff = 16 / (28 + 16.0) * (28 * amu / 3 / kB * (dv2) + TS(3) - tn) + tn;
        kreac = (Teff <= 1500) ? 1e-11 * std::pow(300 / Teff, 0.23) : 3.6e-12 * std::pow(300 / Teff, -0.41);
        betanow = kreac * N(1) * 1e-6;
        PR(1) = PR(1) + betanow * NS(3);
        LO(3) = LO(3) + betanow;
        // N+ + O --> O+ + N
        betanow = 5e-13 * N(1) * 1e-6;
        PR(1) = PR(1) + betanow * NS(5);
        LO(5) = LO(5) + betanow;
        // H+ + O --> O+ + H
        Teff = TS(6);
        betanow = (6.e-10) * (8 / 9.0) * (std::pow((Teff + tn / 4) / (tn + Teff / 16), 0.5)) * N(1) * 1e-6;
        PR(1) = PR(1) + betanow * NS(6);
        LO(6) = LO(6) + betanow;
        // O+ + H --> H+ + O
        betanow = 6.0e-10 * N(4) * 1e-6;
        PR(6) = PR(6) + betanow * NS(1);
        LO(1) = LO(1) + betanow;
        // O2+ + N2 --> NO+ + NO
        betanow = 5e-16 * N(3) * 1e-6;
        PR(2) = PR(2) + betanow * NS(4);
        LO(4) = LO(4) + betanow;
        // O2+ + N --> NO+ + O
        betanow = 1.2e-10 * N(5) * 1e-6;
        PR(2) = PR(2) + betanow * NS(4);
        LO(4) = LO(4) + betanow;
        // O2+ + NO --> NO+ + O2
        betanow = 4.6e-10 * N(6) * 1e-6;
        PR(2) = PR(2) + betanow * NS(4);
        LO(4) = LO(4) + betanow;
        // N2+ + O --> NO+ + N
        Teff = 16 / (28 + 16.0) * (28 * amu / 3 / kB * (dv2) + TS(3) - tn) + tn;
        kreac = (Teff <= 1500) ? 1.4e-10 * std::pow(300 / Teff, 0.44) : 5.2e-11 * std::pow(300 / Teff, -0.2);
        betanow = kreac * N(1) * 1e-6;
        PR(2) = PR(2) + betanow * NS(3);
        LO(3) = LO(3) + betanow;
        // N2+ + NO --> NO+ + N2
        betanow = 4.1e-10 * N(6) * 1e-6;
        PR(2) = PR(2) + betanow * NS(3);
        LO(3) = LO(3) + betanow;
        // N+ + O2 --> NO+ + O
        betanow = 2.6e-10 * N(3) * 1e-6;
        PR(2) = PR(2) + betanow * NS(5);
        LO(5) = LO(5) + betanow;
        // NO+ + e --> N + O
        betanow = 4.2e-7 * std::pow(300 / TS(LSP), 0.85) * NS(LSP) * 1e-6;
        LO(2) = LO(2) + betanow;
        // N2+ + O2 --> O2+ + N2
        Teff = 32 / (28 + 32.0) * (28 * amu / 3 / kB * (dv2) + TS(3) - tn) + tn;
        betanow = 5e-11 * (300 / Teff) * N(3) * 1e-6;
        PR(4) = PR(4) + betanow * NS(3);
        LO(3) = LO(3) + betanow;
        // N2+ + e --> N + N
        betanow = 1.8e-7 * std::pow(300 / TS(LSP), 0.39) * NS(LSP) * 1e-6;
        LO(3) = LO(3) + betanow;
        // N+ + O2 --> O2+ + N
        betanow = 3.1e-10 * N(3) * 1e-6;
        PR(4) = PR(4) + betanow * NS(5);
        LO(5) = LO(5) + betanow;
        // O2+ + e- --> O + O
        kreac = (Te <= 1200) ? 1.95e-7 * std::pow(300 / Te, 0.70) : 7.38e-8 * std::pow(1200 / Te, 0.56);
        betanow = kreac * NS(LSP) * 1e-6;
        LO(4) = LO(4) + betanow;
        // N+ + H --> H+ + N
        betanow = 3.6e-12 * N(4) * 1e-6;
        PR(6) = PR(6) + betanow * NS(5);
        LO(5) = LO(5) + betanow;
        // H+ + e --> H + hv
        betanow = 3.7e-12 * std::pow(250 / TS(LSP), 0.7) * NS(LSP) * 1e-6;
        LO(6) = LO(6) + betanow;
      }
}

// ---- collisions.f90:12-55 collision coefficient tables (lsp x ln and lsp x lsp, filled
// row by row by reshape(..., order=[2,1])); default-REAL literals widened to real(wp) --------
constexpr int LN = 4;  // phys_consts.in.f90:39 (O, N2, O2, H)
struct CollTables {
  double Csn[LSP][LN], C2sn1[LSP][LN], C2sn2[LSP][LN], Csj[LSP][LSP], mn[LN];
  CollTables() {
    const float csn[LSP][LN] = {{-1, 6.82e-10f, 6.64e-10f, -1},       {2.44e-10f, 4.34e-10f, 4.27e-10f, 0.69e-10f},
                                {2.58e-10f, -1, 4.49e-10f, 0.74e-10f}, {2.31e-10f, 4.13e-10f, -1, 0.65e-10f},
                                {4.42e-10f, 7.47e-10f, 7.25e-10f, 1.45e-10f}, {-1, 33.6e-10f, 32.0e-10f, -1},
                                {-1, -1, -1, -1}};
    const float c1[LSP][LN] = {{3.67e-11f, 0, 0, 4.63e-12f}, {0, 0, 0, 0}, {0, 5.14e-11f, 0, 0},
                               {0, 0, 2.59e-11f, 0},         {0, 0, 0, 0}, {6.61e-11f, 0, 0, 2.65e-10f},
                               {-1, -1, -1, -1}};
    const float c2[LSP][LN] = {{0.064f, 0, 0, -1}, {0, 0, 0, 0},         {0, 0.069f, 0, 0},   {0, 0, 0.073f, 0},
                               {0, 0, 0, 0},       {0.047f, 0, 0, 0.083f}, {-1, -1, -1, -1}};
    const float csj[LSP][LSP] = {{0.22f, 0.26f, 0.25f, 0.26f, 0.22f, 0.077f, 1.87e-3f},
                                 {0.14f, 0.16f, 0.16f, 0.17f, 0.13f, 0.042f, 9.97e-4f},
                                 {0.15f, 0.17f, 0.17f, 0.18f, 0.14f, 0.045f, 1.07e-3f},
                                 {0.13f, 0.16f, 0.15f, 0.16f, 0.12f, 0.039f, 9.347e-4f},
                                 {0.25f, 0.28f, 0.28f, 0.28f, 0.24f, 0.088f, 2.136e-3f},
                                 {1.23f, 1.25f, 1.25f, 1.25f, 1.23f, 0.90f, 29.7e-3f},
                                 {54.5f, 54.5f, 54.5f, 54.5f, 54.5f, 54.5f, 38.537f}};
    for (int i = 0; i < LSP; ++i) {
      for (int j = 0; j < LN; ++j) {
        Csn[i][j] = (double)csn[i][j];
        C2sn1[i][j] = (double)c1[i][j];
        C2sn2[i][j] = (double)c2[i][j];
      }
      for (int j = 0; j < LSP; ++j) Csj[i][j] = (double)csj[i][j];
    }
    const double m[LN] = {16, 28, 32, 1};  // phys_consts.in.f90:41
    for (int j = 0; j < LN; ++j) mn[j] = m[j] * amu;
  }
};
const CollTables KC;
const double pi_c = 4 * std::atan(1.0);  // phys_consts.in.f90:20

// collisions.f90:58-114 maxwell_colln for one cell: isp (0-based species), isp2 (0-based
// neutral); nn2 = nn(.,isp2), Tn and Ts(isp) of the cell.
inline double maxwell_colln(int isp, int isp2, double nn2, double tn, double ts) {
  if (isp < LSP - 1) {
    if (KC.Csn[isp][isp2] < 0) {  // resonant
      if (isp == 0 && isp2 == 3) {
        const double Teff = tn + ts / 16;
        return KC.C2sn1[isp][isp2] * std::pow(Teff, 0.5) * nn2 * 1e-6;
      }
      const double Teff = 0.5 * (tn + ts);
      const double a = 1 - KC.C2sn2[isp][isp2] * std::log10(Teff);
      return KC.C2sn1[isp][isp2] * (a * a) * (std::pow(Teff, 0.5)) * nn2 * 1e-6;
    }
    return KC.Csn[isp][isp2] * nn2 * 1e-6;  // nonresonant
  }
  const double Teff = ts;  // electron-neutral
  switch (isp2) {
    case 0: return 8.9e-11 * (1.0 + 5.7e-4 * Teff) * (std::pow(Teff, 0.5)) * nn2 * 1e-6;
    case 1: return 2.33e-11 * (1.0 - 1.21e-4 * Teff) * (Teff)*nn2 * 1e-6;
    case 2: return 1.82e-10 * (1.0 + 3.6e-2 * (std::pow(Teff, 0.5))) * (std::pow(Teff, 0.5)) * nn2 * 1e-6;
    default: return 4.5e-9 * (1.0 - 1.35e-4 * Teff) * (std::pow(Teff, 0.5)) * nn2 * 1e-6;
  }
}

// collisions.f90:117-159 coulomb_colln for one cell: nusj, Phisj, Psisj (zero for isp == isp2).
inline void coulomb_colln(int isp, int isp2, double ns2, double ts1, double ts2, double v1, double v2, double& nu,
                          double& Phi, double& Psi) {
  if (isp == isp2) {
    nu = Phi = Psi = 0.0;
    return;
  }
  const double ms1 = K.ms[isp], ms2 = K.ms[isp2];
  const double Teff = (ms2 * ts1 + ms1 * ts2) / (ms2 + ms1);
  nu = KC.Csj[isp][isp2] * ns2 * 1e-6 / std::pow(Teff, 1.5);
  const double mred = ms1 * ms2 / (ms1 + ms2);
  const double W = std::fabs(v1 - v2) / std::sqrt(2 * kB * Teff / mred);
  Psi = std::exp(-(W * W));
  if (W < 0.1)
    Phi = 1;
  else
    Phi = 3.0 / 4 * std::sqrt(pi_c) * std::erf(W) / (W * W * W) - 3.0 / 2 / (W * W) * Psi;
}

// sources.f90:396-485 srcsEnergy: production and loss rates of the energy equations.
// nn: interior (lx1,lx2,lx3,>=4) neutral densities O, N2, O2, H; the rest as
// ora_srcs_continuity.  Pr, Lo zeroed first.
void ora_srcs_energy(const ora_grid* G, const double* nn, const double* vn1, const double* vn2, const double* vn3,
                     const double* Tn, const double* ns, const double* vs1, const double* vs2, const double* vs3,
                     const double* Ts, double* Pr, double* Lo) {
  Ix X(G);
  const long long nc = X.nc();
  for (long long q = 0; q < LSP * nc; ++q) Pr[q] = Lo[q] = 0.0;
  const double sfact = elchrg / kB * (K.gammas[LSP - 1] - 1);
  for (int i3 = 1; i3 <= G->lx3; ++i3)
    for (int i2 = 1; i2 <= G->lx2; ++i2)
      for (int i1 = 1; i1 <= G->lx1; ++i1) {
        const long long c = X.c(i1, i2, i3), k = X.g(i1, i2, i3);
        const double tn = Tn[c];
        auto NS = [&](int s) { return ns[s * X.ng + k]; };
        auto TS = [&](int s) { return Ts[s * X.ng + k]; };
        auto V1 = [&](int s) { return vs1[s * X.ng + k]; };
        auto V2 = [&](int s) { return vs2[s * X.ng + k]; };
        auto V3 = [&](int s) { return vs3[s * X.ng + k]; };
        for (int isp = 0; isp < LSP; ++isp) {
          double& pr = Pr[isp * nc + c];
          double& lo = Lo[isp * nc + c];
          const double ms = K.ms[isp], gm1 = K.gammas[isp] - 1;
          for (int isp2 = 0; isp2 < LN; ++isp2) {  // ion-neutral
            const double nu = maxwell_colln(isp, isp2, nn[isp2 * nc + c], tn, TS(isp));
            double fact = 2 * nu / (ms + KC.mn[isp2]);
            pr = pr + NS(isp) * ms * kB / gm1 * fact * tn;
            lo = lo + ms * fact;
            fact = fact * KC.mn[isp2] / 3;
            const double d1 = V1(isp) - vn1[c], d2 = V2(isp) - vn2[c], d3 = V3(isp) - vn3[c];
            pr = pr + NS(isp) * ms / gm1 * ((d1 * d1) + (d2 * d2) + (d3 * d3)) * fact;
          }
          for (int isp2 = 0; isp2 < LSP; ++isp2) {  // ion-ion
            double nu, Phi, Psi;
            coulomb_colln(isp, isp2, NS(isp2), TS(isp), TS(isp2), V1(isp), V1(isp2), nu, Phi, Psi);
            double fact = 2 * nu * Psi / (ms + K.ms[isp2]);
            pr = pr + NS(isp) * ms * kB / gm1 * fact * TS(isp2);
            lo = lo + ms * fact;
            fact = 2 * nu * Phi / (ms + K.ms[isp2]) * K.ms[isp2] / 3;
            const double d1 = V1(isp) - V1(isp2), d2 = V2(isp) - V2(isp2), d3 = V3(isp) - V3(isp2);
            pr = pr + NS(isp) * ms / gm1 * ((d1 * d1) + (d2 * d2) + (d3 * d3)) * fact;
          }
        }
        // inelastic electron collisions: rotational, then vibrational excitation
        const double Te = TS(LSP - 1);
        double nu = sfact * 6.9e-14 * nn[2 * nc + c] * 1e-6 / std::sqrt(Te);  // O2 rotational
        double iePT = nu * tn;
        double ieLT = nu;
        nu = sfact * 2.9e-14 * nn[1 * nc + c] * 1e-6 / std::sqrt(Te);  // N2 rotational
        iePT = iePT + nu * tn;
        ieLT = ieLT + nu;
        double f = 1.06e4 + 7.51e3 * std::tanh(1.10e-3 * (Te - 1800));
        const double g = 3300 + 1.233 * (Te - 1000) - 2.056e-4 * (Te - 1000) * (Te - 4000);
        double fact = sfact * 2.99e-12 * nn[1 * nc + c] * 1e-6 * std::exp(f * (Te - 2000) / Te / 2000) *
                      (std::exp(-g * (Te - tn) / Te / tn) - 1);  // N2 vibrational
        iePT = iePT - fmax_f(fact, 0.0);
        f = 3300 - 839 * std::sin(1.91e-4 * (Te - 2700));
        fact = sfact * 5.196e-13 * nn[2 * nc + c] * 1e-6 * std::exp(f * (Te - 700) / Te / 700) *
               (std::exp(-2770 * (Te - tn) / Te / tn) - 1);  // O2 vibrational
        iePT = iePT - fmax_f(fact, 0.0);
        Pr[(LSP - 1) * nc + c] = Pr[(LSP - 1) * nc + c] + iePT * NS(LSP - 1) * kB / (K.gammas[LSP - 1] - 1);
        Lo[(LSP - 1) * nc + c] = Lo[(LSP - 1) * nc + c] + ieLT;
      }
}

// calculus/gradient.f90:79-150 grad3D1_curv_23 along one x1 line of n points with grid x1
// indices i0 .. i0+n-1: f[j], h1 at those cells, dx1 = x%dx1(i0:i0+n-1) (dx1[j] is grid
// index i0+j).  The first point divides by dx1(i0), as the reference does.
inline void grad1_line(int n, const double* f, const double* h1, const double* dx1, double* out) {
  out[0] = (f[1] - f[0]) / dx1[0] / h1[0];
  for (int j = 1; j < n - 1; ++j) out[j] = (f[j + 1] - f[j - 1]) / (dx1[j + 1] + dx1[j]) / h1[j];
  out[n - 1] = (f[n - 1] - f[n - 2]) / dx1[n - 1] / h1[n - 1];
}

// sources.f90:279-393 srcsMomentum_curv on a single rank (both x1 ends global: the x1
// gradients over 1..lx1).  nn: interior (lx1,lx2,lx3,>=4); vn1, Tn, Q (lx1,lx2,lx3,lsp), alt,
// g1: interior; ns, vs1, vs2, vs3, Ts, E1: ghosted.  Pr, Lo zeroed first.
void ora_srcs_momentum(const ora_grid* G, const double* nn, const double* vn1, const double* Tn, const double* ns,
                       const double* vs1, const double* vs2, const double* vs3, const double* Ts, const double* E1,
                       const double* Q, const double* alt, const double* g1, double* Pr, double* Lo) {
  Ix X(G);
  const long long nc = X.nc();
  const int n = G->lx1;
  for (long long q = 0; q < LSP * nc; ++q) Pr[q] = Lo[q] = 0.0;
  std::vector<double> hl(n + 2), dl(n + 2), fl(n + 2), gl(n + 2), h1l(n), dxl(n), dh2(n), dh3(n), epol(n), pg(n),
      gq(n), pr_(n);
  for (int i3 = 1; i3 <= G->lx3; ++i3)
    for (int i2 = 1; i2 <= G->lx2; ++i2) {
      // dh2/dx1, dh3/dx1: grad3D1 over x1 indices 0..lx1+1, kept at 1..lx1
      for (int j = 0; j < n + 2; ++j) dl[j] = G->dx1[j];  // x%dx1(0:lx1+1)
      for (int j = 0; j < n + 2; ++j) hl[j] = G->h1[X.g(j, i2, i3)];
      for (int j = 0; j < n + 2; ++j) fl[j] = G->h2[X.g(j, i2, i3)];
      grad1_line(n + 2, fl.data(), hl.data(), dl.data(), gl.data());
      for (int j = 0; j < n; ++j) dh2[j] = gl[j + 1];
      for (int j = 0; j < n + 2; ++j) fl[j] = G->h3[X.g(j, i2, i3)];
      grad1_line(n + 2, fl.data(), hl.data(), dl.data(), gl.data());
      for (int j = 0; j < n; ++j) dh3[j] = gl[j + 1];
      // x1 gradients over 1..lx1
      for (int j = 0; j < n; ++j) {
        h1l[j] = G->h1[X.g(j + 1, i2, i3)];
        dxl[j] = G->dx1[j + 1];  // x%dx1(1:lx1)
      }
      // ambipolar field: Epol1 = kB Te / qe * d log(ne kB Te)/dx1
      for (int j = 0; j < n; ++j) {
        const long long k = X.g(j + 1, i2, i3) + (LSP - 1) * X.ng;
        fl[j] = std::log(ns[k] * kB * Ts[k]);
      }
      grad1_line(n, fl.data(), h1l.data(), dxl.data(), gl.data());
      for (int j = 0; j < n; ++j) epol[j] = kB * Ts[X.g(j + 1, i2, i3) + (LSP - 1) * X.ng] / K.qs[LSP - 1] * gl[j];
      for (int isp = 0; isp < LSP; ++isp) {
        // ion pressure term pressure * d log(pressure)/dx1, and dQ/dx1
        for (int j = 0; j < n; ++j) {
          const long long k = X.g(j + 1, i2, i3) + isp * X.ng;
          pr_[j] = ns[k] * kB * Ts[k];
          fl[j] = std::log(pr_[j]);
        }
        grad1_line(n, fl.data(), h1l.data(), dxl.data(), pg.data());
        for (int j = 0; j < n; ++j) fl[j] = Q[isp * nc + X.c(j + 1, i2, i3)];
        grad1_line(n, fl.data(), h1l.data(), dxl.data(), gq.data());
        for (int j = 0; j < n; ++j) {
          const int i1 = j + 1;
          const long long c = X.c(i1, i2, i3), kg = X.g(i1, i2, i3), k = kg + isp * X.ng;
          double& pr = Pr[isp * nc + c];
          double& lo = Lo[isp * nc + c];
          const double ms = K.ms[isp];
          for (int isp2 = 0; isp2 < LN; ++isp2) {  // ion-neutral
            const double nu = maxwell_colln(isp, isp2, nn[isp2 * nc + c], Tn[c], Ts[k]);
            lo = lo + nu;
            pr = pr + ns[k] * ms * nu * vn1[c];
          }
          for (int isp2 = 0; isp2 < LSP; ++isp2) {  // ion-ion
            double nu, Phi, Psi;
            const long long k2 = kg + isp2 * X.ng;
            coulomb_colln(isp, isp2, ns[k2], Ts[k], Ts[k2], vs1[k], vs1[k2], nu, Phi, Psi);
            lo = lo + nu * Phi;
            pr = pr + ns[k] * ms * nu * Phi * vs1[k2];
          }
          const double ionpress = pr_[j] * pg[j];
          const double h1h2h3 = G->h1[kg] * G->h2[kg] * G->h3[kg];
          const double geom = (vs2[k] * vs2[k] * G->h3[kg] * dh2[j] + vs3[k] * vs3[k] * G->h2[kg] * dh3[j]) * ns[k] *
                              ms / h1h2h3;
          const double e1f = (alt[c] < 100e3) ? 0.0 : E1[kg];
          pr = pr + ns[k] * K.qs[isp] * (e1f + epol[j]) - ionpress - gq[j] + geom + ns[k] * ms * g1[c];
        }
      }
    }
}

// calculus.in.f90:174-196 ETD_uncoupled on interior arrays of n values.
void ora_etd_uncoupled(long long n, const double* f, const double* P, const double* L, double dt, double* out) {
  for (long long q = 0; q < n; ++q) {
    const double Ldt = L[q] * dt;
    const double expL = std::exp(-1.0 * Ldt);
    out[q] = (Ldt > 1e-10) ? f[q] * expL + P[q] / L[q] * (1 - expL) : f[q] + P[q] * dt;
  }
}

// multifluid.f90:532-549 mass_source_loss_solve.  Pr, Lo, Prprecip: interior
// (lx1,lx2,lx3,lsp) / (.,lsp-1); Pr is updated in place as the reference does; ns ghosted.
void ora_mass_source_loss_solve(const ora_grid* G, double dt, double* Pr, const double* Lo, const double* Prprecip,
                                double* ns) {
  Ix X(G);
  const long long nc = X.nc();
  for (int s = 0; s < LSP - 1; ++s)
    for (long long q = 0; q < nc; ++q) Pr[s * nc + q] = Pr[s * nc + q] + Prprecip[s * nc + q];
  std::vector<double> f(nc), o(nc);
  for (int s = 0; s < LSP - 1; ++s) {
    double* n = ns + s * X.ng;
    for (int i3 = 1; i3 <= G->lx3; ++i3)
      for (int i2 = 1; i2 <= G->lx2; ++i2)
        for (int i1 = 1; i1 <= G->lx1; ++i1) f[X.c(i1, i2, i3)] = n[X.g(i1, i2, i3)];
    ora_etd_uncoupled(nc, f.data(), Pr + s * nc, Lo + s * nc, dt, o.data());
    for (int i3 = 1; i3 <= G->lx3; ++i3)
      for (int i2 = 1; i2 <= G->lx2; ++i2)
        for (int i1 = 1; i1 <= G->lx1; ++i1) n[X.g(i1, i2, i3)] = o[X.c(i1, i2, i3)];
  }
  // ns(:,:,:,lsp) = sum(ns(:,:,:,1:lsp-1),4), ghosts included
  for (long long k = 0; k < X.ng; ++k) {
    double sum = 0.0;
    for (int s = 0; s < LSP - 1; ++s) sum = sum + ns[s * X.ng + k];
    ns[(LSP - 1) * X.ng + k] = sum;
  }
}

// multifluid.f90:500-528 momentum_source_loss_solve (J1 not used, as in the reference).
void ora_momentum_source_loss_solve(const ora_grid* G, double dt, const double* Pr, const double* Lo,
                                    const double* ns, double* rhovs1, double* vs1) {
  Ix X(G);
  const long long nc = X.nc();
  std::vector<double> f(nc), o(nc);
  for (int s = 0; s < LSP - 1; ++s) {
    double* r = rhovs1 + s * X.ng;
    for (int i3 = 1; i3 <= G->lx3; ++i3)
      for (int i2 = 1; i2 <= G->lx2; ++i2)
        for (int i1 = 1; i1 <= G->lx1; ++i1) f[X.c(i1, i2, i3)] = r[X.g(i1, i2, i3)];
    ora_etd_uncoupled(nc, f.data(), Pr + s * nc, Lo + s * nc, dt, o.data());
    for (int i3 = 1; i3 <= G->lx3; ++i3)
      for (int i2 = 1; i2 <= G->lx2; ++i2)
        for (int i1 = 1; i1 <= G->lx1; ++i1) r[X.g(i1, i2, i3)] = o[X.c(i1, i2, i3)];
    for (long long k = 0; k < X.ng; ++k)
      vs1[s * X.ng + k] = r[k] / (K.ms[s] * fmax_f(ns[s * X.ng + k], mindensdiv));
  }
  for (long long k = 0; k < X.ng; ++k) {
    double chrgflux = 0.0;
    for (int s = 0; s < LSP - 1; ++s) chrgflux = chrgflux + ns[s * X.ng + k] * K.qs[s] * vs1[s * X.ng + k];
    const long long ke = (LSP - 1) * X.ng + k;
    vs1[ke] = -1 / fmax_f(ns[ke], mindensdiv) / K.qs[LSP - 1] * chrgflux;
    rhovs1[ke] = ns[ke] * K.ms[LSP - 1] * vs1[ke];
  }
}

// multifluid.f90:474-495 energy_source_loss_solve.  Qeprecip: interior (lx1,lx2,lx3).
void ora_energy_source_loss_solve(const ora_grid* G, double dt, double* Pr, const double* Lo,
                                  const double* Qeprecip, double* rhoes, double* Ts, const double* ns) {
  Ix X(G);
  const long long nc = X.nc();
  std::vector<double> f(nc), o(nc);
  for (int s = 0; s < LSP; ++s) {
    if (s == LSP - 1)
      for (long long q = 0; q < nc; ++q) Pr[s * nc + q] = Pr[s * nc + q] + Qeprecip[q];
    double* re = rhoes + s * X.ng;
    for (int i3 = 1; i3 <= G->lx3; ++i3)
      for (int i2 = 1; i2 <= G->lx2; ++i2)
        for (int i1 = 1; i1 <= G->lx1; ++i1) f[X.c(i1, i2, i3)] = re[X.g(i1, i2, i3)];
    ora_etd_uncoupled(nc, f.data(), Pr + s * nc, Lo + s * nc, dt, o.data());
    for (int i3 = 1; i3 <= G->lx3; ++i3)
      for (int i2 = 1; i2 <= G->lx2; ++i2)
        for (int i1 = 1; i1 <= G->lx1; ++i1) re[X.g(i1, i2, i3)] = o[X.c(i1, i2, i3)];
    for (long long k = 0; k < X.ng; ++k) {
      const double T = (K.gammas[s] - 1) / kB * re[k] / fmax_f(ns[s * X.ng + k], mindensdiv);
      Ts[s * X.ng + k] = fmax_f(T, 100.0);
    }
  }
}

int ora_fluid_adv_compression(const ora_grid* G, double* fluidvars, double* fluidauxvars, const double* J1,
                              double* vs1i, double* vs2i, double* vs3i, const double* nn, const double* Tn,
                              double dt, double Teinf, int diffsolvetype) {
  std::vector<double> Q;
  return fluid_adv_compression_q(G, fluidvars, fluidauxvars, J1, vs1i, vs2i, vs3i, nn, Tn, dt, Teinf, diffsolvetype,
                                 Q);
}

// app/main.f90:280-381 fluid_adv in full on a single rank: the step with compression, then
// (after the ionization, whose rates Prionize (lx1,lx2,lx3,lsp-1) and Qeionize (lx1,lx2,lx3)
// are inputs here) set_global_boundaries, the energy, momentum and mass source/loss solves
// (libgemini.f90:1154-1200) with the compression step's Q, and clean_param(3), (2), (1).
// nn: interior (lx1,lx2,lx3,>=6) neutral densities O, N2, O2, H, N, NO (the diffusion reads
// the first three); vn1..3, Tn, alt, g1: interior; E1, J1: ghosted.
int ora_fluid_adv_full(const ora_grid* G, double* fluidvars, double* fluidauxvars, const double* E1,
                       const double* J1, double* vs1i, double* vs2i, double* vs3i, const double* nn,
                       const double* vn1, const double* vn2, const double* vn3, const double* Tn, const double* alt,
                       const double* g1, const double* Prionize, const double* Qeionize, double dt, double Teinf,
                       int diffsolvetype) {
  Ix X(G);
  std::vector<double> Q;
  const int rc = fluid_adv_compression_q(G, fluidvars, fluidauxvars, J1, vs1i, vs2i, vs3i, nn, Tn, dt, Teinf,
                                         diffsolvetype, Q);
  if (rc != 0) return rc;
  double* ns = fluidvars;
  double* vs1 = fluidvars + LSP * X.ng;
  double* vs2 = fluidvars + 2 * LSP * X.ng;
  double* vs3 = fluidvars + 3 * LSP * X.ng;
  double* Ts = fluidvars + 4 * LSP * X.ng;
  double* rhovs1 = fluidauxvars;
  double* rhoes = fluidauxvars + LSP * X.ng;
  const long long nc = X.nc();
  std::vector<double> Pr((size_t)LSP * nc), Lo((size_t)LSP * nc), Prion(Prionize, Prionize + (LSP - 1) * nc);
  ora_set_global_boundaries_allspec(G, ns, rhovs1, vs1, vs2, vs3, rhoes, vs1i, LSP);
  ora_srcs_energy(G, nn, vn1, vn2, vn3, Tn, ns, vs1, vs2, vs3, Ts, Pr.data(), Lo.data());
  ora_energy_source_loss_solve(G, dt, Pr.data(), Lo.data(), Qeionize, rhoes, Ts, ns);
  ora_srcs_momentum(G, nn, vn1, Tn, ns, vs1, vs2, vs3, Ts, E1, Q.data(), alt, g1, Pr.data(), Lo.data());
  ora_momentum_source_loss_solve(G, dt, Pr.data(), Lo.data(), ns, rhovs1, vs1);
  ora_srcs_continuity(G, nn, vn1, vn2, vn3, Tn, ns, vs1, vs2, vs3, Ts, Pr.data(), Lo.data());
  ora_mass_source_loss_solve(G, dt, Pr.data(), Lo.data(), Prion.data(), ns);
  ora_clean_param(G, 3, Ts);
  ora_clean_param(G, 2, vs1);
  ora_clean_param(G, 1, ns);
  return 0;
}

// libgemini_mpi.f90:449-482 dt_select with temporal_mpi.f90:26-66 dt_comm on a single rank:
// the CFL step, clipped so that t + dt does not pass the next GLOW output (when flagglow)
// and then the next output, floored at 1e-6, and -- from the second iteration -- grown by
// at most dtscale = 2 (libgemini_mpi.f90:38) over the previous step.  (ora_dt_calc floors
// first; flooring before and after the clips gives the reference's clip-then-floor.)
double ora_dt_select(const ora_grid* G, double tcfl, const double* Ts, const double* vs1, const double* vs2,
                     const double* vs3, double t, double tout, double tglowout, int flagglow, int it,
                     double dtprev) {
  double dt = ora_dt_calc(G, tcfl, Ts, vs1, vs2, vs3, nullptr);
  if (flagglow != 0 && t + dt > tglowout) dt = tglowout - t;
  if (t + dt > tout) dt = tout - t;
  dt = fmax_f(dt, 1e-6);
  const double dtscale = 2;
  if (it > 1 && dt / dtprev > dtscale) dt = dtscale * dtprev;
  return dt;
}

void ora_set_diffusion_solver(int mode) { g_diff_solver = mode; }
void ora_set_pow_mode(int mode) { g_pow_mode = mode; }
double ora_pow25(double x) { return pow25(x); }

int ora_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void ora_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}


// Checker for the device's exact division (test infrastructure): with y = RN(1/b),
// q0 = RN(a*y), r = fma(-q0, b, a), q = fma(r, y, q0) must equal RN(a/b) whenever the
// device's guard accepts (|a| in [2^-500, 2^500), |y| in [2^-400, 2^400)); a zero
// numerator returns q0.  Random operands over the guarded range plus near-representable
// quotients (a = RN(b*q) for random q), which are the hard cases of the correction.
// Returns the number of mismatches; *checked receives the number of guarded cases.
long long ora_markstein_mismatches(long long n, unsigned long long seed, long long* checked) {
  unsigned long long st = seed * 0x9E3779B97F4A7C15ull + 1;
  auto next = [&]() {
    st ^= st << 13;
    st ^= st >> 7;
    st ^= st << 17;
    return st;
  };
  auto rnd = [&](int emin, int emax) {
    const unsigned long long m = (next() >> 11) | (1ull << 52);  // 53-bit significand
    const int e = emin + (int)(next() % (unsigned long long)(emax - emin + 1));
    const double v = std::ldexp((double)m, e - 52);
    return (next() & 1) ? -v : v;
  };
  auto guard = [](double a, double y) {
    const double aa = std::fabs(a), ay = std::fabs(y);
    return aa >= std::ldexp(1.0, -500) && aa < std::ldexp(1.0, 500) && ay >= std::ldexp(1.0, -400) &&
           ay < std::ldexp(1.0, 400);
  };
  long long bad = 0, cnt = 0;
  for (long long i = 0; i < n; ++i) {
    const double b = rnd(-399, 399);
    double a;
    if (i % 3 == 0) {
      a = rnd(-499, 499);
    } else {
      const double q = rnd(-60, 60);
      a = b * q;  // a/b lands next to a representable quotient
      if (i % 3 == 2) a = std::nextafter(a, (next() & 1) ? 1e308 : -1e308);
    }
    if (i % 1000 == 0) a = (i % 2000 == 0) ? 0.0 : -0.0;
    const double y = 1.0 / b;
    const double q0 = a * y;
    const double r = std::fma(-q0, b, a);
    const double q1 = std::fma(r, y, q0);
    double q;
    if (guard(a, y)) {
      q = q1;
    } else if (a == 0.0 && std::fabs(y) >= std::ldexp(1.0, -400) && std::fabs(y) < std::ldexp(1.0, 400)) {
      q = q0;
    } else {
      continue;
    }
    ++cnt;
    const double ref = a / b;
    if (std::memcmp(&q, &ref, sizeof(double)) != 0) ++bad;
  }
  if (checked) *checked = cnt;
  return bad;
}

}  // extern "C"
