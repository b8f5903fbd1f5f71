// The source/loss solves of the source sub-step (libgemini.f90:1154-1200): per-cell bodies.
//
//   etd       calculus.in.f90:174-196 ETD_uncoupled: f exp(-L dt) + P/L (1 - exp(-L dt)), or
//             f + P dt when L dt <= 1e-10;
//   mass      multifluid.f90:532-549 mass_source_loss_solve: Pr += Prprecip (in place), the
//             ETD step of ns for the six ion species at interior cells, then the electron
//             density as the sum of the ion densities over every cell, ghosts included;
//   momentum  multifluid.f90:500-528 momentum_source_loss_solve: the ETD step of rhovs1 for
//             the ions at interior cells, vs1 = rhovs1 / (m max(n, 1e-5)) over every cell, and
//             the electron drift from the ion current, vs1e = -1/max(ne, 1e-5)/qe * sum n q v;
//   energy    multifluid.f90:474-495 energy_source_loss_solve: Pr(lsp) += Qeprecip (in place),
//             the ETD step of rhoes for every species at interior cells, then
//             Ts = max((gamma-1)/kB rhoe / max(n, 1e-5), 100) over every cell.
//
// Every per-cell quantity depends on the same cell only, so one body handles one cell of the
// ghosted block (all species), and the same code runs on the device (one thread per cell)
// and, compiled for the host, over every cell on a CPU.  Pr, Lo, Prprecip and Qeprecip are
// interior arrays (lx1, lx2, lx3, species) in column-major order.  Every operation follows
// the reference's order; exp is the platform's double exp (the device's on the GPU).
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define GEMS_HD __host__ __device__ __forceinline__
#else
#define GEMS_HD inline
#endif

namespace gems {

constexpr int NSP = 7;
constexpr double KB_ = 1.38064852e-23;   // phys_consts.in.f90:24
constexpr double MINDENSDIV_ = 1.0e-5;   // phys_consts.in.f90:84

struct View {
  int lx1, lx2, lx3;
  long long s2, s3, ng;
  double ms[NSP], qs[NSP], gam[NSP];  // species masses, charges, adiabatic indices
};

GEMS_HD double fmax_s(double a, double b) { return (a > b) ? a : b; }
GEMS_HD long long ncell(const View& v) { return (long long)v.lx1 * v.lx2 * v.lx3; }

// ghosted linear index k -> whether it is an interior cell, and then its column-major
// interior index c
GEMS_HD bool interior(const View& v, long long k, long long& c) {
  const int i1 = (int)(k % v.s2) - 1;
  const int i2 = (int)((k / v.s2) % (v.lx2 + 4)) - 1;
  const int i3 = (int)(k / v.s3) - 1;
  if (i1 < 1 || i1 > v.lx1 || i2 < 1 || i2 > v.lx2 || i3 < 1 || i3 > v.lx3) return false;
  c = (long long)(i1 - 1) + (long long)v.lx1 * ((i2 - 1) + (long long)v.lx2 * (i3 - 1));
  return true;
}

GEMS_HD double etd(double f, double P, double L, double dt) {
  const double Ldt = L * dt;
  const double expL = exp(-1.0 * Ldt);
  return (Ldt > 1e-10) ? f * expL + P / L * (1 - expL) : f + P * dt;
}

GEMS_HD void mass_cell(const View& v, long long k, double dt, double* Pr, const double* Lo, const double* Prprecip,
                       double* ns) {
  long long c = 0;
  const bool in = interior(v, k, c);
  const long long nc = ncell(v);
  double sum = 0.0;
  for (int s = 0; s < NSP - 1; ++s) {
    double n = ns[s * v.ng + k];
    if (in) {
      const double P = Pr[s * nc + c] + Prprecip[s * nc + c];
      Pr[s * nc + c] = P;
      n = etd(n, P, Lo[s * nc + c], dt);
      ns[s * v.ng + k] = n;
    }
    sum = sum + n;
  }
  ns[(NSP - 1) * v.ng + k] = sum;
}

GEMS_HD void momentum_cell(const View& v, long long k, double dt, const double* Pr, const double* Lo, const double* ns,
                           double* rhovs1, double* vs1) {
  long long c = 0;
  const bool in = interior(v, k, c);
  const long long nc = ncell(v);
  double chrg = 0.0;
  for (int s = 0; s < NSP - 1; ++s) {
    double r = rhovs1[s * v.ng + k];
    if (in) {
      r = etd(r, Pr[s * nc + c], Lo[s * nc + c], dt);
      rhovs1[s * v.ng + k] = r;
    }
    const double n = ns[s * v.ng + k];
    const double u = r / (v.ms[s] * fmax_s(n, MINDENSDIV_));
    vs1[s * v.ng + k] = u;
    chrg = chrg + n * v.qs[s] * u;
  }
  const long long ke = (NSP - 1) * v.ng + k;
  const double ne = ns[ke];
  const double ue = -1 / fmax_s(ne, MINDENSDIV_) / v.qs[NSP - 1] * chrg;
  vs1[ke] = ue;
  rhovs1[ke] = ne * v.ms[NSP - 1] * ue;
}

GEMS_HD void energy_cell(const View& v, long long k, double dt, double* Pr, const double* Lo, const double* Qeprecip,
                         double* rhoes, double* Ts, const double* ns) {
  long long c = 0;
  const bool in = interior(v, k, c);
  const long long nc = ncell(v);
  for (int s = 0; s < NSP; ++s) {
    double re = rhoes[s * v.ng + k];
    if (in) {
      double P = Pr[s * nc + c];
      if (s == NSP - 1) {
        P = P + Qeprecip[c];
        Pr[s * nc + c] = P;
      }
      re = etd(re, P, Lo[s * nc + c], dt);
      rhoes[s * v.ng + k] = re;
    }
    const double T = (v.gam[s] - 1) / KB_ * re / fmax_s(ns[s * v.ng + k], MINDENSDIV_);
    Ts[s * v.ng + k] = fmax_s(T, 100.0);
  }
}

}  // namespace gems
