// The production/loss rates of the source sub-step (sources.f90) as per-cell bodies:
//
//   continuity  sources.f90:18-276 srcsContinuity: the 21 ion-chemistry reactions of one
//               interior cell, in the reference's order, into Pr and Lo of all seven species
//               (the electrons' stay 0);
//   energy      sources.f90:396-485 srcsEnergy for one (cell, species): elastic exchange with
//               the four neutrals (collisions.f90:58-114 maxwell_colln) and with every charged
//               species (collisions.f90:117-159 coulomb_colln), and for the electrons the
//               rotational and vibrational inelastic losses to N2 and O2;
//   momentum    sources.f90:279-393 srcsMomentum_curv on a single rank for one (cell,
//               species): collisions with neutrals and charged species, the ambipolar field,
//               the pressure gradient, the artificial-viscosity gradient, the curvature terms,
//               the parallel field (zeroed below 100 km) and gravity.
//
// The x1 gradients (calculus/gradient.f90:79-150 grad3D1_curv_23) are evaluated at the cell
// itself from its x1 neighbours: centred in the interior, one-sided at the line ends, where
// the reference divides the first point's difference by dx1 of that point.  The metric
// gradients dh2/dx1, dh3/dx1 are taken over the line 0..lx1+1, so they are centred at every
// interior cell.
//
// Integer powers are expanded as gfortran expands them (x**2 = x*x, x**3 = (x*x)*x,
// x**4 = (x*x)*(x*x)); real powers call pow; the collision coefficient tables are the
// reference's default-REAL (float) literals widened to double.  Every expression follows the
// reference's operation order, so the same bodies compiled for the host with the C library's
// math functions reproduce the reference restatement bit for bit; on the device the math
// functions (pow, exp, log, log10, erf, tanh, sin) are the device's own, and the powers 0.5
// and 1.5 come from the square root (pow_half, pow_3half).
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define GEMR_HD __host__ __device__ __forceinline__
#else
#define GEMR_HD inline
#endif

namespace gemr {

constexpr int NSP = 7;  // O+, NO+, N2+, O2+, N+, H+, e-
constexpr int NNEU = 4;  // collision partners O, N2, O2, H (phys_consts.in.f90:39)
constexpr double AMU_ = 1.660539040e-27;  // phys_consts.in.f90:26
constexpr double KB_ = 1.38064852e-23;    // phys_consts.in.f90:24
constexpr double ELCHRG_ = 1.60217662e-19;  // phys_consts.in.f90:25

struct View {
  int lx1, lx2, lx3;
  long long s2, s3, ng, c3;
  const double *h1, *h2, *h3;  // ghosted metric factors (x3 stride c3), or null (unit metric)
  const double* yh1;           // device only: RN(1/h1) in the same layout, or null (unit metric)
  const double* dx1;           // backward differences dx1(j), j = 0..lx1+2
  double ms[NSP], qs[NSP], gam[NSP];
  double pi;  // 4 atan(1), formed on the host
  // device only: RN(1/(ms_i + mn_j)) and RN(1/(ms_i + ms_j)), formed on the host (qdk)
  double ymn[NSP][NNEU], yms[NSP][NSP];
};

GEMR_HD long long ncell(const View& v) { return (long long)v.lx1 * v.lx2 * v.lx3; }
GEMR_HD long long gix(const View& v, int i1, int i2, int i3) {
  return (long long)(i1 + 1) + v.s2 * (i2 + 1) + v.s3 * (i3 + 1);
}
GEMR_HD double hm(const double* h, const View& v, int i1, int i2, int i3) {
  return h ? h[(long long)(i1 + 1) + v.s2 * (i2 + 1) + v.c3 * (i3 + 1)] : 1.0;
}
GEMR_HD void cell_of(const View& v, long long c, int& i1, int& i2, int& i3) {
  i1 = (int)(c % v.lx1) + 1;
  const long long r = c / v.lx1;
  i2 = (int)(r % v.lx2) + 1;
  i3 = (int)(r / v.lx2) + 1;
}
GEMR_HD double fmax_r(double a, double b) { return (a > b) ? a : b; }
GEMR_HD double p2(double x) { return x * x; }
GEMR_HD double p3(double x) { return x * x * x; }
GEMR_HD double p4(double x) {
  const double t = x * x;
  return t * t;
}

// collisions.f90:12-55 coefficient tables (rows: charged species; columns: O, N2, O2, H or
// the charged species), default-REAL literals; constant memory on the device
#ifdef __CUDACC__
#define GEMR_TABLE __constant__ const
#else
#define GEMR_TABLE static const
#endif
GEMR_TABLE float kCsn[NSP][NNEU] = {{-1, 6.82e-10f, 6.64e-10f, -1},          {2.44e-10f, 4.34e-10f, 4.27e-10f, 0.69e-10f},
                                    {2.58e-10f, -1, 4.49e-10f, 0.74e-10f},    {2.31e-10f, 4.13e-10f, -1, 0.65e-10f},
                                    {4.42e-10f, 7.47e-10f, 7.25e-10f, 1.45e-10f}, {-1, 33.6e-10f, 32.0e-10f, -1},
                                    {-1, -1, -1, -1}};
GEMR_TABLE float kC2sn1[NSP][NNEU] = {{3.67e-11f, 0, 0, 4.63e-12f}, {0, 0, 0, 0}, {0, 5.14e-11f, 0, 0},
                                      {0, 0, 2.59e-11f, 0},         {0, 0, 0, 0}, {6.61e-11f, 0, 0, 2.65e-10f},
                                      {-1, -1, -1, -1}};
GEMR_TABLE float kC2sn2[NSP][NNEU] = {{0.064f, 0, 0, -1}, {0, 0, 0, 0},           {0, 0.069f, 0, 0}, {0, 0, 0.073f, 0},
                                      {0, 0, 0, 0},       {0.047f, 0, 0, 0.083f}, {-1, -1, -1, -1}};
GEMR_TABLE float kCsj[NSP][NSP] = {{0.22f, 0.26f, 0.25f, 0.26f, 0.22f, 0.077f, 1.87e-3f},
                                   {0.14f, 0.16f, 0.16f, 0.17f, 0.13f, 0.042f, 9.97e-4f},
                                   {0.15f, 0.17f, 0.17f, 0.18f, 0.14f, 0.045f, 1.07e-3f},
                                   {0.13f, 0.16f, 0.15f, 0.16f, 0.12f, 0.039f, 9.347e-4f},
                                   {0.25f, 0.28f, 0.28f, 0.28f, 0.24f, 0.088f, 2.136e-3f},
                                   {1.23f, 1.25f, 1.25f, 1.25f, 1.23f, 0.90f, 29.7e-3f},
                                   {54.5f, 54.5f, 54.5f, 54.5f, 54.5f, 54.5f, 38.537f}};
GEMR_TABLE double kMn[NNEU] = {16, 28, 32, 1};  // neutral masses / amu, phys_consts.in.f90:41

struct Coll {
  static GEMR_HD double csn(int i, int j) { return (double)kCsn[i][j]; }
  static GEMR_HD double c2sn1(int i, int j) { return (double)kC2sn1[i][j]; }
  static GEMR_HD double c2sn2(int i, int j) { return (double)kC2sn2[i][j]; }
  static GEMR_HD double csj(int i, int j) { return (double)kCsj[i][j]; }
  static GEMR_HD double mn(int j) { return kMn[j] * AMU_; }
};

// a/b for a constant divisor b whose correctly rounded reciprocal y = RN(1/b) was formed on
// the host.  On the device: q0 = RN(a*y), the exact remainder a - b*q0 and RN(q0 + r*y),
// which is the IEEE quotient whenever |a| lies in [2^-500, 2^500) (Markstein; every y here
// is near 2^±90); a zero numerator gives the correctly signed zero, anything else the IEEE
// division.  The host build divides.
GEMR_HD double qdk(double a, double b, double y) {
#ifdef __CUDA_ARCH__
  const double q0 = a * y;
  const double r = __fma_rn(-q0, b, a);
  const double q1 = __fma_rn(r, y, q0);
  if (((unsigned)__double2hiint(a) & 0x7fffffffu) - (523u << 20) < (1000u << 20)) return q1;
  if (a == 0.0) return q0;
  return a / b;
#else
  (void)y;
  return a / b;
#endif
}
constexpr double Y3 = 1.0 / 3;  // RN(1/3)

// qdk for a divisor formed at run time: y = RN(1/b) from the device's correctly rounded
// reciprocal, and the fast form also requires |y| in [2^-400, 2^400].  The host build divides.
GEMR_HD double qdk_v(double a, double b, double y) {
#ifdef __CUDA_ARCH__
  const double q0 = a * y;
  const double r = __fma_rn(-q0, b, a);
  const double q1 = __fma_rn(r, y, q0);
  const unsigned ha = (unsigned)__double2hiint(a) & 0x7fffffffu, hy = (unsigned)__double2hiint(y) & 0x7fffffffu;
  const bool yok = hy - (623u << 20) < (800u << 20);
  if ((ha - (523u << 20) < (1000u << 20)) & yok) return q1;
  if (a == 0.0 && yok) return q0;
  return a / b;
#else
  (void)y;
  return a / b;
#endif
}
// RN(1/b) on the device (the reciprocal qdk_v needs); the host build, which divides, gets 0
GEMR_HD double rcp_dev(double b) {
#ifdef __CUDA_ARCH__
  return __drcp_rn(b);
#else
  (void)b;
  return 0.0;
#endif
}

// x**0.5 and x**1.5 of the collision and reaction fits.  The host build calls pow, as the
// reference does; the device forms them from its correctly rounded square root (x**0.5
// correctly rounded, x**1.5 = x*sqrt(x) within 1.5 ulp), a fraction of the cost of its pow
// and as close to the exact power as the few-ulp device pow it replaces.
GEMR_HD double pow_half(double x) {
#ifdef __CUDA_ARCH__
  return sqrt(x);
#else
  return pow(x, 0.5);
#endif
}
GEMR_HD double pow_3half(double x) {
#ifdef __CUDA_ARCH__
  return x * sqrt(x);
#else
  return pow(x, 1.5);
#endif
}

// collisions.f90:58-114 for one cell: charged species isp, neutral isp2 of density nn2
GEMR_HD double maxwell_colln(int isp, int isp2, double nn2, double tn, double ts) {
  if (isp < NSP - 1) {
    if (Coll::csn(isp, isp2) < 0) {  // resonant
      if (isp == 0 && isp2 == 3) {
        const double Teff = tn + ts / 16;
        return Coll::c2sn1(isp, isp2) * pow_half(Teff) * nn2 * 1e-6;
      }
      const double Teff = 0.5 * (tn + ts);
      const double a = 1 - Coll::c2sn2(isp, isp2) * log10(Teff);
      return Coll::c2sn1(isp, isp2) * (a * a) * (pow_half(Teff)) * nn2 * 1e-6;
    }
    return Coll::csn(isp, isp2) * nn2 * 1e-6;
  }
  const double Teff = ts;
  switch (isp2) {
    case 0: return 8.9e-11 * (1.0 + 5.7e-4 * Teff) * (pow_half(Teff)) * nn2 * 1e-6;
    case 1: return 2.33e-11 * (1.0 - 1.21e-4 * Teff) * (Teff)*nn2 * 1e-6;
    case 2: return 1.82e-10 * (1.0 + 3.6e-2 * (pow_half(Teff))) * (pow_half(Teff)) * nn2 * 1e-6;
    default: return 4.5e-9 * (1.0 - 1.35e-4 * Teff) * (pow_half(Teff)) * nn2 * 1e-6;
  }
}

// collisions.f90:117-159, the part symmetric in the two species: Teff**1.5, Phi and Psi of
// the pair (isp, isp2).  Every operation is a commutative sum or product of the two sides or
// a function of such (no contraction into fused multiply-adds in these builds), so swapping
// the species gives the same bits and one evaluation serves both.
struct CoulPair {
  double P, Phi, Psi;  // Teff**1.5, Phi, Psi
  double yP;           // RN(1/P) on the device (rcp_dev)
};
GEMR_HD CoulPair coulomb_pair(const View& v, int isp, int isp2, double ts1, double ts2, double v1, double v2) {
  const double ms1 = v.ms[isp], ms2 = v.ms[isp2];
  const double Teff = (ms2 * ts1 + ms1 * ts2) / (ms2 + ms1);
  CoulPair q;
  q.P = pow_3half(Teff);
  q.yP = rcp_dev(q.P);
  const double mred = ms1 * ms2 / (ms1 + ms2);
  const double W = fabs(v1 - v2) / sqrt(2 * KB_ * Teff / mred);
  q.Psi = exp(-(W * W));
  if (W < 0.1)
    q.Phi = 1;
  else
    q.Phi = 3.0 / 4 * sqrt(v.pi) * erf(W) / (W * W * W) - 3.0 / 2 / (W * W) * q.Psi;
  return q;
}

// Pair source that evaluates each pair where it is needed
struct DirectPairs {
  GEMR_HD CoulPair operator()(const View& v, int isp, int isp2, double ts1, double ts2, double v1, double v2) const {
    return coulomb_pair(v, isp, isp2, ts1, ts2, v1, v2);
  }
};

// collisions.f90:117-159 for one cell: nu, Phi, Psi of species isp with isp2 (zero if equal);
// the pair's symmetric part comes from `pairs`
template <class Pairs>
GEMR_HD void coulomb_colln(const View& v, int isp, int isp2, double ns2, double ts1, double ts2, double v1, double v2,
                           double& nu, double& Phi, double& Psi, const Pairs& pairs) {
  if (isp == isp2) {
    nu = Phi = Psi = 0.0;
    return;
  }
  const CoulPair q = pairs(v, isp, isp2, ts1, ts2, v1, v2);
  nu = qdk_v(Coll::csj(isp, isp2) * ns2 * 1e-6, q.P, q.yP);
  Phi = q.Phi;
  Psi = q.Psi;
}

// ---- continuity: one interior cell c ------------------------------------------------------
// nn: interior (lx1,lx2,lx3, O N2 O2 H N NO); vn1..3, Tn: interior; ns, vs1..3, Ts: ghosted
GEMR_HD void continuity_cell(const View& v, long long c, const double* nn, const double* vn1, const double* vn2,
                             const double* vn3, const double* Tn, const double* ns, const double* vs1,
                             const double* vs2, const double* vs3, const double* Ts, double* Pr, double* Lo) {
  const long long nc = ncell(v);
  int i1, i2, i3;
  cell_of(v, c, i1, i2, i3);
  const long long k = gix(v, i1, i2, i3);
  double pr[NSP], lo[NSP];
  for (int s = 0; s < NSP; ++s) pr[s] = lo[s] = 0.0;
  // species and neutrals numbered from 1 as in the reference
#define NEU(j) nn[((j)-1) * nc + c]
#define NSx(s) ns[((s)-1) * v.ng + k]
#define TSx(s) Ts[((s)-1) * v.ng + k]
  const double tn = Tn[c];
  const double Te = TSx(NSP);
  const double dv2 = p2(vs1[k] - vn1[c]) + p2(vs2[k] - vn2[c]) + p2(vs3[k] - vn3[c]);
  double kreac = 0.0, Teff, b;
  // O+ + N2 -> NO+ + N
  Teff = 28 / (16 + 28.0) * (16 * AMU_ / 3 / KB_ * (dv2) + TSx(1) - tn) + tn;
  if (Teff <= 3725)
    kreac = 1.71676e-12 - 7.19934e-13 * (Teff / 300) + 1.33276e-13 * p2(Teff / 300) - 9.28213e-15 * p3(Teff / 300) +
            6.39557e-16 * p4(Teff / 300);
  if (Teff > 3725 && Teff <= 30000)
    kreac = -1.52489e-11 + 7.67112e-13 * (Teff / 300) + 1.19064e-13 * p2(Teff / 300) - 1.30858e-15 * p3(Teff / 300) +
            4.67756e-18 * p4(Teff / 300);
  if (Teff > 30000)
    kreac = -1.52489e-11 + 7.67112e-13 * (100) + 1.19064e-13 * (10000) - 1.30858e-15 * (1000000) +
            4.67756e-18 * (100000000);
  b = kreac * NEU(2) * 1e-6;
  pr[1] = pr[1] + b * NSx(1);
  lo[0] = lo[0] + b;
  // O+ + O2 -> O2+ + O
  Teff = 32 / (16 + 32.0) * (16 * AMU_ / 3 / KB_ * (dv2) + TSx(1) - tn) + tn;
  if (Teff <= 4800)
    kreac = 2.78932e-11 - 6.92612e-12 * (Teff / 300) + 8.67684e-13 * p2(Teff / 300) - 3.47251e-14 * p3(Teff / 300) +
            5.07097e-16 * p4(Teff / 300);
  if (Teff > 4800 && Teff <= 30000)
    kreac = -1.74046e-11 + 3.02328e-12 * Teff / 300 - 2.39214e-15 * p2(Teff / 300) - 4.02394e-17 * p3(Teff / 300);
  if (Teff > 30000) kreac = -1.74046e-11 + 3.02328e-12 * 100 - 2.39214e-15 * 10000 - 4.02394e-17 * 1000000;
  b = kreac * NEU(3) * 1e-6;
  pr[3] = pr[3] + b * NSx(1);
  lo[0] = lo[0] + b;
  // O+ + NO -> NO+ + O
  Teff = 30 / (16 + 30.0) * (16 * AMU_ / 3 / KB_ * (dv2) + TSx(1) - tn) + tn;
  if (Teff <= 3800)
    kreac = 6.40408e-13 - 1.33888e-13 * (Teff / 300) + 7.65103e-14 * p2(Teff / 300) - 3.11509e-15 * p3(Teff / 300) +
            6.62374e-17 * p4(Teff / 300);
  if (Teff > 3800 && Teff <= 30000)
    kreac = -7.48312e-13 + 2.31502e-13 * (Teff / 300) + 3.07160e-14 * p2(Teff / 300) - 2.65436e-16 * p3(Teff / 300) +
            7.76665e-19 * p4(Teff / 300);
  if (Teff > 30000)
    kreac = -7.48312e-13 + 2.31502e-13 * (100) + 3.07160e-14 * (10000) - 2.65436e-16 * (1000000) +
            7.76665e-19 * (100000000);
  b = kreac * NEU(6) * 1e-6;
  pr[1] = pr[1] + b * NSx(1);
  lo[0] = lo[0] + b;
  // O+ + e -> O + hv
  b = 3.7e-12 * pow(250 / TSx(NSP), 0.7) * NSx(NSP) * 1e-6;
  lo[0] = lo[0] + b;
  // N2+ + O -> O+ + N2
  Teff = 16 / (28 + 16.0) * (28 * AMU_ / 3 / KB_ * (dv2) + TSx(3) - tn) + tn;
  kreac = (Teff <= 1500) ? 1e-11 * pow(300 / Teff, 0.23) : 3.6e-12 * pow(300 / Teff, -0.41);
  b = kreac * NEU(1) * 1e-6;
  pr[0] = pr[0] + b * NSx(3);
  lo[2] = lo[2] + b;
  // N+ + O -> O+ + N
  b = 5e-13 * NEU(1) * 1e-6;
  pr[0] = pr[0] + b * NSx(5);
  lo[4] = lo[4] + b;
  // H+ + O -> O+ + H
  Teff = TSx(6);
  b = (6.e-10) * (8 / 9.0) * (pow_half((Teff + tn / 4) / (tn + Teff / 16))) * NEU(1) * 1e-6;
  pr[0] = pr[0] + b * NSx(6);
  lo[5] = lo[5] + b;
  // O+ + H -> H+ + O
  b = 6.0e-10 * NEU(4) * 1e-6;
  pr[5] = pr[5] + b * NSx(1);
  lo[0] = lo[0] + b;
  // O2+ + N2 -> NO+ + NO
  b = 5e-16 * NEU(3) * 1e-6;
  pr[1] = pr[1] + b * NSx(4);
  lo[3] = lo[3] + b;
  // O2+ + N -> NO+ + O
  b = 1.2e-10 * NEU(5) * 1e-6;
  pr[1] = pr[1] + b * NSx(4);
  lo[3] = lo[3] + b;
  // O2+ + NO -> NO+ + O2
  b = 4.6e-10 * NEU(6) * 1e-6;
  pr[1] = pr[1] + b * NSx(4);
  lo[3] = lo[3] + b;
  // N2+ + O -> NO+ + N
  Teff = 16 / (28 + 16.0) * (28 * AMU_ / 3 / KB_ * (dv2) + TSx(3) - tn) + tn;
  kreac = (Teff <= 1500) ? 1.4e-10 * pow(300 / Teff, 0.44) : 5.2e-11 * pow(300 / Teff, -0.2);
  b = kreac * NEU(1) * 1e-6;
  pr[1] = pr[1] + b * NSx(3);
  lo[2] = lo[2] + b;
  // N2+ + NO -> NO+ + N2
  b = 4.1e-10 * NEU(6) * 1e-6;
  pr[1] = pr[1] + b * NSx(3);
  lo[2] = lo[2] + b;
  // N+ + O2 -> NO+ + O
  b = 2.6e-10 * NEU(3) * 1e-6;
  pr[1] = pr[1] + b * NSx(5);
  lo[4] = lo[4] + b;
  // NO+ + e -> N + O
  b = 4.2e-7 * pow(300 / TSx(NSP), 0.85) * NSx(NSP) * 1e-6;
  lo[1] = lo[1] + b;
  // N2+ + O2 -> O2+ + N2
  Teff = 32 / (28 + 32.0) * (28 * AMU_ / 3 / KB_ * (dv2) + TSx(3) - tn) + tn;
  b = 5e-11 * (300 / Teff) * NEU(3) * 1e-6;
  pr[3] = pr[3] + b * NSx(3);
  lo[2] = lo[2] + b;
  // N2+ + e -> N + N
  b = 1.8e-7 * pow(300 / TSx(NSP), 0.39) * NSx(NSP) * 1e-6;
  lo[2] = lo[2] + b;
  // N+ + O2 -> O2+ + N
  b = 3.1e-10 * NEU(3) * 1e-6;
  pr[3] = pr[3] + b * NSx(5);
  lo[4] = lo[4] + b;
  // O2+ + e -> O + O
  kreac = (Te <= 1200) ? 1.95e-7 * pow(300 / Te, 0.70) : 7.38e-8 * pow(1200 / Te, 0.56);
  b = kreac * NSx(NSP) * 1e-6;
  lo[3] = lo[3] + b;
  // N+ + H -> H+ + N
  b = 3.6e-12 * NEU(4) * 1e-6;
  pr[5] = pr[5] + b * NSx(5);
  lo[4] = lo[4] + b;
  // H+ + e -> H + hv
  b = 3.7e-12 * pow(250 / TSx(NSP), 0.7) * NSx(NSP) * 1e-6;
  lo[5] = lo[5] + b;
#undef NEU
#undef NSx
#undef TSx
  for (int s = 0; s < NSP; ++s) {
    Pr[s * nc + c] = pr[s];
    Lo[s * nc + c] = lo[s];
  }
}

// ---- energy: index t = isp * ncell + c ----------------------------------------------------
// nn: interior (lx1,lx2,lx3, O N2 O2 H ...); the rest as continuity_cell
template <class Pairs = DirectPairs>
GEMR_HD void energy_rate(const View& v, long long t, const double* nn, const double* vn1, const double* vn2,
                         const double* vn3, const double* Tn, const double* ns, const double* vs1, const double* vs2,
                         const double* vs3, const double* Ts, double* Pr, double* Lo, const Pairs& pairs = Pairs()) {
  const long long nc = ncell(v);
  const int isp = (int)(t / nc);
  const long long c = t - isp * nc;
  int i1, i2, i3;
  cell_of(v, c, i1, i2, i3);
  const long long k = gix(v, i1, i2, i3);
  const double tn = Tn[c];
  const double ms = v.ms[isp], gm1 = v.gam[isp] - 1;
  const double nsk = ns[isp * v.ng + k], tsk = Ts[isp * v.ng + k];
  const double u1 = vs1[isp * v.ng + k], u2 = vs2[isp * v.ng + k], u3 = vs3[isp * v.ng + k];
  double pr = 0.0, lo = 0.0;
  for (int j = 0; j < NNEU; ++j) {  // with the neutrals
    const double nu = maxwell_colln(isp, j, nn[j * nc + c], tn, tsk);
    double fact = qdk(2 * nu, ms + Coll::mn(j), v.ymn[isp][j]);
    pr = pr + nsk * ms * KB_ / gm1 * fact * tn;
    lo = lo + ms * fact;
    fact = qdk(fact * Coll::mn(j), 3, Y3);
    const double d1 = u1 - vn1[c], d2 = u2 - vn2[c], d3 = u3 - vn3[c];
    pr = pr + nsk * ms / gm1 * ((d1 * d1) + (d2 * d2) + (d3 * d3)) * fact;
  }
  for (int j = 0; j < NSP; ++j) {  // with the charged species
    const long long kj = j * v.ng + k;
    double nu, Phi, Psi;
    coulomb_colln(v, isp, j, ns[kj], tsk, Ts[kj], u1, vs1[kj], nu, Phi, Psi, pairs);
    double fact = qdk(2 * nu * Psi, ms + v.ms[j], v.yms[isp][j]);
    pr = pr + nsk * ms * KB_ / gm1 * fact * Ts[kj];
    lo = lo + ms * fact;
    fact = qdk(qdk(2 * nu * Phi, ms + v.ms[j], v.yms[isp][j]) * v.ms[j], 3, Y3);
    const double d1 = u1 - vs1[kj], d2 = u2 - vs2[kj], d3 = u3 - vs3[kj];
    pr = pr + nsk * ms / gm1 * ((d1 * d1) + (d2 * d2) + (d3 * d3)) * fact;
  }
  if (isp == NSP - 1) {  // inelastic electron losses: rotational, then vibrational excitation
    const double sfact = ELCHRG_ / KB_ * (v.gam[NSP - 1] - 1);
    const double Te = tsk;
    double nu = sfact * 6.9e-14 * nn[2 * nc + c] * 1e-6 / sqrt(Te);  // O2 rotational
    double iePT = nu * tn;
    double ieLT = nu;
    nu = sfact * 2.9e-14 * nn[1 * nc + c] * 1e-6 / sqrt(Te);  // N2 rotational
    iePT = iePT + nu * tn;
    ieLT = ieLT + nu;
    double f = 1.06e4 + 7.51e3 * tanh(1.10e-3 * (Te - 1800));
    const double g = 3300 + 1.233 * (Te - 1000) - 2.056e-4 * (Te - 1000) * (Te - 4000);
    double fact = sfact * 2.99e-12 * nn[1 * nc + c] * 1e-6 * exp(f * (Te - 2000) / Te / 2000) *
                  (exp(-g * (Te - tn) / Te / tn) - 1);  // N2 vibrational
    iePT = iePT - fmax_r(fact, 0.0);
    f = 3300 - 839 * sin(1.91e-4 * (Te - 2700));
    fact = sfact * 5.196e-13 * nn[2 * nc + c] * 1e-6 * exp(f * (Te - 700) / Te / 700) *
           (exp(-2770 * (Te - tn) / Te / tn) - 1);  // O2 vibrational
    iePT = iePT - fmax_r(fact, 0.0);
    pr = pr + iePT * nsk * KB_ / (v.gam[NSP - 1] - 1);
    lo = lo + ieLT;
  }
  Pr[t] = pr;
  Lo[t] = lo;
}

// ---- momentum: index t = isp * ncell + c --------------------------------------------------
// The divisors of the x1 gradients at interior cell (i1, i2, i3): e, the line difference's
// divisor (dx1(i1+1) + dx1(i1) inside the line, dx1(1) and dx1(lx1) at its ends), and h1,
// with their reciprocals for qdk_v on the device
struct X1Div {
  double e, ye, h1, yh1;
};
GEMR_HD X1Div x1_div(const View& v, int i1, int i2, int i3) {
  X1Div q;
  q.e = (i1 == 1) ? v.dx1[1] : (i1 == v.lx1) ? v.dx1[v.lx1] : v.dx1[i1 + 1] + v.dx1[i1];
  q.ye = rcp_dev(q.e);
  q.h1 = hm(v.h1, v, i1, i2, i3);
#ifdef __CUDA_ARCH__
  q.yh1 = hm(v.yh1, v, i1, i2, i3);
#else
  q.yh1 = 0.0;  // the host build divides
#endif
  return q;
}

// x1 derivative of f at interior x1 index i (1..lx1) over the line 1..lx1, as
// grad3D1_curv_23 forms it: fm, f0, fp at i-1, i, i+1 (ends use only the side present)
GEMR_HD double dx1_line(const View& v, int i, double fm, double f0, double fp, const X1Div& q) {
  if (i == 1) return qdk_v(qdk_v(fp - f0, q.e, q.ye), q.h1, q.yh1);
  if (i == v.lx1) return qdk_v(qdk_v(f0 - fm, q.e, q.ye), q.h1, q.yh1);
  return qdk_v(qdk_v(fp - fm, q.e, q.ye), q.h1, q.yh1);
}

// The two x1 log-gradient terms of momentum_rate, evaluated where they are needed: the
// ambipolar field kB Te / qe * d log(ne kB Te)/dx1 and the species' d log(ns kB Ts)/dx1 at
// interior cell (i1, .) with ghosted index kg and x1 neighbours km, kp inside 1..lx1
struct DirectX1 {
  GEMR_HD double epol(const View& v, const double* ns, const double* Ts, int i1, long long kg, long long km,
                      long long kp, const X1Div& q) const {
    const long long e = (long long)(NSP - 1) * v.ng;
    const double le0 = log(ns[e + kg] * KB_ * Ts[e + kg]);
    const double lem = log(ns[e + km] * KB_ * Ts[e + km]);
    const double lep = log(ns[e + kp] * KB_ * Ts[e + kp]);
    return KB_ * Ts[e + kg] / v.qs[NSP - 1] * dx1_line(v, i1, lem, le0, lep, q);
  }
  GEMR_HD double pg(const View& v, const double* ns, const double* Ts, long long s0, int i1, long long kg,
                    long long km, long long kp, const X1Div& q) const {
    const double lp0 = log(ns[s0 + kg] * KB_ * Ts[s0 + kg]);
    const double lpm = log(ns[s0 + km] * KB_ * Ts[s0 + km]);
    const double lpp = log(ns[s0 + kp] * KB_ * Ts[s0 + kp]);
    return dx1_line(v, i1, lpm, lp0, lpp, q);
  }
};

// nn: interior (lx1,lx2,lx3, O N2 O2 H ...); vn1, Tn, alt, g1: interior; Q: interior
// (lx1,lx2,lx3,lsp); ns, vs1..3, Ts, E1: ghosted
template <class Pairs = DirectPairs, class X1 = DirectX1>
GEMR_HD void momentum_rate(const View& v, long long t, const double* nn, const double* vn1, const double* Tn,
                           const double* ns, const double* vs1, const double* vs2, const double* vs3, const double* Ts,
                           const double* E1, const double* Q, const double* alt, const double* g1, double* Pr,
                           double* Lo, const Pairs& pairs = Pairs(), const X1& x1 = X1()) {
  const long long nc = ncell(v);
  const int isp = (int)(t / nc);
  const long long c = t - isp * nc;
  int i1, i2, i3;
  cell_of(v, c, i1, i2, i3);
  const long long kg = gix(v, i1, i2, i3), k = kg + isp * v.ng;
  const double ms = v.ms[isp];
  const X1Div q = x1_div(v, i1, i2, i3);
  const double h1 = q.h1, h2 = hm(v.h2, v, i1, i2, i3), h3 = hm(v.h3, v, i1, i2, i3);
  // dh2/dx1, dh3/dx1 over the line 0..lx1+1 (centred at every interior cell; inside the
  // line dd is the gradients' divisor e)
  const double dd = v.dx1[i1 + 1] + v.dx1[i1];
  const double ydd = (i1 == 1 || i1 == v.lx1) ? rcp_dev(dd) : q.ye;
  const double dh2 = qdk_v(qdk_v(hm(v.h2, v, i1 + 1, i2, i3) - hm(v.h2, v, i1 - 1, i2, i3), dd, ydd), h1, q.yh1);
  const double dh3 = qdk_v(qdk_v(hm(v.h3, v, i1 + 1, i2, i3) - hm(v.h3, v, i1 - 1, i2, i3), dd, ydd), h1, q.yh1);
  const int im = (i1 > 1) ? i1 - 1 : i1, ip = (i1 < v.lx1) ? i1 + 1 : i1;  // neighbours inside 1..lx1
  const long long km = gix(v, im, i2, i3), kp = gix(v, ip, i2, i3);
  // ambipolar field kB Te / qe * d log(ne kB Te)/dx1
  const double epol = x1.epol(v, ns, Ts, i1, kg, km, kp, q);
  // pressure * d log(pressure)/dx1 and dQ/dx1
  const long long s0 = (long long)isp * v.ng;
  const double pres = ns[s0 + kg] * KB_ * Ts[s0 + kg];
  const double pg = x1.pg(v, ns, Ts, s0, i1, kg, km, kp, q);
  const long long qb = (long long)isp * nc;
  const long long cm = c - (i1 - im), cp = c + (ip - i1);
  const double gq = dx1_line(v, i1, Q[qb + cm], Q[qb + c], Q[qb + cp], q);
  double pr = 0.0, lo = 0.0;
  for (int j = 0; j < NNEU; ++j) {  // with the neutrals
    const double nu = maxwell_colln(isp, j, nn[j * nc + c], Tn[c], Ts[k]);
    lo = lo + nu;
    pr = pr + ns[k] * ms * nu * vn1[c];
  }
  for (int j = 0; j < NSP; ++j) {  // with the charged species
    double nu, Phi, Psi;
    const long long k2 = kg + (long long)j * v.ng;
    coulomb_colln(v, isp, j, ns[k2], Ts[k], Ts[k2], vs1[k], vs1[k2], nu, Phi, Psi, pairs);
    lo = lo + nu * Phi;
    pr = pr + ns[k] * ms * nu * Phi * vs1[k2];
  }
  const double ionpress = pres * pg;
  const double h1h2h3 = h1 * h2 * h3;
  const double geom = (vs2[k] * vs2[k] * h3 * dh2 + vs3[k] * vs3[k] * h2 * dh3) * ns[k] * ms / h1h2h3;
  const double e1f = (alt[c] < 100e3) ? 0.0 : E1[kg];
  pr = pr + ns[k] * v.qs[isp] * (e1f + epol) - ionpress - gq + geom + ns[k] * ms * g1[c];
  Pr[t] = pr;
  Lo[t] = lo;
}

}  // namespace gemr
