// Field-aligned heat diffusion with the reference's own band solve (multifluid.f90:309-342,
// collisions.f90:162-199, diffusion.f90:24-152, PDEparabolic.f90:19-346).
//
// One (x1 column, species) per thread.  The thread walks its column along x1 and, for each
// row, forms the thermal conductivity (thermal_conduct), the diffusion coefficients
// (diffusion_prep) and the TRBDF2 / backward-Euler band row in registers, with the
// reference's operation order.  Each band system is then factored and solved exactly as
// the reference's gbsv call does it (PDEparabolic.f90:142,216,337 -> gbsv.in.f90:90 ->
// LAPACK dgbsv with kl = ku = 2: dgbtrf -> dgbtf2, then dgbtrs -> dtbsv), specialised to
// the tridiagonal matrices the reference stores in that band:
//
//   dgbtf2 step j (rows j and j+1 are the only pivot candidates: row j+2 holds a structural
//   zero in column j, so its multiplier is 0 and its updates add zeros):
//     current row j = (p, q) in columns (j, j+1); original row j+1 = (s, d, e | r).
//     IDAMAX picks row j+1 only when |s| > |p| (ties keep row j).
//     no interchange: U(j) = (p, q, 0), recip = 1/p, m = recip*s (DSCAL), DGER:
//                     p' = d - m*q, q' = e;            dgbtrs: y(j) = b, b' = r - m*b
//     interchange:    U(j) = (s, d, e), recip = 1/s, m = recip*p, DGER:
//                     p' = q - m*d, q' = 0 - m*e;      dgbtrs: y(j) = r, b' = b - m*r
//   dtbsv (upper, no transpose, non-unit, bandwidth kl+ku), columns from the last:
//     x(i) = ((y(i) - x(i+2)*U(i,i+2)) - x(i+1)*U(i,i+1)) / U(i,i)
//   (the products with the zero fill entries U(i,i+3), U(i,i+4) subtract zeros).
// Every division is an IEEE division (or the exact reciprocal-corrected one for grid
// divisors), nothing is contracted, so the solution equals, bit for bit, the reference
// arithmetic with reference-BLAS semantics for IDAMAX/DSWAP/DSCAL/DGER/DTBSV.  The only
// departure: T**2.5 is the correctly rounded value (pow25), where the reference calls the
// C library's pow, which is not correctly rounded for about 1 argument in 1200.
//
// The forward elimination runs while the rows are formed; the factor rows U(i,i),
// U(i,i+1), U(i,i+2) and the eliminated right-hand side y(i) go to a per-thread scratch
// (4 doubles per row; the warp's 32 threads interleaved, so every scratch access is one
// coalesced 256-byte line), and the back substitution reads them back from the last row.
// The TRBDF2 half-step solution replaces y(i) in place and the BDF2 stage re-forms the
// coefficients from T and n.
//
// The body is written once for a column accessor, so the same code runs on the device
// (thread per column) and, compiled for the host, over every column on a CPU.
#pragma once

#ifdef __CUDACC__
#define GEMD_HD __host__ __device__ __forceinline__
#else
#define GEMD_HD inline
#include <cmath>
#include <cstring>
#endif

namespace gemd {

constexpr int NSP = 7;
constexpr double KB = 1.38064852e-23;     // phys_consts.in.f90:24
constexpr double ELCHRG = 1.60217662e-19;  // phys_consts.in.f90:25
constexpr double MINDENSDIV = 1.0e-5;      // phys_consts.in.f90:84

GEMD_HD double fma_rn(double a, double b, double c) {
#ifdef __CUDA_ARCH__
  return __fma_rn(a, b, c);
#else
  return std::fma(a, b, c);
#endif
}

GEMD_HD unsigned hi_abs(double x) {
#ifdef __CUDA_ARCH__
  return (unsigned)__double2hiint(x) & 0x7fffffffu;
#else
  unsigned long long u;
  std::memcpy(&u, &x, 8);
  return (unsigned)(u >> 32) & 0x7fffffffu;
#endif
}

GEMD_HD double sqrt_rn(double x) {
#ifdef __CUDA_ARCH__
  return sqrt(x);
#else
  return std::sqrt(x);
#endif
}

#ifdef __CUDA_ARCH__
__device__ __noinline__ double div_rn_slow(double a, double b) { return a / b; }
#else
inline double div_rn_slow(double a, double b) { return a / b; }
#endif

// a/b for a divisor with a precomputed correctly rounded reciprocal y = RN(1/b): q0 = RN(a*y),
// one exact remainder r = a - b*q0 and q = RN(q0 + r*y), which is the IEEE quotient RN(a/b)
// whenever |a| is in (2^-500, 2^500) and |y| in [2^-400, 2^400] (Markstein); a zero numerator
// gives the correctly signed zero; anything else takes the IEEE division.
GEMD_HD double qdiv(double a, double b, double y) {
  const double q0 = a * y;
  const double r = fma_rn(-q0, b, a);
  const double q1 = fma_rn(r, y, q0);
  const unsigned ha = hi_abs(a), hy = hi_abs(y);
  if ((ha - (523u << 20) < (1000u << 20)) & (hy - (623u << 20) < (800u << 20))) return q1;
  if (a == 0.0 && (hy - (623u << 20) < (800u << 20))) return q0;
  return div_rn_slow(a, b);
}

GEMD_HD double fmax_f(double a, double b) { return (a > b) ? a : b; }
GEMD_HD double fabs_f(double a) { return (a < 0.0) ? -a : a; }

// x**2.5 as x*x*sqrt(x) in double-double (fma for the exact product errors), rounded once:
// the correctly rounded value except in vanishingly rare near-halfway cases.
GEMD_HD double pow25(double x) {
  if (!(x > 0.0)) {
#ifdef __CUDA_ARCH__
    return pow(x, 2.5);
#else
    return std::pow(x, 2.5);
#endif
  }
  const double s = sqrt_rn(x);
  const double es = fma_rn(-s, s, x);
  const double sl = es / (2.0 * s);
  const double x2 = x * x;
  const double x2l = fma_rn(x, x, -x2);
  const double p = x2 * s;
  const double pl = fma_rn(x2, s, -p);
  return p + (pl + (x2 * sl + x2l * s));
}

// Per-column constants of one solve.
struct LuK {
  int n;          // lx1
  int s;          // species (6 = electrons)
  double dt;
  double tmin, tmax;  // Dirichlet values of rows 1 and lx1 (diffusion.f90:54-79)
  double c0;          // (gamma_s - 1)/kB
  double tcoef;       // ions: thermal_coeff(s) (collisions.f90:51-53)
};

// thermal_conduct + diffusion_prep of interior cell i (collisions.f90:162-199,
// diffusion.f90:24-52; A = E = 0): C = (gamma-1)/kB / max(n,1e-5) / (h1 h2 h3),
// D = lambda h2 h3 / h1, B = C beta / h1 (electrons; 0 for the ions).
template <bool UNIT, bool ELEC, class Acc>
GEMD_HD void cell_coef(const Acc& a, const LuK& k, int i, double& C, double& D, double& B) {
  const double T = a.T(i), nv = a.n(i);
  double h1 = 1.0, h2 = 1.0, h3 = 1.0, yh1 = 1.0, ha1 = 1.0, yha1 = 1.0;
  if (!UNIT) a.metrics(i, h1, h2, h3, yh1, ha1, yha1);
  const double T25 = pow25(T);
  double lam, Bc = 0.0;
  if (!ELEC) {
    lam = k.tcoef * T25;
  } else {
    double n1, n2, n3, j1;
    a.neutrals(i, n1, n2, n3, j1);
    const double sq = sqrt_rn(T);
    const double X = n1 * 1.1e-16 * (1 + 5.7e-4 * T) + n2 * 2.82e-17 * sq * (1 - 1.21e-4 * T) +
                     n3 * 2.2e-16 * (1 + 3.6e-2 * sq);
    lam = ELCHRG * 100 * 7.7e5 * T25 / (1 + 3.22e4 * (T * T) / nv * X);
    Bc = 5.0 / 2 * KB / ELCHRG * j1;  // beta (collisions.f90:197)
  }
  C = qdiv(k.c0 / fmax_f(nv, MINDENSDIV), ha1, yha1);
  D = qdiv(lam * h2 * h3, h1, yh1);
  B = ELEC ? qdiv(C * Bc, h1, yh1) : 0.0;
}

// The band rows (PDEparabolic.f90:66-136 TR, 150-210 BDF2, 250-319 backward Euler) from the
// per-row conduction factors q- = C Dh(i)/dx1i/dx1(i), q+ = C Dh(i+1)/dx1i/dx1(i+1) and the
// advection factor bq = B/(dx1(i+1)+dx1(i)).
enum Stage { ST_TR = 0, ST_BDF2 = 1, ST_BE = 2 };

struct LuState {
  double p, q, b;  // current (partially eliminated) row j and its right-hand side
};

// One dgbtf2/dgbtrs step with the original row j+1 = (s, d, e | r); writes U(j) and y(j).
template <class Acc>
GEMD_HD void lu_step(const Acc& a, int j, LuState& st, double s, double d, double e, double r) {
  double u0, u1, u2, y, m;
  if (fabs_f(s) > fabs_f(st.p)) {  // IDAMAX takes row j+1: interchange (DSWAP)
    u0 = s;
    u1 = d;
    u2 = e;
    y = r;
    m = (1.0 / s) * st.p;  // DSCAL(1/pivot)
    const double p1 = st.q - m * d;
    st.q = 0.0 - m * e;
    st.p = p1;
    st.b = st.b - m * r;
  } else {
    u0 = st.p;
    u1 = st.q;
    u2 = 0.0;
    y = st.b;
    m = (1.0 / st.p) * s;
    st.p = d - m * st.q;
    st.q = e;
    st.b = r - m * st.b;
  }
  a.S(j, 0) = u0;
  a.S(j, 1) = u1;
  a.S(j, 2) = u2;
  a.S(j, 3) = y;
}

// Forward pass of one stage over rows 1..n: forms every band row, eliminates, stores the
// factor rows.  STG = ST_BDF2 reads the TR solution from the y slots (row i's slot is read
// before row i's factor row is written).
template <bool UNIT, bool ELEC, int STG, class Acc>
GEMD_HD void lu_forward(const Acc& a, const LuK& k) {
  const int n = k.n;
  const double dt = k.dt;
  const double dt2 = dt / 2, ydt2 = 1 / (dt / 2);
  const double dt3 = dt / 3, ydt3 = 1 / (dt / 3);
  const double ydt = 1 / dt;
  LuState st{1.0, 0.0, k.tmin};  // row 1: identity, right-hand side Tsminx1
  // sliding window over cells: D(i-1), D(i), C(i), B(i) and T(i-1), T(i)
  double Cc, Dc, Bcur;
  cell_coef<UNIT, ELEC>(a, k, 1, Cc, Dc, Bcur);
  double Dm = Dc;  // D(1), becomes D(i-1) for i = 2
  cell_coef<UNIT, ELEC>(a, k, 2, Cc, Dc, Bcur);
  double Tm = a.T(1), Tc = a.T(2);
  for (int j = 1; j < n; ++j) {
    const int i = j + 1;  // the row brought in
    double s, d, e, r;
    if (i == n) {
      s = 0.0;
      d = 1.0;
      e = 0.0;
      r = k.tmax;
    } else {
      double Cn, Dn, Bn;
      cell_coef<UNIT, ELEC>(a, k, i + 1, Cn, Dn, Bn);
      const double Tp = a.T(i + 1);
      const double Dhm = 0.5 * (Dm + Dc), Dhp = 0.5 * (Dc + Dn);  // PDEparabolic.f90:49
      const double qm = qdiv(qdiv(Cc * Dhm, a.dxi(i), a.ydxi(i)), a.dx(i), a.ydx(i));
      const double qp = qdiv(qdiv(Cc * Dhp, a.dxi(i), a.ydxi(i)), a.dx(i + 1), a.ydx(i + 1));
      const double bq = ELEC ? qdiv(Bcur, a.dxs(i), a.ydxs(i)) : 0.0;
      if (STG == ST_TR) {
        s = -(qm / 2) + bq / 2;
        d = ydt2 + qp / 2 + qm / 2;
        e = -(qp / 2) - bq / 2;
        const double Pd = qp / 2 + qm / 2;
        r = qdiv(Tc, dt2, ydt2) - s * Tm - Pd * Tc - e * Tp;
      } else if (STG == ST_BDF2) {
        s = -qm + bq;
        d = ydt3 + qp + qm;
        e = -qp - bq;
        const double tr = a.S(i, 3);
        r = -qdiv(1 / 3.0 * Tc, dt3, ydt3) + qdiv(4 / 3.0 * tr, dt3, ydt3);
      } else {
        s = -qm + bq;
        d = ydt + qp + qm;
        e = -qp - bq;
        r = qdiv(Tc, dt, ydt);
      }
      Dm = Dc;
      Dc = Dn;
      Cc = Cn;
      Bcur = Bn;
      Tm = Tc;
      Tc = Tp;
    }
    lu_step(a, j, st, s, d, e, r);
  }
  a.S(n, 0) = st.p;
  a.S(n, 1) = 0.0;
  a.S(n, 2) = 0.0;
  a.S(n, 3) = st.b;
}

// dtbsv back substitution; OUT(i, x) receives the solution from row n down to row 1.
template <class Acc, class Out>
GEMD_HD void lu_backward(const Acc& a, int n, Out out) {
  double x2 = 0.0;                   // x(i+2)
  double x1 = a.S(n, 3) / a.S(n, 0);  // x(n)
  out(n, x1);
  for (int i = n - 1; i >= 1; --i) {
    double x = a.S(i, 3);
    if (i <= n - 2) x = x - x2 * a.S(i, 2);
    x = x - x1 * a.S(i, 1);
    x = x / a.S(i, 0);
    out(i, x);
    x2 = x1;
    x1 = x;
  }
}

// The whole solve of one (column, species): TRBDF2 (solver 2) or backward Euler (solver 1).
// STORE(i, T) receives the new temperature of row i (before the max(T,100) floor).
template <bool UNIT, bool ELEC, class Acc, class Store>
GEMD_HD void lu_column(const Acc& a, const LuK& k, int solver, Store store) {
  const int n = k.n;
  if (solver == 2) {
    lu_forward<UNIT, ELEC, ST_TR>(a, k);
    lu_backward(a, n, [&](int i, double x) { a.S(i, 3) = x; });  // TR solution into y(i)
    lu_forward<UNIT, ELEC, ST_BDF2>(a, k);
  } else {
    lu_forward<UNIT, ELEC, ST_BE>(a, k);
  }
  lu_backward(a, n, store);
}

}  // namespace gemd
