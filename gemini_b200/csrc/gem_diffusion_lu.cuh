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
// (LU_ROW slots per row; the warp's 32 threads interleaved, so every scratch access is one
// coalesced 256-byte line), and the back substitution reads them back from the last row.
// The TRBDF2 half-step solution replaces y(i) in place; the per-row conduction factors are
// formed once, in the TR stage, and kept in the scratch for the BDF2 stage.
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

// qdiv for a divisor whose reciprocal comes from a grid table: gem_grid_create rejects grids
// with a tabulated reciprocal outside [2^-400, 2^400], so only the numerator is range-checked.
GEMD_HD double qdiv_t(double a, double b, double y) {
  const double q0 = a * y;
  const double r = fma_rn(-q0, b, a);
  const double q1 = fma_rn(r, y, q0);
  if (hi_abs(a) - (523u << 20) < (1000u << 20)) return q1;
  if (a == 0.0) return q0;
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

// Correctly rounded 1/x (the reference's ONE / AB(KV+1,J) in DSCAL).
GEMD_HD double rcp_rn(double x) {
#ifdef __CUDA_ARCH__
  return __drcp_rn(x);
#else
  return 1.0 / x;
#endif
}

// The streaming inputs of one interior cell: state values and, for the electrons, the
// neutral densities and J1.  Loaded ahead of use (the metric factors, small tables that the
// warp's lanes share, are read when the coefficients are formed).
struct CellIn {
  double T, n, n1, n2, n3, j1;
};

template <bool ELEC, class Acc>
GEMD_HD CellIn load_cell(const Acc& a, int i) {
  CellIn c;
  c.T = a.T(i);
  c.n = a.n(i);
  if (ELEC) {
    a.neutrals(i, c.n1, c.n2, c.n3, c.j1);
  } else {
    c.n1 = c.n2 = c.n3 = c.j1 = 0.0;
  }
  return c;
}

// thermal_conduct + diffusion_prep of interior cell i (collisions.f90:162-199,
// diffusion.f90:24-52; A = E = 0): C = (gamma-1)/kB / max(n,1e-5) / (h1 h2 h3),
// D = lambda h2 h3 / h1, B = C beta / h1 (electrons; 0 for the ions).
template <bool UNIT, bool ELEC, class Acc>
GEMD_HD void cell_coef(const Acc& a, const LuK& k, int i, const CellIn& c, double& C, double& D, double& B) {
  const double T = c.T, nv = c.n;
  double h1 = 1.0, h2 = 1.0, h3 = 1.0, yh1 = 1.0, ha1 = 1.0, yha1 = 1.0;
  if (!UNIT) a.metrics(i, h1, h2, h3, yh1, ha1, yha1);
  const double T25 = pow25(T);
  double lam, Bc = 0.0;
  if (!ELEC) {
    lam = k.tcoef * T25;
  } else {
    const double sq = sqrt_rn(T);
    const double X = c.n1 * 1.1e-16 * (1 + 5.7e-4 * T) + c.n2 * 2.82e-17 * sq * (1 - 1.21e-4 * T) +
                     c.n3 * 2.2e-16 * (1 + 3.6e-2 * sq);
    lam = ELCHRG * 100 * 7.7e5 * T25 / (1 + 3.22e4 * (T * T) / nv * X);
    Bc = 5.0 / 2 * KB / ELCHRG * c.j1;  // beta (collisions.f90:197)
  }
  C = qdiv_t(k.c0 / fmax_f(nv, MINDENSDIV), ha1, yha1);
  D = qdiv_t(lam * h2 * h3, h1, yh1);
  B = ELEC ? qdiv_t(C * Bc, h1, yh1) : 0.0;
}

// The band rows (PDEparabolic.f90:66-136 TR, 150-210 BDF2, 250-319 backward Euler) from the
// per-row conduction factors q- = C Dh(i)/dx1i/dx1(i), q+ = C Dh(i+1)/dx1i/dx1(i+1) and the
// advection factor bq = B/(dx1(i+1)+dx1(i)).
enum Stage { ST_TR = 0, ST_BDF2 = 1, ST_BE = 2 };

struct LuState {
  double p, q, b;  // current (partially eliminated) row j and its right-hand side
};

// One dgbtf2/dgbtrs step with the original row j+1 = (s, d, e | r); writes U(j) and y(j).
// U(j,j+2) is nonzero only on interchanged rows, so it is stored only from the first
// interchange of the column on (fs: that row, n+1 while there is none); the back
// substitution uses +0.0, the value an uninterchanged row holds, for the rows before it.
template <class Acc>
GEMD_HD void lu_step(const Acc& a, int j, LuState& st, int& fs, double s, double d, double e, double r) {
  double u0, u1, u2, y, m;
  if (fabs_f(s) > fabs_f(st.p)) {  // IDAMAX takes row j+1: interchange (DSWAP)
    if (fs > j) fs = j;
    u0 = s;
    u1 = d;
    u2 = e;
    y = r;
    m = rcp_rn(s) * st.p;  // DSCAL(1/pivot)
    const double p1 = st.q - m * d;
    st.q = 0.0 - m * e;
    st.p = p1;
    st.b = st.b - m * r;
  } else {
    u0 = st.p;
    u1 = st.q;
    u2 = 0.0;
    y = st.b;
    m = rcp_rn(st.p) * s;
    st.p = d - m * st.q;
    st.q = e;
    st.b = r - m * st.b;
  }
  a.sst(j, 0, u0);
  a.sst(j, 1, u1);
  if (j >= fs) a.sst(j, 2, u2);
  a.sst(j, 3, y);
}

// Scratch slots of a row: the factor row U(i,i), U(i,i+1), U(i,i+2) and y(i) (slots 0-3;
// the TR solution replaces y(i)), and for TRBDF2 the conduction/advection factors q-, q+,
// bq of the row (slots 4-6), formed once for both stages.
constexpr int LU_ROW = 8;  // scratch slots per row

// Forward pass of the first stage (TR half step, or the backward-Euler step) over rows
// 1..n: forms every band row from T and n, eliminates, stores the factor rows (and, for
// TR, the row factors for the BDF2 stage); returns the first interchanged row (n+1: none).  Software-pipelined: each iteration forms row
// i+1 (conductivities, factors, band row -- independent of the elimination) next to the
// elimination step of row i, and the cell inputs are loaded two rows ahead of their use.
struct BandRow {
  double s, d, e, r;  // sub-diagonal, diagonal, super-diagonal, right-hand side
};

template <bool UNIT, bool ELEC, int STG, class Acc>
GEMD_HD int lu_forward_first(const Acc& a, const LuK& k) {
  const int n = k.n;
  const double dt = k.dt;
  const double dt2 = dt / 2, ydt2 = 1 / (dt / 2);
  const double ydt = 1 / dt;
  auto cell = [&](int i) { return load_cell<ELEC>(a, i < n ? i : n); };
  const CellIn c1 = cell(1), c2 = cell(2);
  CellIn cA = cell(3), cB = cell(4);  // cells i+1, i+2 of the next row formed (i = 2)
  // sliding window over cells: D(i-1), D(i), C(i), B(i) and T(i-1), T(i)
  double Cc, Dc, Bcur, Dm;
  cell_coef<UNIT, ELEC>(a, k, 1, c1, Cc, Dm, Bcur);  // D(1)
  cell_coef<UNIT, ELEC>(a, k, 2, c2, Cc, Dc, Bcur);
  double Tm = c1.T, Tc = c2.T;
  // forms row i (2 <= i <= n) and advances the window
  auto form = [&](int i) -> BandRow {
    BandRow w;
    if (i == n) {
      w.s = 0.0;
      w.d = 1.0;
      w.e = 0.0;
      w.r = k.tmax;
      return w;
    }
    const CellIn cn = cA;  // cell i+1
    cA = cB;
    cB = cell(i + 3);
    double Cn, Dn, Bn;
    cell_coef<UNIT, ELEC>(a, k, i + 1, cn, Cn, Dn, Bn);
    const double Tp = cn.T;
    const double Dhm = 0.5 * (Dm + Dc), Dhp = 0.5 * (Dc + Dn);  // PDEparabolic.f90:49
    const double qm = qdiv_t(qdiv_t(Cc * Dhm, a.dxi(i), a.ydxi(i)), a.dx(i), a.ydx(i));
    const double qp = qdiv_t(qdiv_t(Cc * Dhp, a.dxi(i), a.ydxi(i)), a.dx(i + 1), a.ydx(i + 1));
    const double bq = ELEC ? qdiv_t(Bcur, a.dxs(i), a.ydxs(i)) : 0.0;
    if (STG == ST_TR) {
      a.sst(i, 4, qm);
      a.sst(i, 5, qp);
      if (ELEC) a.sst(i, 6, bq);
      w.s = -(qm / 2) + bq / 2;
      w.d = ydt2 + qp / 2 + qm / 2;
      w.e = -(qp / 2) - bq / 2;
      const double Pd = qp / 2 + qm / 2;
      w.r = qdiv(Tc, dt2, ydt2) - w.s * Tm - Pd * Tc - w.e * Tp;
    } else {
      w.s = -qm + bq;
      w.d = ydt + qp + qm;
      w.e = -qp - bq;
      w.r = qdiv(Tc, dt, ydt);
    }
    Dm = Dc;
    Dc = Dn;
    Cc = Cn;
    Bcur = Bn;
    Tm = Tc;
    Tc = Tp;
    return w;
  };
  LuState st{1.0, 0.0, k.tmin};  // row 1: identity, right-hand side Tsminx1
  int fs = n + 1;
  BandRow w = form(2);
  for (int j = 1; j < n; ++j) {
    const BandRow cur = w;  // row j+1
    if (j + 2 <= n) w = form(j + 2);
    lu_step(a, j, st, fs, cur.s, cur.d, cur.e, cur.r);
  }
  a.sst(n, 0, st.p);  // U(n,n+1), U(n,n+2) lie outside the matrix: never read
  a.sst(n, 3, st.b);
  return fs;
}

// Forward pass of the BDF2 stage: the rows from the stored q-, q+, bq, the TR solution in
// y(i) and T (all loaded two rows ahead; row r's slots 0-3 are rewritten only when row r+1
// is brought in, after row r's TR value was read).  Returns the first interchanged row.
template <bool ELEC, class Acc>
GEMD_HD int lu_forward_bdf2(const Acc& a, const LuK& k) {
  const int n = k.n;
  const double dt3 = k.dt / 3, ydt3 = 1 / (k.dt / 3);
  struct RowIn {
    double qm, qp, bq, tr, T;
  };
  auto rin = [&](int i) {
    const int c = i < n - 1 ? i : n - 1;
    RowIn v;
    v.qm = a.sld(c, 4);
    v.qp = a.sld(c, 5);
    v.bq = ELEC ? a.sld(c, 6) : 0.0;
    v.tr = a.sld(c, 3);
    v.T = a.T(c);
    return v;
  };
  RowIn rA = rin(2), rB = rin(3);  // rows i, i+1 of the next row formed (i = 2)
  auto form = [&](int i) -> BandRow {
    BandRow w;
    if (i == n) {
      w.s = 0.0;
      w.d = 1.0;
      w.e = 0.0;
      w.r = k.tmax;
      return w;
    }
    const RowIn v = rA;
    rA = rB;
    rB = rin(i + 2);
    w.s = -v.qm + v.bq;
    w.d = ydt3 + v.qp + v.qm;
    w.e = -v.qp - v.bq;
    w.r = -qdiv(1 / 3.0 * v.T, dt3, ydt3) + qdiv(4 / 3.0 * v.tr, dt3, ydt3);
    return w;
  };
  LuState st{1.0, 0.0, k.tmin};
  int fs = n + 1;
  BandRow w = form(2);
  for (int j = 1; j < n; ++j) {
    const BandRow cur = w;  // row j+1
    if (j + 2 <= n) w = form(j + 2);
    lu_step(a, j, st, fs, cur.s, cur.d, cur.e, cur.r);
  }
  a.sst(n, 0, st.p);
  a.sst(n, 3, st.b);
  return fs;
}

// dtbsv back substitution from row n down to row 1 (fs: the forward pass's first
// interchanged row; U(i,i+2) = +0.0 above it).  OUT.pre(i) loads what OUT needs for row i;
// OUT(i, x, pre) receives the solution.  Factor rows and OUT's inputs are loaded
// GEMD_BWD_DEPTH rows ahead of their use.
struct RowF {
  double u0, u1, u2, y;
};
#ifndef GEMD_BWD_DEPTH
#define GEMD_BWD_DEPTH 4
#endif

template <class Acc, class Out>
GEMD_HD void lu_backward(const Acc& a, int n, int fs, const Out& out) {
  using Pre = decltype(out.pre(1));
  auto row = [&](int i) {
    RowF r;
    r.u0 = a.sld(i, 0);
    r.u1 = i < n ? a.sld(i, 1) : 0.0;
    r.u2 = (i >= fs && i < n - 1) ? a.sld(i, 2) : 0.0;
    r.y = a.sld(i, 3);
    return r;
  };
  constexpr int DP = GEMD_BWD_DEPTH;
  RowF W[DP];
  Pre P[DP];
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
  for (int q = 0; q < DP; ++q) {
    const int i = n - q >= 1 ? n - q : 1;
    W[q] = row(i);
    P[q] = out.pre(i);
  }
  double x1 = 0.0, x2 = 0.0;  // x(i+1), x(i+2)
  for (int i0 = n; i0 >= 1; i0 -= DP) {
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
    for (int q = 0; q < DP; ++q) {
      const int i = i0 - q;
      if (i >= 1) {
        const RowF r = W[q];
        const Pre pr = P[q];
        if (i - DP >= 1) {
          W[q] = row(i - DP);
          P[q] = out.pre(i - DP);
        }
        double x = r.y;
        if (i <= n - 2) x = x - x2 * r.u2;
        if (i <= n - 1) x = x - x1 * r.u1;
        x = x / r.u0;
        out(i, x, pr);
        x2 = x1;
        x1 = x;
      }
    }
  }
}

// OUT for the TR stage: the half-step solution replaces y(i).
template <class Acc>
struct StoreTR {
  const Acc& a;
  GEMD_HD double pre(int) const { return 0.0; }
  GEMD_HD void operator()(int i, double x, double) const { a.sst(i, 3, x); }
};

// The whole solve of one (column, species): TRBDF2 (solver 2) or backward Euler (solver 1).
// OUT receives the new temperature of each row (before the max(T,100) floor).
template <bool UNIT, bool ELEC, class Acc, class Out>
GEMD_HD void lu_column(const Acc& a, const LuK& k, int solver, const Out& out) {
  const int n = k.n;
  int fs;
  if (solver == 2) {
    fs = lu_forward_first<UNIT, ELEC, ST_TR>(a, k);
    lu_backward(a, n, fs, StoreTR<Acc>{a});
    fs = lu_forward_bdf2<ELEC>(a, k);
  } else {
    fs = lu_forward_first<UNIT, ELEC, ST_BE>(a, k);
  }
  lu_backward(a, n, fs, out);
}

}  // namespace gemd
