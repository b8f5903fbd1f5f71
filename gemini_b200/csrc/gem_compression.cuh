// The compression sub-step (app/main.f90:320-338): per-index bodies of its kernels.
//
//   artvisc  multifluid.f90:237-268 VNRicht_artvisc, xicon = 3 (multifluid.f90:43): Q of
//            every interior cell and species (0 for the electrons), from vs1 at x1 +- 1 as
//            the advection left it (ghosts included);
//   rk2_*    sources_mpi.f90:68-111 RK2_global_boundary on a single rank: zero-order hold
//            of vs1 along x1, then of vs1, vs2, vs3 along x2 and (non-periodic grids) x3 --
//            one pass per direction, each pass reading only cells it does not write;
//   cmp      multifluid.f90:274-302 compression with calculus/div.f90:110-200 div3D_curv_23:
//            the centred slab divergence of each species' velocity at an interior cell (the
//            three direction terms summed in order, each only when that dimension is longer
//            than 1, then divided by (h1*h2)*h3), and the half- and full-step updates of rhoes.
//
// Each body handles one linear index of its kernel's range, so the same code runs on the
// device (one thread per index) and, compiled for the host, over the whole range on a CPU.
// Every operation follows the reference's order; divisions are IEEE divisions.
#pragma once

#ifdef __CUDACC__
#define GEMC_HD __host__ __device__ __forceinline__
#else
#define GEMC_HD inline
#endif

namespace gemc {

constexpr int NSP = 7;

// The arrays the bodies read.  Ghosted blocks (-1:lx1+2,-1:lx2+2,-1:lx3+2) with strides
// s2, s3 and ng per species; metric factors h1..h3 in the same ghosted layout but with x3
// stride c3 (s3, or 0 when they do not vary along x3), or null on unit-metric grids (read as
// 1, which leaves every product exact); dx tables: backward differences dx(j), j = 0..l+2.
struct View {
  int lx1, lx2, lx3, flagper;
  long long s2, s3, ng, c3;
  const double *h1, *h2, *h3;
  const double *dx1, *dx2, *dx3;
  double ms[NSP], gm1[NSP];  // species masses, gamma - 1
};

GEMC_HD long long gix(const View& v, int i1, int i2, int i3) {
  return (long long)(i1 + 1) + v.s2 * (i2 + 1) + v.s3 * (i3 + 1);
}
GEMC_HD double hm(const double* h, const View& v, int i1, int i2, int i3) {
  return h ? h[(long long)(i1 + 1) + v.s2 * (i2 + 1) + v.c3 * (i3 + 1)] : 1.0;
}
GEMC_HD long long ncell(const View& v) { return (long long)v.lx1 * v.lx2 * v.lx3; }
// interior cell c (column-major 1:lx1,1:lx2,1:lx3) -> indices
GEMC_HD void cell_of(const View& v, long long c, int& i1, int& i2, int& i3) {
  i1 = (int)(c % v.lx1) + 1;
  const long long r = c / v.lx1;
  i2 = (int)(r % v.lx2) + 1;
  i3 = (int)(r / v.lx2) + 1;
}

// index t in [0, ncell*NSP): Q(t), t = s*ncell + cell
GEMC_HD void artvisc(const View& v, long long t, const double* ns, const double* vs1, double* Q) {
  const long long nc = ncell(v);
  const int s = (int)(t / nc);
  if (s >= NSP - 1) {
    Q[t] = 0.0;
    return;
  }
  int i1, i2, i3;
  cell_of(v, t - s * nc, i1, i2, i3);
  const double* u = vs1 + s * v.ng;
  const double vl = 0.5 * (u[gix(v, i1 - 1, i2, i3)] + u[gix(v, i1, i2, i3)]);
  const double vr = 0.5 * (u[gix(v, i1, i2, i3)] + u[gix(v, i1 + 1, i2, i3)]);
  const double dv = vr - vl;
  const double m = (dv < 0.0) ? dv : 0.0;
  Q[t] = ns[s * v.ng + gix(v, i1, i2, i3)] * v.ms[s] * 0.25 * 9.0 * (m * m);
}

// x1 pass, index t in [0, (lx2+4)*(lx3+4)*NSP): both x1 ghosts of vs1 of one (i2, i3, s)
GEMC_HD void rk2_x1(const View& v, long long t, double* vs1) {
  const int n2 = v.lx2 + 4, n3 = v.lx3 + 4;
  const int s = (int)(t / ((long long)n2 * n3));
  const long long r = t - (long long)s * n2 * n3;
  const int i2 = (int)(r % n2) - 1, i3 = (int)(r / n2) - 1;
  double* u = vs1 + s * v.ng;
  u[gix(v, 0, i2, i3)] = u[gix(v, 1, i2, i3)];
  u[gix(v, v.lx1 + 1, i2, i3)] = u[gix(v, v.lx1, i2, i3)];
}

// x2 pass, index t in [0, (lx1+4)*(lx3+4)*NSP*3): both x2 ghosts of one (i1, i3, s, component)
GEMC_HD void rk2_x2(const View& v, long long t, double* vs1, double* vs2, double* vs3) {
  const int n1 = v.lx1 + 4, n3 = v.lx3 + 4;
  const long long per = (long long)n1 * n3;
  const int q = (int)(t / per);  // component * NSP + species
  const long long r = t - q * per;
  const int i1 = (int)(r % n1) - 1, i3 = (int)(r / n1) - 1;
  const int c = q / NSP, s = q - c * NSP;
  double* u = ((c == 0) ? vs1 : (c == 1) ? vs2 : vs3) + s * v.ng;
  u[gix(v, i1, 0, i3)] = u[gix(v, i1, 1, i3)];
  u[gix(v, i1, v.lx2 + 1, i3)] = u[gix(v, i1, v.lx2, i3)];
}

// x3 pass (non-periodic grids), index t in [0, (lx1+4)*(lx2+4)*NSP*3)
GEMC_HD void rk2_x3(const View& v, long long t, double* vs1, double* vs2, double* vs3) {
  const int n1 = v.lx1 + 4, n2 = v.lx2 + 4;
  const long long per = (long long)n1 * n2;
  const int q = (int)(t / per);
  const long long r = t - q * per;
  const int i1 = (int)(r % n1) - 1, i2 = (int)(r / n1) - 1;
  const int c = q / NSP, s = q - c * NSP;
  double* u = ((c == 0) ? vs1 : (c == 1) ? vs2 : vs3) + s * v.ng;
  u[gix(v, i1, i2, 0)] = u[gix(v, i1, i2, 1)];
  u[gix(v, i1, i2, v.lx3 + 1)] = u[gix(v, i1, i2, v.lx3)];
}

// index t in [0, ncell*NSP): the compression update of rhoes at one interior cell and species
GEMC_HD void cmp(const View& v, long long t, const double* vs1, const double* vs2, const double* vs3,
                 const double* Q, double* rhoes, double dt) {
  const long long nc = ncell(v);
  const int s = (int)(t / nc);
  int i1, i2, i3;
  cell_of(v, t - s * nc, i1, i2, i3);
  const double* f1 = vs1 + s * v.ng;
  const double* f2 = vs2 + s * v.ng;
  const double* f3 = vs3 + s * v.ng;
  const double *h1 = v.h1, *h2 = v.h2, *h3 = v.h3;
  double d;
  {
    const double tp = hm(h2, v, i1 + 1, i2, i3) * hm(h3, v, i1 + 1, i2, i3) * f1[gix(v, i1 + 1, i2, i3)];
    const double tm = hm(h2, v, i1 - 1, i2, i3) * hm(h3, v, i1 - 1, i2, i3) * f1[gix(v, i1 - 1, i2, i3)];
    d = (tp - tm) / (v.dx1[i1 + 1] + v.dx1[i1]);
  }
  if (v.lx2 > 1) {
    const double tp = hm(h1, v, i1, i2 + 1, i3) * hm(h3, v, i1, i2 + 1, i3) * f2[gix(v, i1, i2 + 1, i3)];
    const double tm = hm(h1, v, i1, i2 - 1, i3) * hm(h3, v, i1, i2 - 1, i3) * f2[gix(v, i1, i2 - 1, i3)];
    d = d + (tp - tm) / (v.dx2[i2 + 1] + v.dx2[i2]);
  }
  if (v.lx3 > 1) {
    const double tp = hm(h1, v, i1, i2, i3 + 1) * hm(h2, v, i1, i2, i3 + 1) * f3[gix(v, i1, i2, i3 + 1)];
    const double tm = hm(h1, v, i1, i2, i3 - 1) * hm(h2, v, i1, i2, i3 - 1) * f3[gix(v, i1, i2, i3 - 1)];
    d = d + (tp - tm) / (v.dx3[i3 + 1] + v.dx3[i3]);
  }
  const double dv = d / (hm(h1, v, i1, i2, i3) * hm(h2, v, i1, i2, i3) * hm(h3, v, i1, i2, i3));
  const double q = Q[t];
  double* re = rhoes + s * v.ng + gix(v, i1, i2, i3);
  const double p = *re;
  const double half = p - dt / 2 * (p * v.gm1[s] + q) * dv;
  *re = p - dt * (half * v.gm1[s] + q) * dv;
}

}  // namespace gemc
