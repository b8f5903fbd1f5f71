// TEST INFRASTRUCTURE -- not part of the product.  The per-column body of the device
// diffusion kernel k_diffusion_lu (gemini_b200/csrc/gem_diffusion_lu.cuh), compiled for the
// host and run over every (column, species) of a grid, so that its arithmetic can be checked
// bit for bit against the oracle's restatement of the reference's LAPACK band solve on a CPU.
// The metric tables are built as gem_grid_create builds the device's: h1*h2*h3 left to right,
// correctly rounded reciprocals, dx(j)+dx(j+1).
#include <vector>

#include "../gemini_b200/csrc/gem_diffusion_lu.cuh"

namespace {

struct HostAcc {
  const double *Tc, *nc;
  const double *h1, *h2, *h3, *yh1, *ha1, *yha1;
  const double *n1, *n2, *n3, *J1c;
  const double *dx_, *ydx_, *dxs_, *ydxs_, *dxi_, *ydxi_;
  double* sc;
  double T(int i) const { return Tc[i]; }
  double n(int i) const { return nc[i]; }
  void metrics(int i, double& a1, double& a2, double& a3, double& y1, double& ha, double& yha) const {
    a1 = h1[i];
    a2 = h2[i];
    a3 = h3[i];
    y1 = yh1[i];
    ha = ha1[i];
    yha = yha1[i];
  }
  void neutrals(int i, double& a, double& b, double& c, double& j) const {
    a = n1[i];
    b = n2[i];
    c = n3[i];
    j = J1c[i];
  }
  double dx(int i) const { return dx_[i]; }
  double ydx(int i) const { return ydx_[i]; }
  double dxi(int i) const { return dxi_[i - 1]; }
  double ydxi(int i) const { return ydxi_[i - 1]; }
  double dxs(int i) const { return dxs_[i]; }
  double ydxs(int i) const { return ydxs_[i]; }
  double sld(int i, int k) const { return sc[(i - 1) * gemd::LU_ROW + k]; }
  void sst(int i, int k, double v) const { sc[(i - 1) * gemd::LU_ROW + k] = v; }
};

struct HostStore {
  double* Tout;
  double pre(int) const { return 0.0; }
  void operator()(int i, double x, double) const { Tout[i] = gemd::fmax_f(x, 100.0); }
};

const double c_gammas[7] = {5.0 / 3, 7.0 / 5, 7.0 / 5, 7.0 / 5, 5.0 / 3, 5.0 / 3, 5.0 / 3};
const double c_tcoef[6] = {(double)0.1019e-12f, (double)0.0747e-12f, (double)0.0754e-12f,
                           (double)0.0701e-12f, (double)0.1068e-12f, (double)0.3986e-12f};

}  // namespace

extern "C" {

struct HDiff {
  int lx1, lx2, lx3, gridflag, solver, unit;
  double dt, Teinf;
  const double *h1, *h2, *h3;  // ghosted metric factors (ignored when unit)
  const double *dx1, *dx1i;    // dx1(0:lx1+2), dx1i(1:lx1)
  const double* Ttop;          // optional per-column exospheric temperature (x2 fastest)
};

// energy_diffusion (non-fused form of the device kernel): each interior column and species
// solved in place in Ts; the x1 ghost layers receive max(Dirichlet value, 100).
int hd_energy_diffusion(const HDiff* h, const double* ns, double* Ts, const double* J1, const double* nn,
                        const double* Tn) {
  const int lx1 = h->lx1, lx2 = h->lx2, lx3 = h->lx3;
  if (lx1 < 4) return -1;
  const long long s2 = lx1 + 4, s3 = s2 * (lx2 + 4), ng = s3 * (lx3 + 4);
  const long long nc = (long long)lx1 * lx2 * lx3;
  std::vector<double> ones(ng, 1.0), yh1(ng), ha1(ng), yha1(ng);
  const double* H1 = h->unit ? ones.data() : h->h1;
  const double* H2 = h->unit ? ones.data() : h->h2;
  const double* H3 = h->unit ? ones.data() : h->h3;
  for (long long q = 0; q < ng; ++q) {
    yh1[q] = 1.0 / H1[q];
    ha1[q] = H1[q] * H2[q] * H3[q];
    yha1[q] = 1.0 / ha1[q];
  }
  std::vector<double> ydx(lx1 + 3), dxs(lx1 + 2), ydxs(lx1 + 2), ydxi(lx1);
  for (int j = 0; j < lx1 + 3; ++j) ydx[j] = 1.0 / h->dx1[j];
  for (int j = 0; j < lx1 + 2; ++j) {
    dxs[j] = h->dx1[j] + h->dx1[j + 1];
    ydxs[j] = 1.0 / dxs[j];
  }
  for (int j = 0; j < lx1; ++j) ydxi[j] = 1.0 / h->dx1i[j];
  std::vector<double> scr((size_t)lx1 * gemd::LU_ROW);
  for (int s = 0; s < 7; ++s)
    for (int i3 = 1; i3 <= lx3; ++i3)
      for (int i2 = 1; i2 <= lx2; ++i2) {
        const long long m0 = 1 + s2 * (i2 + 1) + s3 * (i3 + 1);  // cell (0, i2, i3)
        const long long q0 = (long long)lx1 * ((i2 - 1) + (long long)lx2 * (i3 - 1)) - 1;
        HostAcc a;
        a.Tc = Ts + s * ng + m0;
        a.nc = ns + s * ng + m0;
        a.h1 = H1 + m0;
        a.h2 = H2 + m0;
        a.h3 = H3 + m0;
        a.yh1 = yh1.data() + m0;
        a.ha1 = ha1.data() + m0;
        a.yha1 = yha1.data() + m0;
        a.n1 = nn + q0;
        a.n2 = nn + nc + q0;
        a.n3 = nn + 2 * nc + q0;
        a.J1c = J1 + m0;
        a.dx_ = h->dx1;
        a.ydx_ = ydx.data();
        a.dxs_ = dxs.data();
        a.ydxs_ = ydxs.data();
        a.dxi_ = h->dx1i;
        a.ydxi_ = ydxi.data();
        a.sc = scr.data();
        const double tn1 = Tn[q0 + 1], tnl = Tn[q0 + lx1];
        const double tinf = h->Ttop ? h->Ttop[(i2 - 1) + (long long)lx2 * (i3 - 1)] : h->Teinf;
        gemd::LuK k;
        k.n = lx1;
        k.s = s;
        k.dt = h->dt;
        k.tmin = h->gridflag == 1 ? tinf : tn1;
        k.tmax = h->gridflag == 2 ? tinf : tnl;
        k.c0 = (c_gammas[s] - 1.0) / gemd::KB;
        k.tcoef = s < 6 ? c_tcoef[s] : 0.0;
        double* Tout = Ts + s * ng + m0;
        const HostStore store{Tout};
        if (h->unit) {
          if (s == 6) gemd::lu_column<true, true>(a, k, h->solver, store);
          else gemd::lu_column<true, false>(a, k, h->solver, store);
        } else {
          if (s == 6) gemd::lu_column<false, true>(a, k, h->solver, store);
          else gemd::lu_column<false, false>(a, k, h->solver, store);
        }
        Tout[0] = gemd::fmax_f(k.tmin, 100.0);
        Tout[lx1 + 1] = gemd::fmax_f(k.tmax, 100.0);
      }
  return 0;
}

}  // extern "C"
