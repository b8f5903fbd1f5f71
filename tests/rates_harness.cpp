// TEST INFRASTRUCTURE -- not part of the product.  The per-cell bodies of the device
// production/loss rate kernels (gemini_b200/csrc/gem_rates.cuh), compiled for the host with
// the C library's math functions and run over every index of each kernel's range, so that
// their index arithmetic and their bits can be checked against the oracle on a CPU.
#include "../gemini_b200/csrc/gem_rates.cuh"

extern "C" {

struct HRView {
  int lx1, lx2, lx3;
  long long c3;
  const double *h1, *h2, *h3, *dx1;
  const double *ms, *qs, *gam;
  double pi;
};

static gemr::View mk(const HRView* h) {
  gemr::View v;
  v.lx1 = h->lx1;
  v.lx2 = h->lx2;
  v.lx3 = h->lx3;
  v.s2 = h->lx1 + 4;
  v.s3 = (long long)(h->lx1 + 4) * (h->lx2 + 4);
  v.ng = v.s3 * (h->lx3 + 4);
  v.c3 = h->c3;
  v.h1 = h->h1;
  v.yh1 = nullptr;  // read by the device build only
  v.h2 = h->h2;
  v.h3 = h->h3;
  v.dx1 = h->dx1;
  for (int s = 0; s < gemr::NSP; ++s) {
    v.ms[s] = h->ms[s];
    v.qs[s] = h->qs[s];
    v.gam[s] = h->gam[s];
  }
  v.pi = h->pi;
  return v;
}

void hr_continuity(const HRView* hv, const double* nn, const double* vn1, const double* vn2, const double* vn3,
                   const double* Tn, const double* fv, double* Pr, double* Lo) {
  const gemr::View v = mk(hv);
  const long long n = gemr::ncell(v);
  for (long long c = 0; c < n; ++c)
    gemr::continuity_cell(v, c, nn, vn1, vn2, vn3, Tn, fv, fv + 7 * v.ng, fv + 14 * v.ng, fv + 21 * v.ng,
                          fv + 28 * v.ng, Pr, Lo);
}

void hr_energy(const HRView* hv, const double* nn, const double* vn1, const double* vn2, const double* vn3,
               const double* Tn, const double* fv, double* Pr, double* Lo) {
  const gemr::View v = mk(hv);
  const long long n = gemr::ncell(v) * gemr::NSP;
  for (long long t = 0; t < n; ++t)
    gemr::energy_rate(v, t, nn, vn1, vn2, vn3, Tn, fv, fv + 7 * v.ng, fv + 14 * v.ng, fv + 21 * v.ng,
                      fv + 28 * v.ng, Pr, Lo);
}

void hr_momentum(const HRView* hv, const double* nn, const double* vn1, const double* Tn, const double* fv,
                 const double* E1, const double* Q, const double* alt, const double* g1, double* Pr, double* Lo) {
  const gemr::View v = mk(hv);
  const long long n = gemr::ncell(v) * gemr::NSP;
  for (long long t = 0; t < n; ++t)
    gemr::momentum_rate(v, t, nn, vn1, Tn, fv, fv + 7 * v.ng, fv + 14 * v.ng, fv + 21 * v.ng, fv + 28 * v.ng, E1,
                        Q, alt, g1, Pr, Lo);
}

// the symmetric part of one Coulomb pair (Teff**1.5, Phi, Psi): the device kernels evaluate
// it once per unordered pair and give both species the same bits
void hr_coulomb_pair(const HRView* hv, int isp, int isp2, double ts1, double ts2, double v1, double v2, double* out) {
  const gemr::View v = mk(hv);
  const gemr::CoulPair q = gemr::coulomb_pair(v, isp, isp2, ts1, ts2, v1, v2);
  out[0] = q.P;
  out[1] = q.Phi;
  out[2] = q.Psi;
}

}  // extern "C"
