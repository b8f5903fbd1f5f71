// TEST INFRASTRUCTURE -- not part of the product.  The per-cell bodies of the device
// source/loss solves (gemini_b200/csrc/gem_sources.cuh), compiled for the host and run over
// every cell of the ghosted block, so that their index arithmetic and their bits can be
// checked against the oracle on a CPU.
#include "../gemini_b200/csrc/gem_sources.cuh"

extern "C" {

struct HSView {
  int lx1, lx2, lx3;
  const double *ms, *qs, *gam;
};

static gems::View mk(const HSView* h) {
  gems::View v;
  v.lx1 = h->lx1;
  v.lx2 = h->lx2;
  v.lx3 = h->lx3;
  v.s2 = h->lx1 + 4;
  v.s3 = (long long)(h->lx1 + 4) * (h->lx2 + 4);
  v.ng = v.s3 * (h->lx3 + 4);
  for (int s = 0; s < gems::NSP; ++s) {
    v.ms[s] = h->ms[s];
    v.qs[s] = h->qs[s];
    v.gam[s] = h->gam[s];
  }
  return v;
}

void hs_mass(const HSView* hv, double dt, double* Pr, const double* Lo, const double* Prprecip, double* ns) {
  const gems::View v = mk(hv);
  for (long long k = 0; k < v.ng; ++k) gems::mass_cell(v, k, dt, Pr, Lo, Prprecip, ns);
}

void hs_momentum(const HSView* hv, double dt, const double* Pr, const double* Lo, const double* ns, double* rhovs1,
                 double* vs1) {
  const gems::View v = mk(hv);
  for (long long k = 0; k < v.ng; ++k) gems::momentum_cell(v, k, dt, Pr, Lo, ns, rhovs1, vs1);
}

void hs_energy(const HSView* hv, double dt, double* Pr, const double* Lo, const double* Qeprecip, double* rhoes,
               double* Ts, const double* ns) {
  const gems::View v = mk(hv);
  for (long long k = 0; k < v.ng; ++k) gems::energy_cell(v, k, dt, Pr, Lo, Qeprecip, rhoes, Ts, ns);
}

}  // extern "C"
