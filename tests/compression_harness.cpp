// TEST INFRASTRUCTURE -- not part of the product.  The per-index bodies of the device
// compression kernels (gemini_b200/csrc/gem_compression.cuh), compiled for the host and run
// over every index of each kernel's range, so that their index arithmetic and their bits can
// be checked against the oracle on a CPU.
#include "../gemini_b200/csrc/gem_compression.cuh"

extern "C" {

struct HView {
  int lx1, lx2, lx3, flagper;
  long long c3;
  const double *h1, *h2, *h3, *dx1, *dx2, *dx3;
  const double *ms, *gm1;
};

static gemc::View mk(const HView* h) {
  gemc::View v;
  v.lx1 = h->lx1;
  v.lx2 = h->lx2;
  v.lx3 = h->lx3;
  v.flagper = h->flagper;
  v.s2 = h->lx1 + 4;
  v.s3 = (long long)(h->lx1 + 4) * (h->lx2 + 4);
  v.ng = v.s3 * (h->lx3 + 4);
  v.c3 = h->c3;
  v.h1 = h->h1;
  v.h2 = h->h2;
  v.h3 = h->h3;
  v.dx1 = h->dx1;
  v.dx2 = h->dx2;
  v.dx3 = h->dx3;
  for (int s = 0; s < gemc::NSP; ++s) {
    v.ms[s] = h->ms[s];
    v.gm1[s] = h->gm1[s];
  }
  return v;
}

void hc_artvisc(const HView* hv, const double* ns, const double* vs1, double* Q) {
  const gemc::View v = mk(hv);
  const long long n = gemc::ncell(v) * gemc::NSP;
  for (long long t = 0; t < n; ++t) gemc::artvisc(v, t, ns, vs1, Q);
}

void hc_rk2(const HView* hv, double* vs1, double* vs2, double* vs3) {
  const gemc::View v = mk(hv);
  const long long n1 = (long long)(v.lx2 + 4) * (v.lx3 + 4) * gemc::NSP;
  for (long long t = 0; t < n1; ++t) gemc::rk2_x1(v, t, vs1);
  const long long n2 = (long long)(v.lx1 + 4) * (v.lx3 + 4) * gemc::NSP * 3;
  for (long long t = 0; t < n2; ++t) gemc::rk2_x2(v, t, vs1, vs2, vs3);
  if (!v.flagper) {
    const long long n3 = (long long)(v.lx1 + 4) * (v.lx2 + 4) * gemc::NSP * 3;
    for (long long t = 0; t < n3; ++t) gemc::rk2_x3(v, t, vs1, vs2, vs3);
  }
}

void hc_compression(const HView* hv, const double* vs1, const double* vs2, const double* vs3, const double* Q,
                    double* rhoes, double dt) {
  const gemc::View v = mk(hv);
  const long long n = gemc::ncell(v) * gemc::NSP;
  for (long long t = 0; t < n; ++t) gemc::cmp(v, t, vs1, vs2, vs3, Q, rhoes, dt);
}

}  // extern "C"
