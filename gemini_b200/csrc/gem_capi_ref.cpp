// The reference's *_C entry points (include/gemini3d.h) over host memory, implemented on
// top of the device-resident API (gem_fluid.h).  Each call copies the host blocks it reads
// to device staging buffers, runs the device routine and copies back what the reference
// routine writes.  See include/gemini3d_fluid.h for the object mapping and error policy.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <mutex>

#include "../../include/gemini3d_fluid.h"

namespace {

constexpr int LSP = 7;

std::mutex g_mu;
gem_grid* g_grid = nullptr;  // the "current grid" (module globals lx1..lx3 in the reference)
int g_record = 0;
int g_status = GEM_OK;
long long g_dt_calls = 0;

struct Staging {
  gem_grid* grid = nullptr;
  double *F = nullptr, *A = nullptr, *E = nullptr, *dt = nullptr;
  size_t ng = 0;
  gem_work* work = nullptr;  // the CFL reductions' work object of maxcfl_C / dt_select_C
} g_st;

void drop_staging() {
  cudaFree(g_st.F);
  cudaFree(g_st.A);
  cudaFree(g_st.E);
  cudaFree(g_st.dt);
  if (g_st.work) gem_work_destroy(g_st.work);
  g_st = Staging();
}

// the staging's own work object (created on first use, kept with the staging buffers)
int staging_work(gem_grid* g, gem_work** w) {
  if (!g_st.work) {
    const int rc = gem_work_create(g, &g_st.work);
    if (rc) return rc;
  }
  *w = g_st.work;
  return GEM_OK;
}

void fail(int rc, const char* where) {
  g_status = rc;
  if (g_record) return;
  std::fprintf(stderr, "gemini_b200: %s: %s (status %d)\n", where, gem_last_error(), rc);
  std::exit(1);
}

size_t ghosted(gem_grid* g) {
  int a, b, c;
  gem_grid_dims(g, &a, &b, &c);
  return (size_t)(a + 4) * (b + 4) * (c + 4);
}

// staging buffers sized for grid g (re-allocated when the grid changes)
bool stage(gem_grid* g) {
  const size_t ng = ghosted(g);
  if (g_st.grid == g && g_st.ng == ng && g_st.F) return true;
  drop_staging();
  if (cudaMalloc(&g_st.F, ng * 5 * LSP * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&g_st.A, ng * (2 * LSP + 9) * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&g_st.E, ng * 7 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&g_st.dt, 4 * sizeof(double)) != cudaSuccess) {
    g_status = GEM_ENOMEM;
    return false;
  }
  g_st.grid = g;
  g_st.ng = ng;
  return true;
}

enum Blk { BF = 1, BA = 2, BE = 4 };

bool h2d(const double* F, const double* A, const double* E, int which) {
  const size_t ng = g_st.ng;
  if ((which & BF) && cudaMemcpy(g_st.F, F, ng * 5 * LSP * sizeof(double), cudaMemcpyHostToDevice)) return false;
  if ((which & BA) && cudaMemcpy(g_st.A, A, ng * (2 * LSP + 9) * sizeof(double), cudaMemcpyHostToDevice)) return false;
  if ((which & BE) && cudaMemcpy(g_st.E, E, ng * 7 * sizeof(double), cudaMemcpyHostToDevice)) return false;
  return true;
}

bool d2h(double* F, double* A, int which) {
  const size_t ng = g_st.ng;
  if (cudaDeviceSynchronize() != cudaSuccess) return false;
  if ((which & BF) && cudaMemcpy(F, g_st.F, ng * 5 * LSP * sizeof(double), cudaMemcpyDeviceToHost)) return false;
  if ((which & BA) && cudaMemcpy(A, g_st.A, ng * (2 * LSP + 9) * sizeof(double), cudaMemcpyDeviceToHost)) return false;
  return true;
}

gem_grid* grid_of(void** xC) {
  gem_grid* g = (xC && *xC) ? static_cast<gem_grid*>(*xC) : g_grid;
  return g;
}

// one host-block round trip around a device routine
template <class Fn>
void roundtrip(const char* name, gem_grid* g, double* F, double* A, const double* E, int in, int out, Fn fn) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_status = GEM_OK;
  if (!g) return fail(GEM_EINVAL, name);
  if (!stage(g)) return fail(GEM_ENOMEM, name);
  if (!h2d(F, A, E, in)) return fail(GEM_ECUDA, name);
  const int rc = fn();
  if (rc != GEM_OK) return fail(rc, name);
  if (!d2h(F, A, out)) return fail(GEM_ECUDA, name);
}

void sweep_c(const char* name, int dim, int which, double** fv, double** fav, void** iv, void** xC, double* dt) {
  gem_grid* g = grid_of(xC);
  gem_work* w = iv ? static_cast<gem_work*>(*iv) : nullptr;
  roundtrip(name, g, *fv, *fav, nullptr, BF | BA, (which == 0) ? BF : BA, [&]() {
    if (!w) return GEM_EINVAL;
    if (cudaMemcpy(g_st.dt, dt, sizeof(double), cudaMemcpyHostToDevice)) return GEM_ECUDA;
    return gem_sweep_allspec_dev(g, dim, which, g_st.F, g_st.A, w, g_st.dt, nullptr);
  });
}

}  // namespace

extern "C" {

void gem_capi_bind_grid(gem_grid* g) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_grid = g;
}
// called by gem_grid_destroy: drop the binding and the staging buffers of a dying grid
void gem_capi_forget_grid(gem_grid* g) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_grid == g) g_grid = nullptr;
  if (g_st.grid == g) drop_staging();
}
void gem_capi_set_error_mode(int record_only) { g_record = record_only ? 1 : 0; }
int gem_capi_last_status(void) { return g_status; }

void v12rhov1_C(double** fv, double** fav) {
  roundtrip("v12rhov1_C", g_grid, *fv, *fav, nullptr, BF | BA, BA,
            [&]() { return gem_v12rhov1_dev(g_grid, g_st.F, g_st.A, nullptr); });
}
void T2rhoe_C(double** fv, double** fav) {
  roundtrip("T2rhoe_C", g_grid, *fv, *fav, nullptr, BF | BA, BA,
            [&]() { return gem_T2rhoe_dev(g_grid, g_st.F, g_st.A, nullptr); });
}
void rhov12v1_C(double** fv, double** fav) {
  roundtrip("rhov12v1_C", g_grid, *fv, *fav, nullptr, BF | BA, BF,
            [&]() { return gem_rhov12v1_dev(g_grid, g_st.F, g_st.A, nullptr); });
}
void rhoe2T_C(double** fv, double** fav) {
  roundtrip("rhoe2T_C", g_grid, *fv, *fav, nullptr, BF | BA, BF,
            [&]() { return gem_rhoe2T_dev(g_grid, g_st.F, g_st.A, nullptr); });
}

void interface_vels_allspec_C(int* xtype, void** xC, double** fv, void** iv, int* lsp) {
  (void)xtype;
  gem_grid* g = grid_of(xC);
  gem_work* w = iv ? static_cast<gem_work*>(*iv) : nullptr;
  roundtrip("interface_vels_allspec_C", g, *fv, nullptr, nullptr, BF, 0, [&]() {
    if (!w) return GEM_EINVAL;
    return gem_interface_vels_allspec_dev(g, g_st.F, w, *lsp, nullptr);
  });
}

void set_global_boundaries_allspec_C(int* xtype, void** xC, double** fv, double** fav, void** iv, int* lsp) {
  (void)xtype;
  gem_grid* g = grid_of(xC);
  gem_work* w = iv ? static_cast<gem_work*>(*iv) : nullptr;
  roundtrip("set_global_boundaries_allspec_C", g, *fv, *fav, nullptr, BF | BA, BF | BA, [&]() {
    if (!w) return GEM_EINVAL;
    return gem_set_global_boundaries_allspec_dev(g, g_st.F, g_st.A, w, *lsp, nullptr);
  });
}

void halo_allparams_C(int* xtype, void** xC, double** fv, double** fav) {
  (void)xtype;
  gem_grid* g = grid_of(xC);
  roundtrip("halo_allparams_C", g, *fv, *fav, nullptr, BF | BA, BF | BA,
            [&]() { return gem_halo_allparams_dev(g, g_st.F, g_st.A, nullptr); });
}

void halo_fluidvars_C(int* xtype, void** xC, double** fv, double** fav) {
  (void)xtype;
  gem_grid* g = grid_of(xC);
  roundtrip("halo_fluidvars_C", g, *fv, *fav, nullptr, BF | BA, BF | BA,
            [&]() { return gem_halo_fluidvars_dev(g, g_st.F, g_st.A, nullptr); });
}

#define SWEEP_C(name, dim, which)                                                              \
  void name(double** fv, double** fav, void** iv, int* xtype, void** xC, double* dt) {         \
    (void)xtype;                                                                               \
    sweep_c(#name, dim, which, fv, fav, iv, xC, dt);                                           \
  }
SWEEP_C(sweep3_allspec_mass_C, 3, 0)
SWEEP_C(sweep3_allspec_momentum_C, 3, 1)
SWEEP_C(sweep3_allspec_energy_C, 3, 2)
SWEEP_C(sweep1_allspec_mass_C, 1, 0)
SWEEP_C(sweep1_allspec_momentum_C, 1, 1)
SWEEP_C(sweep1_allspec_energy_C, 1, 2)
SWEEP_C(sweep2_allspec_mass_C, 2, 0)
SWEEP_C(sweep2_allspec_momentum_C, 2, 1)
SWEEP_C(sweep2_allspec_energy_C, 2, 2)
#undef SWEEP_C

// libgemini.f90:774-792 etc.: the allparams forms call mass, momentum, energy in turn
#define SWEEP_ALL(name, dim)                                                                   \
  void name(double** fv, double** fav, void** iv, int* xtype, void** xC, double* dt) {         \
    (void)xtype;                                                                               \
    sweep_c(#name, dim, 0, fv, fav, iv, xC, dt);                                               \
    sweep_c(#name, dim, 1, fv, fav, iv, xC, dt);                                               \
    sweep_c(#name, dim, 2, fv, fav, iv, xC, dt);                                               \
  }
SWEEP_ALL(sweep3_allparams_C, 3)
SWEEP_ALL(sweep1_allparams_C, 1)
SWEEP_ALL(sweep2_allparams_C, 2)
#undef SWEEP_ALL

void clean_param_C(int* iparm, int* xtype, void** xC, double** fv) {
  (void)xtype;
  gem_grid* g = grid_of(xC);
  roundtrip("clean_param_C", g, *fv, nullptr, nullptr, BF, BF,
            [&]() { return gem_clean_param_dev(g, *iparm, g_st.F, nullptr); });
}

void energy_diffusion_C(void** cfgC, int* xtype, void** xC, double** fv, double** ev, void** iv, double* dt) {
  (void)xtype;
  gem_grid* g = grid_of(xC);
  gem_work* w = iv ? static_cast<gem_work*>(*iv) : nullptr;
  const gem_cfg* cfg = cfgC ? static_cast<const gem_cfg*>(*cfgC) : nullptr;
  roundtrip("energy_diffusion_C", g, *fv, nullptr, *ev, BF | BE, BF, [&]() {
    if (!w || !cfg) return GEM_EINVAL;
    if (cudaMemcpy(g_st.dt, dt, sizeof(double), cudaMemcpyHostToDevice)) return GEM_ECUDA;
    return gem_energy_diffusion_dev(cfg, g, g_st.F, g_st.E, w, g_st.dt, nullptr);
  });
}

void maxcfl_C(double** fv, int* xtype, void** xC, double* dt, double* maxcfl) {
  (void)xtype;
  gem_grid* g = grid_of(xC);
  roundtrip("maxcfl_C", g, *fv, nullptr, nullptr, BF, 0, [&]() {
    if (cudaMemcpy(g_st.dt, dt, sizeof(double), cudaMemcpyHostToDevice)) return GEM_ECUDA;
    gem_work* w = nullptr;
    int rc = staging_work(g, &w);
    if (rc) return rc;
    rc = gem_maxcfl_dev(g, g_st.F, w, g_st.dt, g_st.dt + 1, nullptr);
    if (!rc && cudaMemcpy(maxcfl, g_st.dt + 1, sizeof(double), cudaMemcpyDeviceToHost)) rc = GEM_ECUDA;
    return rc;
  });
}

// ---- the compression and source sub-steps (libgemini_c.f90:762-793, 852-970;
// libgemini_mpi_c.f90:476-486): Q, Pr, Lo and the source inputs live in the work object

void VNRicht_artvisc_C(double** fv, void** iv) {
  gem_grid* g = g_grid;
  gem_work* w = iv ? static_cast<gem_work*>(*iv) : nullptr;
  roundtrip("VNRicht_artvisc_C", g, *fv, nullptr, nullptr, BF, 0, [&]() {
    double* Q = nullptr;
    if (!w) return GEM_EINVAL;
    int rc = gem_work_substep_buffers(w, nullptr, &Q, nullptr, nullptr);
    return rc ? rc : gem_vnricht_artvisc_dev(g, g_st.F, Q, nullptr);
  });
}

void compression_C(double** fv, double** fav, void** iv, int* xtype, void** xC, double* dt) {
  (void)xtype;
  gem_grid* g = grid_of(xC);
  gem_work* w = iv ? static_cast<gem_work*>(*iv) : nullptr;
  roundtrip("compression_C", g, *fv, *fav, nullptr, BF | BA, BA, [&]() {
    double* Q = nullptr;
    if (!w) return GEM_EINVAL;
    int rc = gem_work_substep_buffers(w, nullptr, &Q, nullptr, nullptr);
    if (rc) return rc;
    if (cudaMemcpy(g_st.dt, dt, sizeof(double), cudaMemcpyHostToDevice)) return GEM_ECUDA;
    return gem_compression_dev(g, g_st.F, g_st.A, Q, g_st.dt, nullptr);
  });
}

void RK2_global_boundary_allspec_C(int* xtype, void** xC, double** fv) {
  (void)xtype;
  gem_grid* g = grid_of(xC);
  roundtrip("RK2_global_boundary_allspec_C", g, *fv, nullptr, nullptr, BF, BF,
            [&]() { return gem_rk2_global_boundary_allspec_dev(g, g_st.F, nullptr); });
}

namespace {
enum SrcPart { SRC_ENERGY = 1, SRC_MOMENTUM = 2, SRC_MASS = 4 };

// source_loss_{energy,momentum,mass}_in (libgemini.f90:1132-1195): the rates of the part
// (sources.f90), then its exponential time-differencing solve (multifluid.f90:474-549)
void source_loss_c(const char* name, int parts, double** fv, double** fav, double** ev, void** iv, void** xC,
                   double* dt) {
  gem_grid* g = grid_of(xC);
  gem_work* w = iv ? static_cast<gem_work*>(*iv) : nullptr;
  roundtrip(name, g, *fv, *fav, *ev, BF | BA | BE, BF | BA, [&]() {
    const gem_source_inputs* in = nullptr;
    double *Q = nullptr, *Pr = nullptr, *Lo = nullptr;
    if (!w) return GEM_EINVAL;
    int rc = gem_work_substep_buffers(w, &in, &Q, &Pr, &Lo);
    if (rc) return rc;
    if (!in) return GEM_EINVAL;  // gem_work_set_sources has not run
    if (cudaMemcpy(g_st.dt, dt, sizeof(double), cudaMemcpyHostToDevice)) return GEM_ECUDA;
    if (parts & SRC_ENERGY) {
      if ((rc = gem_srcs_energy_dev(g, in->nn, in->vn1, in->vn2, in->vn3, in->Tn, g_st.F, Pr, Lo, nullptr))) return rc;
      if ((rc = gem_energy_source_loss_solve_dev(g, g_st.dt, Pr, Lo, in->Qeionize, g_st.F, g_st.A, nullptr)))
        return rc;
    }
    if (parts & SRC_MOMENTUM) {
      if ((rc = gem_srcs_momentum_dev(g, in->nn, in->vn1, in->Tn, g_st.F, g_st.E, Q, in->alt, in->g1, Pr, Lo,
                                      nullptr)))
        return rc;
      if ((rc = gem_momentum_source_loss_solve_dev(g, g_st.dt, Pr, Lo, g_st.F, g_st.A, nullptr))) return rc;
    }
    if (parts & SRC_MASS) {
      if ((rc = gem_srcs_continuity_dev(g, in->nn, in->vn1, in->vn2, in->vn3, in->Tn, g_st.F, Pr, Lo, nullptr)))
        return rc;
      if ((rc = gem_mass_source_loss_solve_dev(g, g_st.dt, Pr, Lo, in->Prionize, g_st.F, nullptr))) return rc;
    }
    return GEM_OK;
  });
}
}  // namespace

void source_loss_energy_C(double** fv, double** fav, double** ev, void** iv, int* xtype, void** xC, double* dt) {
  (void)xtype;
  source_loss_c("source_loss_energy_C", SRC_ENERGY, fv, fav, ev, iv, xC, dt);
}
void source_loss_momentum_C(double** fv, double** fav, double** ev, void** iv, int* xtype, void** xC, double* dt) {
  (void)xtype;
  source_loss_c("source_loss_momentum_C", SRC_MOMENTUM, fv, fav, ev, iv, xC, dt);
}
void source_loss_mass_C(double** fv, double** fav, double** ev, void** iv, int* xtype, void** xC, double* dt) {
  (void)xtype;
  source_loss_c("source_loss_mass_C", SRC_MASS, fv, fav, ev, iv, xC, dt);
}
void source_loss_allparams_C(double** fv, double** fav, double** ev, void** iv, int* xtype, void** xC, double* dt) {
  (void)xtype;
  source_loss_c("source_loss_allparams_C", SRC_ENERGY | SRC_MOMENTUM | SRC_MASS, fv, fav, ev, iv, xC, dt);
}

void dt_select_C(void** cfgC, int* xtype, void** xC, double** fv, double** fav, double* t, double* tout,
                 double* tglowout, double* dt) {
  (void)xtype;
  (void)fav;
  gem_grid* g = grid_of(xC);
  const gem_cfg* cfg = cfgC ? static_cast<const gem_cfg*>(*cfgC) : nullptr;
  double dtnew = 0.0;
  roundtrip("dt_select_C", g, *fv, nullptr, nullptr, BF, 0, [&]() {
    if (!cfg) return GEM_EINVAL;
    gem_work* w = nullptr;
    int rc = staging_work(g, &w);
    if (rc) return rc;
    rc = gem_dt_calc_dev(g, cfg->tcfl, g_st.F, w, g_st.dt, nullptr);
    if (!rc && cudaMemcpy(&dtnew, g_st.dt, sizeof(double), cudaMemcpyDeviceToHost)) rc = GEM_ECUDA;
    return rc;
  });
  if (g_status != GEM_OK) return;
  // dt_calc already applied the final 1e-6 floor; dt_comm clips before the floor
  // (temporal_mpi.f90:55-66), so redo the clip and floor here in that order.
  const double dtprev = *dt;
  double d = dtnew;
  if (cfg->flagglow && *t + d > *tglowout) d = *tglowout - *t;
  if (*t + d > *tout) d = *tout - *t;
  d = (d > 1e-6) ? d : 1e-6;
  if (++g_dt_calls > 1 && d / dtprev > 2) d = 2 * dtprev;  // libgemini_mpi.f90:473-481
  *dt = d;
}

}  // extern "C"
