// fluid_adv in full on a single rank (app/main.f90:280-381), composed from the device
// routines in the reference's order, behind the C ABI (include/gem_fluid.h).  Included by
// gem_fluid.cu after every routine it calls.

#define GEM_TRY(call)            \
  do {                           \
    const int rc_ = (call);      \
    if (rc_ != GEM_OK) return rc_; \
  } while (0)

extern "C" {

int gem_fluid_adv_compression_dev(const gem_cfg* cfg, const gem_grid* g, double* fluidvars, double* fluidauxvars,
                                  const double* electrovars, gem_work* w, double* Q, const double* dt,
                                  void* stream) {
  if (!cfg || check_grid(g) || !fluidvars || !fluidauxvars || !electrovars || !w || !Q || !dt)
    return set_err(GEM_EINVAL, "null argument");
  if (cfg->diffsolvetype != 1 && cfg->diffsolvetype != 2)
    return set_err(GEM_EINVAL, "Unsupported diffusion solver type/mode: %d. Should be either 1 or 2.",
                   cfg->diffsolvetype);
  // advection (app/main.f90:280-319): the fused kernels where the grid allows them (the
  // same results), else the reference's sequence of routines
  const Dims& d = g->dev.d;
  if (d.lx1 >= 4 && !(g->dev.flagper && d.lx3 < 2)) {
    GEM_TRY(advection_keepre(g, fluidvars, fluidauxvars, w, dt, S(stream)));
  } else {
    GEM_TRY(gem_v12rhov1_dev(g, fluidvars, fluidauxvars, stream));
    GEM_TRY(gem_T2rhoe_dev(g, fluidvars, fluidauxvars, stream));
    GEM_TRY(gem_set_global_boundaries_allspec_dev(g, fluidvars, fluidauxvars, w, LSP, stream));
    GEM_TRY(gem_halo_fluidvars_dev(g, fluidvars, fluidauxvars, stream));
    GEM_TRY(gem_interface_vels_allspec_dev(g, fluidvars, w, LSP, stream));
    for (int dim : {3, 1})
      for (int which = 0; which < 3; ++which)
        GEM_TRY(gem_sweep_allspec_dev(g, dim, which, fluidvars, fluidauxvars, w, dt, stream));
    GEM_TRY(gem_halo_allparams_dev(g, fluidvars, fluidauxvars, stream));
    for (int which = 0; which < 3; ++which)
      GEM_TRY(gem_sweep_allspec_dev(g, 2, which, fluidvars, fluidauxvars, w, dt, stream));
    GEM_TRY(gem_rhov12v1_dev(g, fluidvars, fluidauxvars, stream));
    GEM_TRY(gem_clean_param_dev(g, 1, fluidvars, stream));
    GEM_TRY(gem_clean_param_dev(g, 2, fluidvars, stream));
  }
  // compression (app/main.f90:320-338)
  GEM_TRY(gem_vnricht_artvisc_dev(g, fluidvars, Q, stream));
  GEM_TRY(gem_halo_fluidvars_dev(g, fluidvars, fluidauxvars, stream));
  GEM_TRY(gem_rk2_global_boundary_allspec_dev(g, fluidvars, stream));
  GEM_TRY(gem_compression_dev(g, fluidvars, fluidauxvars, Q, dt, stream));
  GEM_TRY(gem_rhoe2T_dev(g, fluidvars, fluidauxvars, stream));
  GEM_TRY(gem_clean_param_dev(g, 3, fluidvars, stream));
  // diffusion (app/main.f90:339-355)
  if (d.lx1 >= 4) {  // the diffusion store with clean_param(3) and T2rhoe folded in (the same results)
    GEM_TRY(diffusion_clean_T2rhoe(cfg, g, fluidvars, fluidauxvars, electrovars, w, dt, S(stream)));
  } else {
    GEM_TRY(gem_energy_diffusion_dev(cfg, g, fluidvars, electrovars, w, dt, stream));
    GEM_TRY(gem_clean_param_dev(g, 3, fluidvars, stream));
    GEM_TRY(gem_T2rhoe_dev(g, fluidvars, fluidauxvars, stream));
  }
  return GEM_OK;
}

int gem_source_loss_allparams_dev(const gem_grid* g, double* fluidvars, double* fluidauxvars,
                                  const double* electrovars, const gem_work* w, const gem_source_inputs* in,
                                  const double* Q, double* Pr, double* Lo, const double* dt, void* stream) {
  if (check_grid(g) || !fluidvars || !fluidauxvars || !electrovars || !w || !in || !Q || !Pr || !Lo || !dt)
    return set_err(GEM_EINVAL, "null argument");
  GEM_TRY(gem_set_global_boundaries_allspec_dev(g, fluidvars, fluidauxvars, w, LSP, stream));
  GEM_TRY(gem_srcs_energy_dev(g, in->nn, in->vn1, in->vn2, in->vn3, in->Tn, fluidvars, Pr, Lo, stream));
  GEM_TRY(gem_energy_source_loss_solve_dev(g, dt, Pr, Lo, in->Qeionize, fluidvars, fluidauxvars, stream));
  GEM_TRY(gem_srcs_momentum_dev(g, in->nn, in->vn1, in->Tn, fluidvars, electrovars, Q, in->alt, in->g1, Pr, Lo,
                                stream));
  GEM_TRY(gem_momentum_source_loss_solve_dev(g, dt, Pr, Lo, fluidvars, fluidauxvars, stream));
  GEM_TRY(gem_srcs_continuity_dev(g, in->nn, in->vn1, in->vn2, in->vn3, in->Tn, fluidvars, Pr, Lo, stream));
  GEM_TRY(gem_mass_source_loss_solve_dev(g, dt, Pr, Lo, in->Prionize, fluidvars, stream));
  GEM_TRY(gem_clean_param_dev(g, 3, fluidvars, stream));
  GEM_TRY(gem_clean_param_dev(g, 2, fluidvars, stream));
  GEM_TRY(gem_clean_param_dev(g, 1, fluidvars, stream));
  return GEM_OK;
}

long long gem_fluid_adv_full_scratch_doubles(const gem_grid* g) {
  if (check_grid(g)) return -1;
  const Dims& d = g->dev.d;
  return 3LL * LSP * d.lx1 * d.lx2 * d.lx3;
}

int gem_fluid_adv_full_dev(const gem_cfg* cfg, const gem_grid* g, double* fluidvars, double* fluidauxvars,
                           const double* electrovars, gem_work* w, const gem_source_inputs* in, double* scratch,
                           const double* dt, void* stream) {
  if (check_grid(g) || !scratch) return set_err(GEM_EINVAL, "null argument");
  const long long n = (long long)LSP * g->dev.d.lx1 * g->dev.d.lx2 * g->dev.d.lx3;
  double* Q = scratch;
  GEM_TRY(gem_fluid_adv_compression_dev(cfg, g, fluidvars, fluidauxvars, electrovars, w, Q, dt, stream));
  return gem_source_loss_allparams_dev(g, fluidvars, fluidauxvars, electrovars, w, in, Q, scratch + n,
                                       scratch + 2 * n, dt, stream);
}

}  // extern "C"

#undef GEM_TRY
