// TEST INFRASTRUCTURE -- not part of the product.  A C++ caller of libgemini_b200.so through
// the reference-named C API only (include/gemini3d_fluid.h): drive_fluid_adv replays the
// reference driver's fluid_adv (libgemini.cpp:143-234) call for call, with host blocks,
// except the routines outside this library -- the solar indices (get_solar_indices_C), the
// average gravity and exospheric temperature (get_gavg_Tinf_C) and the ionization routines
// (clear_ionization_arrays_C, impact_ionization_C, solar_ionization_C), whose results the
// caller loads into the work object beforehand (gem_work_set_sources).  Built with g++ and
// linked against the library by the test, as a maintainer's C++ driver would be.
#include "gemini3d_fluid.h"

extern "C" void drive_fluid_adv(double* pdt, int* plsp, double* fluidvars, double* fluidauxvars,
                                double* electrovars, int* pxtype, void* cfgC, void* xC, void* intvars) {
  int one = 1, two = 2, three = 3;
  v12rhov1_C(&fluidvars, &fluidauxvars);
  T2rhoe_C(&fluidvars, &fluidauxvars);
  // advection substep
  set_global_boundaries_allspec_C(pxtype, &xC, &fluidvars, &fluidauxvars, &intvars, plsp);
  halo_fluidvars_C(pxtype, &xC, &fluidvars, &fluidauxvars);
  interface_vels_allspec_C(pxtype, &xC, &fluidvars, &intvars, plsp);
  sweep3_allspec_mass_C(&fluidvars, &fluidauxvars, &intvars, pxtype, &xC, pdt);
  sweep3_allspec_momentum_C(&fluidvars, &fluidauxvars, &intvars, pxtype, &xC, pdt);
  sweep3_allspec_energy_C(&fluidvars, &fluidauxvars, &intvars, pxtype, &xC, pdt);
  sweep1_allspec_mass_C(&fluidvars, &fluidauxvars, &intvars, pxtype, &xC, pdt);
  sweep1_allspec_momentum_C(&fluidvars, &fluidauxvars, &intvars, pxtype, &xC, pdt);
  sweep1_allspec_energy_C(&fluidvars, &fluidauxvars, &intvars, pxtype, &xC, pdt);
  halo_allparams_C(pxtype, &xC, &fluidvars, &fluidauxvars);
  sweep2_allspec_mass_C(&fluidvars, &fluidauxvars, &intvars, pxtype, &xC, pdt);
  sweep2_allspec_momentum_C(&fluidvars, &fluidauxvars, &intvars, pxtype, &xC, pdt);
  sweep2_allspec_energy_C(&fluidvars, &fluidauxvars, &intvars, pxtype, &xC, pdt);
  rhov12v1_C(&fluidvars, &fluidauxvars);
  clean_param_C(&one, pxtype, &xC, &fluidvars);
  clean_param_C(&two, pxtype, &xC, &fluidvars);
  // compression substep
  VNRicht_artvisc_C(&fluidvars, &intvars);
  halo_fluidvars_C(pxtype, &xC, &fluidvars, &fluidauxvars);
  RK2_global_boundary_allspec_C(pxtype, &xC, &fluidvars);
  compression_C(&fluidvars, &fluidauxvars, &intvars, pxtype, &xC, pdt);
  rhoe2T_C(&fluidvars, &fluidauxvars);
  clean_param_C(&three, pxtype, &xC, &fluidvars);
  // energy diffusion substep
  energy_diffusion_C(&cfgC, pxtype, &xC, &fluidvars, &electrovars, &intvars, pdt);
  clean_param_C(&three, pxtype, &xC, &fluidvars);
  T2rhoe_C(&fluidvars, &fluidauxvars);
  // sources substep
  set_global_boundaries_allspec_C(pxtype, &xC, &fluidvars, &fluidauxvars, &intvars, plsp);
  source_loss_energy_C(&fluidvars, &fluidauxvars, &electrovars, &intvars, pxtype, &xC, pdt);
  source_loss_momentum_C(&fluidvars, &fluidauxvars, &electrovars, &intvars, pxtype, &xC, pdt);
  source_loss_mass_C(&fluidvars, &fluidauxvars, &electrovars, &intvars, pxtype, &xC, pdt);
  clean_param_C(&three, pxtype, &xC, &fluidvars);
  clean_param_C(&two, pxtype, &xC, &fluidvars);
  clean_param_C(&one, pxtype, &xC, &fluidvars);
}
