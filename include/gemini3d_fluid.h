/* gemini3d_fluid.h -- the fluid-advance subset of GEMINI3D's C API (include/gemini3d.h),
 * exported by libgemini_b200.so with the reference's names and signatures so that a C,
 * C++ or Fortran (bind(C)) driver links against it unchanged.
 *
 * Semantics follow the reference: pointers are passed by reference (double**, void**),
 * the blocks are HOST memory in the Fortran layout of libgemini.f90:401-417, and the grid
 * sizes are the library's "current grid" (the reference keeps them as module globals in
 * `grid`, libgemini_c.f90:28).  Each call stages the blocks to the GPU, runs the device
 * kernels and copies the results back -- correct, but every call pays the PCIe copies; the
 * device-resident API in gem_fluid.h is the fast path.
 *
 * Object mapping: xC is a gem_grid* (xtype is accepted and ignored: the device grid holds
 * its own metric arrays, Cartesian or dipole), intvars is a gem_work*, cfgC is a gem_cfg*.
 * Errors: the reference stops the program (error stop); these entry points do the same by
 * default, printing the message to stderr and exiting with status 1.  After
 * gem_capi_set_error_mode(1) they record the status instead (gem_capi_last_status()).
 */
#ifndef GEMINI3D_FLUID_H
#define GEMINI3D_FLUID_H

#include "gem_fluid.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Bind the grid whose sizes the size-less entry points (v12rhov1_C, T2rhoe_C, rhov12v1_C,
 * rhoe2T_C) use; gem_grid_create binds each new grid, gem_grid_destroy unbinds it.
 * Replaces the module globals set by grid_size_in_C / read_grid_C (gemini3d.h:45,117). */
void gem_capi_bind_grid(gem_grid* g);
void gem_capi_set_error_mode(int record_only);
int gem_capi_last_status(void);

/* gemini3d.h:64 -- multifluid.f90:206-214 */
void v12rhov1_C(double** fluidvars, double** fluidauxvars);
/* gemini3d.h:65 -- multifluid.f90:193-202 */
void T2rhoe_C(double** fluidvars, double** fluidauxvars);
/* gemini3d.h:66 -- advec.f90:216-229 via libgemini_c.f90:473-488 */
void interface_vels_allspec_C(int* xtype, void** xC, double** fluidvars, void** intvars, int* lsp);
/* gemini3d.h:67-78 -- advec.f90:233-381 via multifluid.f90:49-126, libgemini_c.f90:513-745 */
void sweep3_allparams_C(double** fluidvars, double** fluidauxvars, void** intvars, int* xtype, void** xC, double* dt);
void sweep3_allspec_mass_C(double** fluidvars, double** fluidauxvars, void** intvars, int* xtype, void** xC, double* dt);
void sweep3_allspec_momentum_C(double** fluidvars, double** fluidauxvars, void** intvars, int* xtype, void** xC, double* dt);
void sweep3_allspec_energy_C(double** fluidvars, double** fluidauxvars, void** intvars, int* xtype, void** xC, double* dt);
void sweep1_allparams_C(double** fluidvars, double** fluidauxvars, void** intvars, int* xtype, void** xC, double* dt);
void sweep1_allspec_mass_C(double** fluidvars, double** fluidauxvars, void** intvars, int* xtype, void** xC, double* dt);
void sweep1_allspec_momentum_C(double** fluidvars, double** fluidauxvars, void** intvars, int* xtype, void** xC, double* dt);
void sweep1_allspec_energy_C(double** fluidvars, double** fluidauxvars, void** intvars, int* xtype, void** xC, double* dt);
void sweep2_allparams_C(double** fluidvars, double** fluidauxvars, void** intvars, int* xtype, void** xC, double* dt);
void sweep2_allspec_mass_C(double** fluidvars, double** fluidauxvars, void** intvars, int* xtype, void** xC, double* dt);
void sweep2_allspec_momentum_C(double** fluidvars, double** fluidauxvars, void** intvars, int* xtype, void** xC, double* dt);
void sweep2_allspec_energy_C(double** fluidvars, double** fluidauxvars, void** intvars, int* xtype, void** xC, double* dt);
/* gemini3d.h:79 -- multifluid.f90:218-233 */
void rhov12v1_C(double** fluidvars, double** fluidauxvars);
/* gemini3d.h:80 -- multifluid.f90:553-688 via libgemini_c.f90:811-825 */
void clean_param_C(int* iparm, int* xtype, void** xC, double** fluidvars);
/* gemini3d.h:83 -- multifluid.f90:179-189 */
void rhoe2T_C(double** fluidvars, double** fluidauxvars);
/* gemini3d.h:84 -- multifluid.f90:309-342 via libgemini_c.f90:827-850 */
void energy_diffusion_C(void** cfgC, int* xtype, void** xC, double** fluidvars, double** electrovars,
                        void** intvars, double* dt);
/* gemini3d.h:94 -- temporal.f90:12-49 via libgemini_c.f90:1043-1056 */
void maxcfl_C(double** fluidvars, int* xtype, void** xC, double* dt, double* maxcfl);
/* gemini3d.h:101 -- advec.f90:137-149 via libgemini_c.f90:491-509 */
void set_global_boundaries_allspec_C(int* xtype, void** xC, double** fluidvars, double** fluidauxvars,
                                     void** intvars, int* lsp);
/* gemini3d.h:136-137 -- multifluid_mpi.f90:12-41 via libgemini_mpi_c.f90:414-459; on one
 * resident grid only the x3 periodic self-wrap remains (mpihalo.f90:147-151) */
void halo_allparams_C(int* xtype, void** xC, double** fluidvars, double** fluidauxvars);
void halo_fluidvars_C(int* xtype, void** xC, double** fluidvars, double** fluidauxvars);
/* gemini3d.h:81 -- multifluid.f90:237-268 VNRicht_artvisc via libgemini_c.f90:762-771; Q stays
 * in the work object (intvars), as the reference keeps it in intvars%Q */
void VNRicht_artvisc_C(double** fluidvars, void** intvars);
/* gemini3d.h:82 -- multifluid.f90:274-302 compression via libgemini_c.f90:775-793 (reads Q) */
void compression_C(double** fluidvars, double** fluidauxvars, void** intvars, int* xtype, void** xC, double* dt);
/* gemini3d.h:139 -- sources_mpi.f90:68-111 RK2_global_boundary via libgemini_mpi_c.f90:476-486 */
void RK2_global_boundary_allspec_C(int* xtype, void** xC, double** fluidvars);
/* gemini3d.h:85-89 -- libgemini.f90:1117-1195 via libgemini_c.f90:852-970: the production and
 * loss rates (sources.f90) and the exponential time-differencing solve (multifluid.f90:474-549)
 * of energy, momentum, mass, or all three in that order.  They read the neutral atmosphere and
 * the ionization rates that gem_work_set_sources loaded into the work object (intvars), and
 * the Q that VNRicht_artvisc_C left there. */
void source_loss_allparams_C(double** fluidvars, double** fluidauxvars, double** electrovars, void** intvars,
                             int* xtype, void** xC, double* dt);
void source_loss_mass_C(double** fluidvars, double** fluidauxvars, double** electrovars, void** intvars, int* xtype,
                        void** xC, double* dt);
void source_loss_momentum_C(double** fluidvars, double** fluidauxvars, double** electrovars, void** intvars,
                            int* xtype, void** xC, double* dt);
void source_loss_energy_C(double** fluidvars, double** fluidauxvars, double** electrovars, void** intvars,
                          int* xtype, void** xC, double* dt);
/* gemini3d.h:140 -- libgemini_mpi.f90:450-485 dt_select with temporal_mpi.f90:27-84 dt_comm
 * on one grid: dt = tcfl-limited CFL step, clipped so that t+dt does not pass tglowout (when
 * cfg->flagglow) or tout, floored at 1e-6; from the second call on, dt may at most double
 * (dtscale = 2, libgemini_mpi.f90:38) relative to the value passed in */
void dt_select_C(void** cfgC, int* xtype, void** xC, double** fluidvars, double** fluidauxvars,
                 double* t, double* tout, double* tglowout, double* dt);

#ifdef __cplusplus
}
#endif

#endif /* GEMINI3D_FLUID_H */
