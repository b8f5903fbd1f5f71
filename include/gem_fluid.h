/* gem_fluid.h -- device-resident C ABI of the B200 fluid-advance library (libgemini_b200.so).
 *
 * This is the path GEMINI3D calls for the multifluid advection sweeps and the
 * field-aligned heat diffusion.  The entry points below take DEVICE pointers to the
 * reference's own memory blocks (same Fortran layout, see below), an explicit stream, and
 * return an int status (no error stop, no host synchronisation unless stated).  The
 * host-pointer entry points with the reference's names and signatures are declared in
 * gemini3d_fluid.h.
 *
 * Memory-block layout (libgemini.f90:401-417, 462-519), Fortran order, x1 fastest,
 * 2 ghost cells per side, lsp = 7 (6 ions + electrons):
 *   fluidvars    (lx1+4, lx2+4, lx3+4, 5*lsp)   ns | vs1 | vs2 | vs3 | Ts
 *   fluidauxvars (lx1+4, lx2+4, lx3+4, 2*lsp+9) rhovs1 | rhoes | 9 MHD scalars (untouched)
 *   electrovars  (lx1+4, lx2+4, lx3+4, 7)       E1 E2 E3 J1 J2 J3 Phi (J1 read)
 * Work arrays carried in gem_work (libgemini.f90:92-129, 284-291):
 *   vs1i (lx1+1,lx2,lx3,lsp), vs2i (lx1,lx2+1,lx3,lsp), vs3i (lx1,lx2,lx3+1,lsp)
 *   nn (lx1,lx2,lx3,3) = n(O), n(N2), n(O2);  Tn (lx1,lx2,lx3)
 * All values are IEEE binary64.  Streams are passed as void* (a cudaStream_t; NULL is
 * the legacy default stream).
 */
#ifndef GEM_FLUID_H
#define GEM_FLUID_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define GEM_OK 0
#define GEM_EINVAL 1      /* bad argument or unsupported size */
#define GEM_ENONFINITE 2  /* non-finite values detected (gem_check_finite) */
#define GEM_ETIMEOUT 3    /* a bounded device wait gave up */
#define GEM_ECUDA 4       /* CUDA runtime error; see gem_last_error() */
#define GEM_ENOMEM 5      /* device allocation failed */

typedef struct gem_grid gem_grid; /* device copy of a curvmesh (meshobj.f90:49-154) */
typedef struct gem_work gem_work; /* interface velocities, neutrals, dt and scratch */

/* Host description of a grid; every array is copied to the device by gem_grid_create.
 * Replaces read_grid_C / set_gridpointer_dyntype (libgemini_c.f90:63-82): the grid
 * object the *_C entry points receive as xC is a gem_grid*. */
typedef struct gem_grid_desc {
  int lx1, lx2, lx3;
  int gridflag; /* 0 closed dipole, 1 open inverted, 2 non-inverted (meshobj.f90:549-570) */
  int flagper;  /* x3 periodic (meshobj.f90:324-335) */
  const double *dx1, *dx1i, *dx2, *dx2i, *dx3, *dx3i; /* dx: l+3 values (0:l+2), dxi: l */
  const double *h1, *h2, *h3;                          /* ghosted (lx1+4)(lx2+4)(lx3+4) */
  const double *h1x1i, *h2x1i, *h3x1i;                 /* (lx1+1, lx2, lx3) */
  const double *h1x2i, *h2x2i, *h3x2i;                 /* (lx1, lx2+1, lx3) */
  const double *h1x3i, *h2x3i, *h3x3i;                 /* (lx1, lx2, lx3+1) */
  const unsigned char* nullpts;                        /* (lx1, lx2, lx3) or NULL */
  int unit_metrics; /* 1 if every metric factor is exactly 1 (Cartesian); the kernels then
                       skip the metric loads -- results are identical */
} gem_grid_desc;

/* Plain-value run parameters (gemini_cfg fields read on this path, config_nml.f90). */
typedef struct gem_cfg {
  double Teinf;      /* exospheric electron temperature for the top Dirichlet BC */
  int diffsolvetype; /* 1 backward Euler, 2 TRBDF2 */
  double tcfl;       /* target CFL number for dt_calc */
  int flagglow;      /* non-zero: dt_select_C also clips dt at the GLOW output time */
} gem_cfg;

const char* gem_last_error(void); /* thread-local message for the last non-zero status */
int gem_version(void);

/* grid and work objects (allocate device memory; synchronous) */
int gem_grid_create(const gem_grid_desc* desc, gem_grid** out);
int gem_grid_destroy(gem_grid* g);
int gem_grid_dims(const gem_grid* g, int* lx1, int* lx2, int* lx3);
/* The work object holds the per-grid state of the step (interface velocities, neutral inputs,
 * dt, reductions).  The diffusion's band-solve scratch (one slot of lx1 x 8 x 32 doubles per
 * resident warp, at most ~1 GB for 384-row columns) is allocated by the first
 * gem_energy_diffusion_dev / gem_fluid_adv_dev call that uses the work object: make that
 * first call before capturing these calls in a CUDA graph.  Work objects that only take part
 * in a gem_batch never allocate it (the batch has its own). */
int gem_work_create(const gem_grid* g, gem_work** out);
/* allocate the work object's diffusion scratch now (before measuring free memory or capturing) */
int gem_work_prepare(gem_work* w, const gem_grid* g);
int gem_work_destroy(gem_work* w);
/* copy neutral inputs (host pointers; nn (lx1,lx2,lx3,3), Tn (lx1,lx2,lx3)) */
int gem_work_set_neutrals(gem_work* w, const double* nn, const double* Tn);
/* host<->device copies of vs1i|vs2i|vs3i (which: 1,2,3); dir 0 host->device, 1 device->host */
int gem_work_interface_vels(gem_work* w, int which, double* host, int dir);
/* device pointer of the work array vs{which}i (which 1..3), of nn (4) or Tn (5) */
double* gem_work_array(gem_work* w, int which);
/* device pointer of the 1-element dt slot inside the work object */
double* gem_work_dt(gem_work* w);
/* Per-column exospheric (top Dirichlet) temperature, lx2*lx3 values with i2 fastest,
 * replacing cfg->Teinf on the gridflag 1 / 2 boundary (diffusion.f90:67-79) for the steps
 * that follow; NULL restores the scalar Teinf.  on_device: Ttop is a device pointer.  No
 * counterpart in the reference (its Teinf is one number); it is the boundary control of
 * the differentiable path.  A batch reads it when created. */
int gem_work_set_top_temperature(gem_work* w, const double* Ttop, int on_device);

/* ---- individual reference routines, device-resident ------------------------------ */
/* multifluid.f90:179-233 conversions over the full ghosted arrays, all species */
int gem_v12rhov1_dev(const gem_grid* g, const double* fluidvars, double* fluidauxvars, void* stream);
int gem_T2rhoe_dev(const gem_grid* g, const double* fluidvars, double* fluidauxvars, void* stream);
int gem_rhov12v1_dev(const gem_grid* g, double* fluidvars, const double* fluidauxvars, void* stream);
int gem_rhoe2T_dev(const gem_grid* g, double* fluidvars, const double* fluidauxvars, void* stream);
/* advec.f90:21-149 (single resident grid: every boundary is global) */
int gem_set_global_boundaries_allspec_dev(const gem_grid* g, double* fluidvars, double* fluidauxvars,
                                          const gem_work* w, int lsp, void* stream);
/* multifluid_mpi.f90:12-41 on one grid: only the x3 periodic self-wrap (mpihalo.f90:147-151) */
int gem_halo_fluidvars_dev(const gem_grid* g, double* fluidvars, double* fluidauxvars, void* stream);
int gem_halo_allparams_dev(const gem_grid* g, double* fluidvars, double* fluidauxvars, void* stream);
/* advec.f90:155-229 */
int gem_interface_vels_allspec_dev(const gem_grid* g, const double* fluidvars, gem_work* w, int lsp,
                                   void* stream);
/* advec.f90:233-381 via multifluid.f90:49-126: dim 1..3; which 0 mass (ns, 1..6),
 * 1 momentum (rhovs1, 1..6, frank 1), 2 energy (rhoes, 1..7); dt is a device pointer */
int gem_sweep_allspec_dev(const gem_grid* g, int dim, int which, double* fluidvars,
                          double* fluidauxvars, const gem_work* w, const double* dt, void* stream);
/* multifluid.f90:553-688; iparm 1 density, 2 velocity, 3 temperature */
int gem_clean_param_dev(const gem_grid* g, int iparm, double* fluidvars, void* stream);
/* multifluid.f90:309-342 with collisions.f90:162-199 and diffusion.f90:24-152.  Each band
 * system (TRBDF2 stages or backward Euler, PDEparabolic.f90:19-346) is factored and solved in
 * the operation order of the reference's LAPACK dgbsv call (dgbtf2 partial pivoting, dgbtrs
 * and dtbsv with reference-BLAS semantics), so the result equals the reference arithmetic bit
 * for bit, T**2.5 being the correctly rounded value.  Ghost cells: the x1 layers 0 and lx1+1
 * receive the Dirichlet values, then max(T,100) over every cell.  The first call with a work
 * object allocates its band-solve scratch (gem_work_create). */
int gem_energy_diffusion_dev(const gem_cfg* cfg, const gem_grid* g, double* fluidvars,
                             const double* electrovars, const gem_work* w, const double* dt,
                             void* stream);
/* temporal_mpi.f90:86-167 dt_calc and the 1e-6 floor of dt_comm; writes *dt_out (device).
 * The result is max(tcfl * min over cells of 1/rate, 1e-6): the reference's dt_calc has no
 * floor (dt_comm applies it after its output clips, temporal_mpi.f90:55-66), so for a CFL step
 * below 1e-6 s this returns the floored value. */
int gem_dt_calc_dev(const gem_grid* g, double tcfl, const double* fluidvars, gem_work* w,
                    double* dt_out, void* stream);
/* temporal.f90:12-49 cflcalc; writes *maxcfl_out (device) */
int gem_maxcfl_dev(const gem_grid* g, const double* fluidvars, gem_work* w, const double* dt,
                   double* maxcfl_out, void* stream);
/* The compression sub-step (app/main.f90:320-338) as the reference's separate calls, after
 * the post-advection clean_param(1), (2):
 *   gem_vnricht_artvisc_dev: multifluid.f90:237-268 VNRicht_artvisc (libgemini.f90
 *     VNRicht_artvisc_C), xicon = 3; writes Q (device, interior (lx1, lx2, lx3, LSP),
 *     column-major; 0 for the electrons) from ns and vs1 as they stand, x1 ghosts included;
 *   gem_rk2_global_boundary_allspec_dev: sources_mpi.f90:68-111 RK2_global_boundary on a
 *     single rank (RK2_global_boundary_allspec_C): zero-order-hold velocity ghosts, x1 (vs1)
 *     then x2 and, unless x3 is periodic, x3 (vs1, vs2, vs3); on periodic grids call
 *     gem_halo_fluidvars_dev first, as the reference does;
 *   gem_compression_dev: multifluid.f90:274-302 compression (compression_C) with
 *     calculus/div.f90:110-200 div3D: the half- and full-step update of rhoes (fluidauxvars
 *     block 2) from each species' velocity divergence and Q; dt is a device pointer.
 * Results equal the reference restatement bit for bit (IEEE divisions, the reference's
 * operation order). */
int gem_vnricht_artvisc_dev(const gem_grid* g, const double* fluidvars, double* Q, void* stream);
int gem_rk2_global_boundary_allspec_dev(const gem_grid* g, double* fluidvars, void* stream);
int gem_compression_dev(const gem_grid* g, const double* fluidvars, double* fluidauxvars, const double* Q,
                        const double* dt, void* stream);

/* The source/loss solves of the source sub-step (libgemini.f90:1154-1200, after the rates):
 * Pr, Lo: device, interior (lx1, lx2, lx3, LSP), column-major, as the rate routines leave
 * them; dt: device pointer.  The exponential time differencing step
 * (calculus.in.f90:174-196 ETD_uncoupled) of each species at interior cells, then the
 * derived fields over every cell, ghosts included:
 *   gem_energy_source_loss_solve_dev: multifluid.f90:474-495 energy_source_loss_solve
 *     (inside source_loss_energy_C): Pr(:,:,:,LSP) += Qeprecip (interior (lx1, lx2, lx3)),
 *     in place as the reference does; rhoes (fluidauxvars block 2) stepped; Ts formed;
 *   gem_momentum_source_loss_solve_dev: multifluid.f90:500-528 momentum_source_loss_solve
 *     (inside source_loss_momentum_C): ion rhovs1 stepped, vs1 formed, electron vs1 and
 *     rhovs1 from the ion current;
 *   gem_mass_source_loss_solve_dev: multifluid.f90:532-549 mass_source_loss_solve (inside
 *     source_loss_mass_C): Pr(:,:,:,1:LSP-1) += Prprecip (interior, LSP-1 species), in
 *     place; ion ns stepped; electron ns = sum of the ion densities.
 * Results equal the reference restatement up to the device's double exp (within 1 ulp). */
int gem_energy_source_loss_solve_dev(const gem_grid* g, const double* dt, double* Pr, const double* Lo,
                                     const double* Qeprecip, double* fluidvars, double* fluidauxvars, void* stream);
int gem_momentum_source_loss_solve_dev(const gem_grid* g, const double* dt, const double* Pr, const double* Lo,
                                       double* fluidvars, double* fluidauxvars, void* stream);
int gem_mass_source_loss_solve_dev(const gem_grid* g, const double* dt, double* Pr, const double* Lo,
                                   const double* Prprecip, double* fluidvars, void* stream);

/* The production and loss rates (sources.f90) the solves above take, into Pr and Lo (device,
 * interior (lx1, lx2, lx3, LSP), column-major; every element written).  nn: device, interior
 * (lx1, lx2, lx3, species), neutral densities O, N2, O2, H, N, NO (the energy and momentum
 * rates read the first four); vn1, vn2, vn3, Tn, alt, g1: device, interior (lx1, lx2, lx3);
 * fluidvars and electrovars: the device state blocks (ns, vs1, vs2, vs3, Ts and E1 read).
 *   gem_srcs_continuity_dev: sources.f90:18-276 srcsContinuity (inside source_loss_mass_C);
 *   gem_srcs_energy_dev: sources.f90:396-485 srcsEnergy with collisions.f90:58-159 (inside
 *     source_loss_energy_C);
 *   gem_srcs_momentum_dev: sources.f90:279-393 srcsMomentum_curv on a single rank (inside
 *     source_loss_momentum_C), with Q from gem_vnricht_artvisc_dev; needs lx1 >= 2.
 * Every expression follows the reference's operation order; the device's pow, exp, log,
 * log10, erf, tanh and sin stand in for the C library's. */
int gem_srcs_continuity_dev(const gem_grid* g, const double* nn, const double* vn1, const double* vn2,
                            const double* vn3, const double* Tn, const double* fluidvars, double* Pr, double* Lo,
                            void* stream);
int gem_srcs_energy_dev(const gem_grid* g, const double* nn, const double* vn1, const double* vn2, const double* vn3,
                        const double* Tn, const double* fluidvars, double* Pr, double* Lo, void* stream);
int gem_srcs_momentum_dev(const gem_grid* g, const double* nn, const double* vn1, const double* Tn,
                          const double* fluidvars, const double* electrovars, const double* Q, const double* alt,
                          const double* g1, double* Pr, double* Lo, void* stream);

/* ---- fluid_adv in full on a single rank (app/main.f90:280-381) --------------------
 * The reference's sequence of the routines above, each a separate launch:
 *   gem_fluid_adv_compression_dev: the advection (v12rhov1, T2rhoe, boundaries, halo,
 *     interface velocities, x3/x1/x2 sweeps, rhov12v1, clean_param(1), (2)), the compression
 *     sub-step (VNRicht_artvisc into Q (device, interior (lx1, lx2, lx3, LSP)), halo,
 *     RK2_global_boundary, compression, rhoe2T, clean_param(3)) and the diffusion
 *     (energy_diffusion, clean_param(3), T2rhoe); the diffusion reads nn and Tn from w;
 *   gem_source_loss_allparams_dev: source_loss_allparams_C's sequence (libgemini.f90
 *     1154-1200): set_global_boundaries, the energy rates and solve (Qeionize added),
 *     the momentum rates (with the compression step's Q) and solve, the continuity rates
 *     and solve (Prionize added), clean_param(3), (2), (1); Pr, Lo: device scratch of
 *     LSP*lx1*lx2*lx3 doubles each;
 *   gem_fluid_adv_full_dev: both, with scratch of gem_fluid_adv_full_scratch_doubles(g)
 *     device doubles (Q, Pr, Lo).
 * The ionization rates (ionization.f90) are inputs, as the reference's impact_ionization
 * and photoionization fill Prionize and Qeionize before this sub-step. */
typedef struct gem_source_inputs {
  const double* nn;        /* interior (lx1, lx2, lx3, 6): O, N2, O2, H, N, NO */
  const double *vn1, *vn2, *vn3, *Tn; /* interior neutral winds and temperature */
  const double *alt, *g1;  /* interior altitude and x1 gravity (meshobj.f90 x%alt, x%g1) */
  const double* Prionize;  /* interior (lx1, lx2, lx3, LSP-1) ion production */
  const double* Qeionize;  /* interior (lx1, lx2, lx3) electron heating */
} gem_source_inputs;
int gem_fluid_adv_compression_dev(const gem_cfg* cfg, const gem_grid* g, double* fluidvars, double* fluidauxvars,
                                  const double* electrovars, gem_work* w, double* Q, const double* dt, void* stream);
int gem_source_loss_allparams_dev(const gem_grid* g, double* fluidvars, double* fluidauxvars,
                                  const double* electrovars, const gem_work* w, const gem_source_inputs* in,
                                  const double* Q, double* Pr, double* Lo, const double* dt, void* stream);
long long gem_fluid_adv_full_scratch_doubles(const gem_grid* g);
/* The reference's work object (gemini_work, libgemini.f90:92-129) carries the neutral
 * atmosphere (intvars%atmos: nn, vn1..3, Tn), the ionization rates (Prionize, Qeionize), the
 * artificial viscosity Q and the rate arrays Pr, Lo that the host-memory sub-step routines
 * of gemini3d_fluid.h (VNRicht_artvisc_C, compression_C, source_loss_*_C) read and write.
 * gem_work_set_sources copies those inputs (HOST memory, the layouts of gem_source_inputs)
 * into device buffers owned by w, and also loads w's diffusion neutrals (O, N2, O2) and Tn
 * from them; the reference fills them with neutral_atmos_winds_C and the ionization routines,
 * which lie outside this library.  gem_work_substep_buffers returns those device buffers
 * (src is NULL until gem_work_set_sources has run); both allocate them on first use. */
int gem_work_set_sources(gem_work* w, const gem_source_inputs* host);
int gem_work_substep_buffers(gem_work* w, const gem_source_inputs** src, double** Q, double** Pr, double** Lo);

/* ---- device-resident time stepping --------------------------------------------------
 * The simulation clock in device memory, so that a loop of steps keeps dt on the device.
 * gem_dt_select_dev: libgemini_mpi.f90:450-483 dt_select with temporal_mpi.f90:27-84
 *   dt_comm on a single rank: the CFL step (gem_dt_calc_dev, into clock->dtcfl), clipped
 *   so that t + dt passes neither the next GLOW output (cfg->flagglow) nor the next output,
 *   floored at 1e-6, and for it > 1 grown by at most 2x over the previous step, which *dt
 *   holds on entry (the reference's intent(inout) dt); writes *dt (device).
 * gem_clock_advance_dev: after a step, t = t + dt (app/main.f90:233) and it = it + 1.
 * The output times are the caller's: it sets tout / tglowout when an output is written.
 * Results equal the reference's arithmetic bit for bit. */
typedef struct gem_clock {
  double t, tout, tglowout; /* simulation time, next output, next GLOW output */
  double dtcfl;             /* the CFL step of the latest selection (written) */
  long long it;             /* iteration counter (get_it()), 1 on the first step */
} gem_clock;
int gem_dt_select_dev(const gem_cfg* cfg, const gem_grid* g, const double* fluidvars, gem_work* w, gem_clock* clock,
                      double* dt, void* stream);
int gem_clock_advance_dev(gem_clock* clock, const double* dt, void* stream);
int gem_fluid_adv_full_dev(const gem_cfg* cfg, const gem_grid* g, double* fluidvars, double* fluidauxvars,
                           const double* electrovars, gem_work* w, const gem_source_inputs* in, double* scratch,
                           const double* dt, void* stream);

/* ---- differentiable path (no counterpart in the reference) ------------------------
 * Vector-Jacobian product of gem_energy_diffusion_dev: given Ybar, the cotangent of the
 * diffusion's output temperature (ghosted 7-species block; interior rows used, including
 * the max(T,100) floor), accumulate the cotangents of its inputs into Tbar (temperature),
 * nbar (densities; both ghosted 7-species blocks, interior rows written, caller zeroes
 * them) and, if not NULL, Ttop_bar (lx2*lx3 per species, species slowest: the exospheric
 * boundary value of each column and species).  Ts / ns are the inputs of the forward call;
 * the kernel recomputes the forward coefficients and both TRBDF2 stages, then solves the
 * transposed systems, one warp per column and species with every per-row array on chip
 * (lx1 up to about 1600). */
/* One field sweep (advec.f90:384-435 along dim, species 0..nsp-1, frank 0/1; x1 sweeps use
 * frank 0) on a caller-provided ghosted field f (nsp species blocks, updated in place) with
 * face velocities v in the reference face layout; dt is a device pointer. */
int gem_sweep_field_dev(const gem_grid* g, int dim, int frank, int nsp, double* f, const double* v,
                        const double* dt, void* stream);
/* Its vector-Jacobian product: f is the sweep's input, obar the output cotangent, fbar must
 * hold a copy of obar on entry and receives the cotangent of f; vbar (optional) receives the
 * cotangent of v. */
int gem_sweep_field_vjp_dev(const gem_grid* g, int dim, int frank, int nsp, const double* f, const double* v,
                            const double* dt, const double* obar, double* fbar, double* vbar, void* stream);
int gem_diffusion_vjp_dev(const gem_cfg* cfg, const gem_grid* g, const double* Ts, const double* ns,
                          const double* electrovars, const gem_work* w, const double* dt, const double* Ybar,
                          double* Tbar, double* nbar, double* Ttop_bar, void* stream);

/* Adjoint of one whole fused step (gem_fluid_adv_dev without compression and sources, on
 * a prescribed dt): given the state before the step (ns, vs1, vs2, vs3, Ts: ghosted
 * 7-species blocks; v1i_lo / v1i_hi: the stale x1 boundary faces of vs1i, (LSP, lx3, lx2)
 * with i2 fastest) and the cotangents of the step's outputs (ns, vs1, Ts after the step,
 * interior cells used; lo_bar_out / hi_bar_out: cotangents of the new boundary faces, may
 * be NULL), write the cotangents of ns, vs1, Ts (ghost cells 0), of the stale faces and,
 * if Ttop_bar is not NULL, of the per-column exospheric temperature set on w (lx2*lx3).
 * vs2 / vs3 are held fixed.  The step's sweeps and conversions are replayed on the
 * device; everything runs on the stream without host synchronisation or allocation.
 * Output buffers must not alias input buffers.  Grids without null cells.  The workspace
 * (about 27 ghosted 7-species fields) belongs to one grid. */
typedef struct gem_step_adjoint gem_step_adjoint;
int gem_step_adjoint_create(const gem_grid* g, gem_step_adjoint** out);
int gem_step_adjoint_destroy(gem_step_adjoint* a);
int gem_step_vjp_dev(const gem_cfg* cfg, const gem_grid* g, const gem_work* w, gem_step_adjoint* a,
                     const double* ns, const double* vs1, const double* vs2, const double* vs3, const double* Ts,
                     const double* v1i_lo, const double* v1i_hi, const double* electrovars, const double* dt,
                     const double* ns_bar_out, const double* vs1_bar_out, const double* Ts_bar_out,
                     const double* lo_bar_out, const double* hi_bar_out, double* ns_bar, double* vs1_bar,
                     double* Ts_bar, double* lo_bar, double* hi_bar, double* Ttop_bar, void* stream);

/* The same in two halves.  The replay (conversions, ghost fill, interface velocities, the
 * nine sweeps with their inputs kept, the post-sweep values) needs only the state before the
 * step, so a backward loop may replay step j-1 into a second workspace, on another stream,
 * while step j's backward runs; the backward then takes the same state pointers (ns, vs1,
 * Ts, faces) and the cotangents.  Order the two halves of one workspace on the device. */
int gem_step_vjp_replay_dev(const gem_cfg* cfg, const gem_grid* g, const gem_work* w, gem_step_adjoint* a,
                            const double* ns, const double* vs1, const double* vs2, const double* vs3,
                            const double* Ts, const double* v1i_lo, const double* v1i_hi, const double* dt,
                            void* stream);
int gem_step_vjp_backward_dev(const gem_cfg* cfg, const gem_grid* g, const gem_work* w, gem_step_adjoint* a,
                              const double* ns, const double* vs1, const double* Ts, const double* v1i_lo,
                              const double* v1i_hi, const double* electrovars, const double* dt,
                              const double* ns_bar_out, const double* vs1_bar_out, const double* Ts_bar_out,
                              const double* lo_bar_out, const double* hi_bar_out, double* ns_bar, double* vs1_bar,
                              double* Ts_bar, double* lo_bar, double* hi_bar, double* Ttop_bar, void* stream);
/* The rest of the forward step from a replayed workspace: the x2 sweep's epilogue
 * (rhov12v1, clean_param, rhoe2T) from the replay's last stage, the ghost epilogue and the
 * energy diffusion, written into fluidvars / fluidauxvars (ns, vs1, Ts and the auxiliary
 * blocks; vs2, vs3 untouched) as gem_fluid_adv_dev on the same state and dt writes them,
 * and the new x1 boundary faces into v1i_lo / v1i_hi ((LSP, lx3, lx2), i2 fastest).  A
 * checkpointed backward recomputes a segment's states with replay + finish, so each step's
 * replay serves both the recompute and that step's backward.  Call it after
 * gem_step_vjp_replay_dev on the same workspace (ordered on the device); it leaves the
 * workspace's replay intact. */
int gem_step_vjp_finish_dev(const gem_cfg* cfg, const gem_grid* g, gem_work* w, const gem_step_adjoint* a,
                            double* fluidvars, double* fluidauxvars, const double* electrovars, const double* dt,
                            double* v1i_lo, double* v1i_hi, void* stream);

/* No counterpart in the reference.  dt_calc (the same result as gem_dt_calc_dev) for callers
 * that cannot allocate device memory or hold a gem_work (for example code that runs inside
 * a pool-managed or already-captured context): it calls no allocator.  Its scratch is a
 * static device array of GEM_DT_NOALLOC_MAX_PLANES * 21 doubles (344 KiB) holding one set of
 * partial maxima per x3 plane; grids with lx3 > GEM_DT_NOALLOC_MAX_PLANES are rejected with
 * GEM_EINVAL.  The first call on each device, made with that device current, resolves the
 * scratch address (cudaGetSymbolAddress), which may initialise the module: make it before
 * any stream capture.  Nothing in the scratch has to start at zero (every partial slot read
 * is written in the same call).  All calls on one device share the one scratch array, so
 * calls whose executions overlap (on different streams or host threads) race: serialise
 * them.  The cached address belongs to the device's current context: after cudaDeviceReset
 * the entry point must not be called again in that process.  The reduction runs one block per
 * x3 plane, each scanning its plane's x2 rows in turn, so grids with few x3 planes (2-D runs
 * have one) run far slower than gem_dt_calc_dev.  Like gem_dt_calc_dev it returns the CFL step
 * floored at 1e-6. */
#define GEM_DT_NOALLOC_MAX_PLANES 2048
int gem_dt_calc_noalloc_dev(const gem_grid* g, double tcfl, const double* fluidvars, double* dt_out,
                            void* stream);

/* ---- batched instances ---------------------------------------------------------------
 * No counterpart in the reference (which runs one simulation per MPI job): n independent
 * simulations, each with its own grid, work object, state blocks (device) and gem_cfg,
 * advanced together.  One gem_batch_step = gem_dt_calc_dev(cfg.tcfl) + gem_fluid_adv_dev
 * for every instance, with the same results bit for bit.  Each phase of the step is one
 * persistent launch over an (instance, block) work list, largest instances first, and the
 * step's launches are captured once into a CUDA graph that later calls replay (on any
 * stream).  Each instance's dt is computed into its work object's dt slot (gem_work_dt).
 * The batch keeps pointers to the objects it was given: they must outlive it and must not
 * move.  Tuning parameters (gem_batch_set_param) rebuild the work lists and the graph. */
typedef struct gem_batch gem_batch;
#define GEM_BATCH_USE_GRAPH 0  /* 1 (default): capture the step into a CUDA graph */
#define GEM_BATCH_DIFF_BLOCKS 1 /* resident diffusion blocks (4 warps each) per SM, 1..4 (default 4) */
#define GEM_BATCH_GRID_PCT 2   /* persistent grid size, % of the occupancy limit (10..400);
                                  0: one block per work item (no persistence) */
int gem_batch_create(int n, const gem_grid* const* grids, gem_work* const* works, double* const* fluidvars,
                     double* const* fluidauxvars, const double* const* electrovars, const gem_cfg* cfgs,
                     gem_batch** out);
int gem_batch_destroy(gem_batch* b);
int gem_batch_size(const gem_batch* b);
int gem_batch_set_param(gem_batch* b, int param, int value);
int gem_batch_step(gem_batch* b, void* stream);
/* The same step with prescribed time steps (host array of n values, copied to the device on
 * `stream` before the step): dt_calc is skipped and instance i advances by host_dts[i].
 * Used by the differentiable path, whose time steps follow a frozen schedule. */
int gem_batch_step_fixed_dt(gem_batch* b, const double* host_dts, void* stream);
/* per-instance dt of the last step (synchronous device->host copies) */
int gem_batch_dts(const gem_batch* b, double* host_dt);
/* launches per step and (instance, block) work items per step */
int gem_batch_info(const gem_batch* b, int* launches_per_step, long long* items_per_step);

/* ---- the fused fluid advance --------------------------------------------------------
 * One call = the advection + diffusion subset of fluid_adv (app/main.f90:280-355,
 * libgemini.cpp:155-210) with compression and sources excluded:
 *   v12rhov1, T2rhoe, set_global_boundaries, halo, interface_vels, sweep3, sweep1, halo,
 *   sweep2, rhov12v1, clean_param(1), clean_param(2), rhoe2T, clean_param(3),
 *   energy_diffusion, clean_param(3), T2rhoe.
 * Asynchronous on `stream`; dt is a device pointer (e.g. written by gem_dt_calc_dev).  Of
 * the work arrays only the x1 boundary faces of vs1i are kept current (the only part read
 * by the next step); gem_interface_vels_allspec_dev fills all faces. */
int gem_fluid_adv_dev(const gem_cfg* cfg, const gem_grid* g, double* fluidvars, double* fluidauxvars,
                      const double* electrovars, gem_work* w, const double* dt, void* stream);

/* The same step through host buffers: copies what the step reads to the device (fluidvars
 * and the J1 field of electrovars), runs gem_dt_calc_dev (if dt_inout < 0, else uses
 * *dt_inout) and gem_fluid_adv_dev, copies back what it writes and synchronises.  The host
 * blocks end exactly as a full round trip would leave them: rhovs1 and rhoes are recomputed
 * from fluidvars over every cell, vs2 and vs3 change only in their ghost cells (so only
 * their ghost shell is copied back), and the 9 MHD scalars and the other electrovars fields
 * are not touched.  The copies back run on a stream of the work object beside the step,
 * each block once the step is done with it (vs2, vs3 after the ghost fill; ns, vs1, rhovs1
 * before the diffusion; Ts, rhoes at the end); pinned host blocks let them overlap the
 * step.  Device staging buffers are allocated on first use and kept in the work object. */
int gem_fluid_adv_host(const gem_cfg* cfg, const gem_grid* g, double* fluidvars, double* fluidauxvars,
                       const double* electrovars, gem_work* w, double* dt_inout, void* stream);

/* Optional per-phase timing of gem_dt_calc_dev + gem_fluid_adv_dev with CUDA events
 * recorded on the launching stream (no synchronisation inside the step).  Phases:
 * 0 dt_calc, 1 ghost fill, 2 x3 sweep, 3 x1 sweep, 4 x2 sweep + epilogue, 5 ghost-cell
 * epilogue, 6 diffusion.  gem_work_phase_timing(w, n) keeps events for up to n steps
 * (0 turns it off); gem_work_phase_times waits for them, returns the mean milliseconds per
 * step of each phase and restarts the count. */
int gem_work_phase_timing(gem_work* w, int max_steps);
int gem_work_phase_times(gem_work* w, double* ms, int nphase_max, int* nphase, int* nsteps);

/* number of non-finite values in the interior of ns, vs1 and Ts (blocks until done) */
int gem_check_finite(const gem_grid* g, const double* fluidvars, gem_work* w, long long* count,
                     void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GEM_FLUID_H */
