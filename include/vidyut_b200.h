/*
 * vidyut_b200.h -- C ABI of the B200-native per-timestep species-and-field
 * update of Vidyut3d on one uniform grid level.
 *
 * The reference has no runtime plugin API: its step is the member function
 * Vidyut::Evolve (Source/Evolve.cpp:69-714) calling solve_potential,
 * update_rxnsrc_at_all_levels, update_explsrc_at_all_levels,
 * compute_elecenergy_source and implicit_solve_scalar, all driven by
 * ParmParse parameters (Source/Vidyut.cpp:358-536) and by case hook headers
 * compiled into the executable.  This header is the C boundary a host
 * driver (C++, or any language with a C FFI) uses in place of that member
 * function.  Case hooks stay compile-time: one shared library is built per
 * case directory, as the reference builds one executable per case.
 *
 * Conventions:
 *   - every function returns a vd_status (0 = VD_OK);
 *   - state arrays are FP64, one component after another, x fastest
 *     (index = i + nx*(j + ny*k) + comp*nx*ny*nz), the layout of one AMReX
 *     box's Array4; component numbering is the reference's
 *     (Source/VarDefines.H:5-38), reported by vd_case_info;
 *   - pointers flagged `on_device` are CUDA device pointers on the
 *     context's device, otherwise host pointers; the caller keeps ownership;
 *   - all work is ordered on one stream owned by the context; a context is
 *     not thread-safe; functions return after the work is complete.
 */
#ifndef VIDYUT_B200_H
#define VIDYUT_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define VD_MAX_SPECIES 64

typedef enum vd_status {
    VD_OK = 0,
    VD_ERR_INVALID_ARG = 1,
    VD_ERR_CUDA = 2,
    VD_ERR_NOT_CONVERGED = 3,
    VD_ERR_UNSUPPORTED = 4,
    VD_ERR_OOM = 5,
    VD_ERR_NONFINITE = 6
} vd_status;

/* Multigrid precision of the two linear solves. */
#define VD_MG_FP64 0          /* FP64 V-cycles (the reference's scheme)   */
#define VD_MG_FP32_REFINED 1  /* FP32 V-cycles inside FP64 refinement     */

/*
 * Run parameters.  Field names are the reference's ParmParse names
 * (prefix `vidyut.` unless noted); defaults are the reference's
 * (Source/Vidyut.H:250-400) and are set by vd_config_init.
 */
typedef struct vd_config {
    /* geometry.* and amr.n_cell (single level, no AMR) */
    int dim;                 /* 2 or 3: the reference's DIM build switch   */
    int n_cell[3];
    double prob_lo[3];
    double prob_hi[3];
    int is_periodic[3];

    /* time stepping: Source/TimeStep.cpp:14-43, Source/Evolve.cpp:214-617 */
    double dt;               /* the fixed step (the reference's fixed_dt)  */
    int num_timestep_correctors;
    /* adaptive step (Source/TimeStep.cpp:14-134, Source/Vidyut.cpp:388-398):
       with adaptive_dt and time > adaptive_dt_delay each step takes
       min(dt_prev * dt_stretch, clamp(min(advective_cfl dt_edrift,
       diffusive_cfl dt_ediff, dielectric_cfl dt_diel_relax), dt_min,
       dt_max)) from the electron time scales of the state it starts from */
    /* semi-implicit electron-Poisson coupling (Source/Evolve.cpp:281-352,
       Source/PotentialSolve.cpp:262-343): the electron solve precedes the
       potential solve, whose operator gets b = -(1 + dt/tau_diel) and whose
       right-hand side the electron density change; repeated
       electron_poisson_maxiters times per corrector iteration */
    int electron_poisson_coupling;
    int electron_poisson_maxiters;
    int adaptive_dt;
    double advective_cfl;
    double diffusive_cfl;
    double dielectric_cfl;
    double dt_min;
    double dt_max;
    double adaptive_dt_delay;
    double dt_stretch;

    /* drift flux: Source/compute_explicit_flux.H:218-415 */
    int hyp_order;           /* 1 upwind, 2 WAF/MINBEE, 5 WENO5            */
    int weno_scheme;         /* 1 JS, 2 M, 3 Z                             */

    /* physics switches */
    int do_reactions;
    int do_transport;
    int do_spacechrg;
    int elecenergy_solve;
    int using_LFA;
    int floor_jh;
    int bound_specden;
    int do_bg_reactions;
    int user_defined_potential;
    int user_defined_species;
    int user_defined_vel;
    double min_species_density;
    double min_electron_density;
    double min_electron_temp;
    double gas_temperature;
    double gas_pressure;

    /* boundary-condition codes PERBC..AXISBC = 0..5 (Source/VarDefines.H:40-45) */
    int pot_bc_lo[3], pot_bc_hi[3];
    int eden_bc_lo[3], eden_bc_hi[3];
    int eenrg_bc_lo[3], eenrg_bc_hi[3];
    int ion_bc_lo[3], ion_bc_hi[3];
    int neutral_bc_lo[3], neutral_bc_hi[3];

    /* applied voltage: Source/HelperFuncs.H:125-161 */
    int voltage_profile;
    double voltage_amp_lo[3];
    double voltage_amp_hi[3];
    double voltage_freq;
    double voltage_dur;
    double voltage_center;

    /* linear solvers (MLMG settings of Source/Vidyut.H:264-284) */
    double linsolve_reltol;
    double linsolve_abstol;
    double linsolve_bot_reltol;
    double linsolve_bot_abstol;
    int linsolve_num_pre_smooth;
    int linsolve_num_post_smooth;
    int linsolve_num_final_smooth;
    int linsolve_num_bottom_smooth;
    int linsolve_maxiter;
    int linsolve_max_coarsening_level;

    /* equation scaling: Source/Vidyut.cpp:480-500 */
    double potential_scale;
    double elecenergy_scale;
    double time_scale;
    double species_scale[VD_MAX_SPECIES];

    int num_bg_species;
    int bg_species_ids[VD_MAX_SPECIES];

    /* B200 additions with no counterpart in the reference */
    int mg_precision;        /* VD_MG_FP64 or VD_MG_FP32_REFINED           */
    int mg_inner_cycles;     /* FP32 V-cycles per FP64 refinement pass     */
    int poisson_warm_start;  /* 1: start the Poisson solve from the last
                                potential (reference: zero guess,
                                Source/PotentialSolve.cpp:479-485)       */
    int device;              /* CUDA device ordinal                        */

    /* multicomponent species solves (Source/Evolve.cpp:458-573,
       Source/Vidyut.cpp:146-186): ions and neutrals solved in chunks of
       comp_ion_chunks / comp_neutral_chunks consecutive components, each
       chunk as one multigrid solve whose stopping test and bottom BiCGStab
       inner products run over all of its components; background species in
       the neutral range take part and are then reset to the step's starting
       value (defaults: off, chunks NUM_IONS and NUM_NEUTRALS) */
    int multicompsolves;
    int comp_ion_chunks;
    int comp_neutral_chunks;
} vd_config;

typedef struct vd_case_info_t {
    int num_species;
    int nvar;
    int e_id;
    int een_id, etemp_id, pot_id, efx_id, ref_id, ejh_id, eih_id, cmask_id;
    int charge[VD_MAX_SPECIES];
    char names[VD_MAX_SPECIES][16];
    char case_name[64];
} vd_case_info_t;

typedef struct vd_solve_stats {
    int iterations;          /* V-cycles (FP32-refined: inner V-cycles)    */
    int refinements;         /* FP64 refinement passes (FP32-refined mode) */
    int converged;
    double initial_residual; /* max-norm, in the solver's scaled units     */
    double final_residual;
} vd_solve_stats;

typedef struct vd_step_stats {
    int steps;
    int poisson_iterations;  /* summed over the steps                      */
    int species_iterations;
    int not_converged;       /* solves that hit linsolve_maxiter           */
    double max_poisson_final_residual;
    double time;             /* simulation time after the last step        */
    double gpu_ms;           /* device time of the steps (CUDA events on
                                the context's stream)                     */
    double dt;               /* step size of the last step                 */
    double dt_edrift;        /* electron time scales of the last step's    */
    double dt_ediff;         /* starting state (adaptive_dt only; DBL_MAX  */
    double dt_diel_relax;    /* where undefined): Source/TimeStep.cpp:46-134 */
    int poisson_refinements; /* FP64 refinement passes of the potential
                                solves (FP32-refined form), summed        */
} vd_step_stats;

/* Kernels that vd_profile_kernel can time launch by launch. */
#define VD_PROF_NONE 0
#define VD_PROF_POISSON_SMOOTH 1     /* FP64 Poisson fine-level RB sweeps   */
#define VD_PROF_EXPLICIT 2           /* fused reaction + drift-flux kernel   */
#define VD_PROF_POISSON_SMOOTH32 3   /* FP32 Poisson fine-level RB sweeps   */
#define VD_PROF_EFIELD 4             /* E = -grad(phi), E/N, potential out   */
#define VD_PROF_POISSON_RHS 5        /* Poisson right-hand side + guess      */
#define VD_PROF_SPECIES_RHS 6        /* implicit-diffusion right-hand side   */

/* Reference defaults (Source/Vidyut.H:250-400). */
vd_status vd_config_init(vd_config* cfg);

/* Set one parameter by its inputs-file name, e.g. ("vidyut.hyp_order", "5"),
 * ("amr.n_cell", "256 256 256"), ("geometry.prob_hi", "0.02 0.02 0.02").
 * Replaces ParmParse in Vidyut::ReadParameters (Source/Vidyut.cpp:358-536)
 * and the BC arrays of the constructor (Source/Vidyut.cpp:97-114). */
vd_status vd_config_set(vd_config* cfg, const char* key, const char* value);

/* Species count, component numbering and names of the compiled-in case
 * (CKSYMS_STR / CKCHRG, Source/PlasmaChem.cpp:11-18). */
vd_status vd_case_info(vd_case_info_t* info);

/* Allocate a context: device state (NVAR components), multigrid
 * hierarchy, work arrays.  Replaces the Vidyut constructor and level
 * allocation (Source/Vidyut.cpp:27-218, Source/GridWork.cpp:68-109). */
vd_status vd_create(const vd_config* cfg, void** ctx);
vd_status vd_destroy(void* ctx);

/* amrex_probinit + initdomaindata of the case (Source/Vidyut.cpp:30-32,
 * Source/GridWork.cpp:94-104): `prob_inputs` is inputs-file text carrying
 * the `prob.*` parameters; time and step count are reset to 0. */
vd_status vd_init_domain(void* ctx, const char* prob_inputs);

/* Copy components [comp, comp+ncomp) of the state in or out. */
vd_status vd_set_state(void* ctx, int comp, int ncomp, const double* src, int on_device);
vd_status vd_get_state(void* ctx, int comp, int ncomp, double* dst, int on_device);

vd_status vd_set_time(void* ctx, double time, int step);
vd_status vd_get_time(void* ctx, double* time, int* step);

/* The current step size: the dt[] entry of a checkpoint
 * (Vidyut::WriteCheckpointFile / ReadCheckpointFile, Source/Plot.cpp:103-108,
 * 157-166).  It is the previous step's dt that an adaptive step stretches;
 * without adaptive_dt every step takes the configured (fixed) dt. */
vd_status vd_set_dt(void* ctx, double dt);
vd_status vd_get_dt(void* ctx, double* dt);

/* Advance `nsteps` coarse steps: the body of Vidyut::Evolve for one level
 * (Source/Evolve.cpp:136-617), with the fixed dt or, with adaptive_dt, the
 * step of Vidyut::ComputeDt (Source/TimeStep.cpp:14-134). */
vd_status vd_step(void* ctx, int nsteps, vd_step_stats* stats);

/* Sub-stages, each on the current state (used as both Sborder and
 * Sborder_old):
 *   vd_poisson_solve       Vidyut::solve_potential (Source/PotentialSolve.cpp:19-554):
 *                          writes Potential, Efield{x,y,z}, ReducedEF.
 *   vd_explicit_rhs        update_rxnsrc_at_all_levels (Source/ScalarSolve.cpp:156-216)
 *                          followed by update_explsrc_at_all_levels
 *                          (Source/ScalarSolve.cpp:81-154) for every
 *                          transported species and, with elecenergy_solve,
 *                          the electron energy: NUM_SPECIES+1 components out
 *                          (no Joule heating; untransported species are 0).
 *   vd_implicit_diffusion  Vidyut::implicit_solve_scalar for one species
 *                          (Source/ScalarSolve.cpp:380-1000) with `expl_src`
 *                          (NUM_SPECIES+1 components) as dsdt_expl: writes
 *                          the species (and Electron_Temp for the energy). */
vd_status vd_poisson_solve(void* ctx, double time, vd_solve_stats* stats);
vd_status vd_explicit_rhs(void* ctx, double time, double* expl_src, int on_device);
vd_status vd_implicit_diffusion(void* ctx, int specid, double time,
                                const double* expl_src, int on_device,
                                vd_solve_stats* stats);

/* Vidyut::implicit_solve_scalar with numspec > 1 (Source/ScalarSolve.cpp:
 * 380-1000, as Source/Evolve.cpp:458-533 calls it for a chunk of ions or
 * neutrals): species [startspec, startspec + numspec) solved together, one
 * multigrid solve whose stopping test (max-norm) and bottom BiCGStab inner
 * products run over all of them; writes every species of the chunk (floored
 * like the reference).  numspec = 1 is vd_implicit_diffusion.  Chunks of
 * more than one species need a 3-D non-periodic grid whose coarsest level
 * holds at most 32 cells (VD_ERR_UNSUPPORTED otherwise). */
vd_status vd_implicit_diffusion_chunk(void* ctx, int startspec, int numspec, double time,
                                      const double* expl_src, int on_device,
                                      vd_solve_stats* stats);

/* Count of non-finite values in the species, energy and potential
 * components (a host-side check in place of amrex::Abort on NaN). */
vd_status vd_check_state(void* ctx, long long* nonfinite);

/* Per-kernel launch counter (for the benchmark's launch accounting). */
vd_status vd_launch_count(void* ctx, long long* launches);

/* Time the launches of one kernel (VD_PROF_*) with CUDA events recorded on
 * the context's stream, until the next vd_profile_kernel call (the
 * multigrid sweeps: one event pair around each run of consecutive sweeps,
 * so that the events do not break their programmatic overlap; the explicit
 * kernel: one pair around the explicit stage of a step);
 * vd_profile_read returns the launches timed, their summed device time and
 * the kernel's algorithmic bytes per launch (one read of each distinct input
 * array, one write of each output); launches that returned at once on a
 * solve's stop flag (a multigrid cycle enqueued past convergence; shorter
 * than a quarter of the median launch) did no work and are left out. */
vd_status vd_profile_kernel(void* ctx, int kernel_id);
vd_status vd_profile_read(void* ctx, long long* launches, double* total_ms,
                          double* bytes_per_launch);

/* Message of the last failing call on this context (or the last failing
 * vd_create when ctx is NULL). */
vd_status vd_last_error(void* ctx, char* buf, int len);

/* Discrete adjoint of N explicit flux + source steps.  No counterpart in the
 * reference (which has no sensitivities); it differentiates this map of the
 * transported (non-background) species u, from the current state:
 *   u <- u + dt ( -div F(u; p_mob) + N_A wdot(u; theta) )
 * F the drift flux of vd_explicit_rhs's schemes (hyp_order, weno_scheme)
 * with v = mu(Te, n_total, |E|) E, the electron mobility times p_mob; ghost
 * cells by clamping (periodic wrap where periodic), zero flux on IHNEUBC and
 * AXISBC walls; E, Te and the background species frozen at the current
 * state; wdot the case's mechanism with every pre-factor A_r multiplied by
 * exp(theta_r).  The state itself is not changed.
 * Objective VD_ADJ_OBJ_ELECTRONS: total electron count sum n_e dV after the
 * last step.  Parameters: theta_0 .. theta_{R-1} (R = reactions), then
 * p_mob; defaults 0 and 1.
 *   vd_adjoint_num_params   R + 1, or 0 when the case's mechanism has no
 *                           differentiable form (the adjoint calls then
 *                           return VD_ERR_UNSUPPORTED);
 *   vd_adjoint_forward      the objective after nsteps steps; species_out
 *                           (optional, host) receives the final u, one
 *                           component of N cells after another in component
 *                           order;
 *   vd_adjoint_run          objective and gradient (n_params entries):
 *                           forward with a device checkpoint every K steps,
 *                           backward with each K-block recomputed from its
 *                           checkpoint ((nsteps/K + max(K,2)) state copies
 *                           of device memory). */
#define VD_ADJ_OBJ_ELECTRONS 0
vd_status vd_adjoint_num_params(void* ctx, int* n_params);
vd_status vd_adjoint_set_params(void* ctx, const double* params, int n_params);
vd_status vd_adjoint_forward(void* ctx, int nsteps, int objective_id, double* objective,
                             double* species_out);
vd_status vd_adjoint_run(void* ctx, int nsteps, int K, int objective_id, double* objective,
                         double* grad_out, int n_params);

/* Poisson solve that allocates no device memory.  No counterpart in the
 * reference: it serves callers that must not allocate device memory while
 * they run, e.g. a host framework whose own memory pool owns the whole
 * device, or code that cannot afford an allocation's implicit device
 * synchronisation.  It solves del^2 phi = rhs (the field solve's operator,
 * second-order Dirichlet closure) with the same red-black multigrid as
 * vd_poisson_solve and the same convergence test, on the current device.
 *   rhs, phi   caller-owned device arrays of n_cell[0]*n_cell[1]*n_cell[2]
 *              doubles, x fastest; phi holds the initial guess on entry and
 *              the solution on return;
 *   bc_lo/hi   PERBC, DIRCBC or HNEUBC per direction; bcval_lo/hi the
 *              Dirichlet face values (may be NULL for all zero);
 *   err        optional buffer for a message (NULL to skip).
 * Its multigrid scratch is one fixed array of 8 MiB per device, built into
 * the library and held by every device that loads it until the process
 * exits; grids needing more (above about 128^3 cells) are rejected with
 * VD_ERR_INVALID_ARG and a message saying how much they need.  Every call
 * looks up that array's device address with the caller's device current
 * (the lookup allocates nothing).  With lazy module loading
 * (CUDA_MODULE_LOADING=LAZY, the default of recent CUDA releases) the first
 * call on a device may be the one that loads the library's device code and
 * with it the 8 MiB array, so make that first call before any stream
 * capture.  Work runs on the legacy default stream; every call reuses the
 * same scratch, so calls that overlap on one device race and must be
 * serialised by the caller. */
vd_status vd_poisson_solve_noalloc(int dim, const int* n_cell, const double* dx,
                                   const int* bc_lo, const int* bc_hi,
                                   const double* bcval_lo, const double* bcval_hi,
                                   const double* rhs, double* phi, double reltol,
                                   double abstol, int maxiter, vd_solve_stats* stats,
                                   char* err, int errlen);

#ifdef __cplusplus
}
#endif

#endif /* VIDYUT_B200_H */
