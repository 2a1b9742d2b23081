/*
 * fhd_b200.h -- C ABI of the B200 (sm_100a) staggered-grid Stokes solver and
 * stochastic flux library.
 *
 * The entry points replace, one for one, the hot-path routines of LowMachFHD
 * (staggered_grid/src_gmres, src_lowMach).  Every declaration cites the
 * reference routine it stands in for.  Two families exist:
 *
 *   fhd_dev_*  : operands are DEVICE pointers in the canonical layout below.
 *                This is what device-resident callers (the time integrator,
 *                batched and served solves) use.
 *   fhd_*      : operands are HOST BoxLib fabs (Fortran column-major with
 *                ghost cells, duplicated periodic faces).  This is the
 *                drop-in boundary a Fortran driver binds through
 *                iso_c_binding: same argument meaning as the reference.
 *
 * Canonical device layout (periodic domain, one box):
 *   n = (nx, ny, nz) cells, nz = 1 in 2D; Nc = nx*ny*nz.
 *   cell (i,j,k)  -> offset i + nx*(j + ny*k)
 *   face array of direction d: Nc entries, entry (i,j,k) is the face on the
 *       low-d side of cell (i,j,k) (periodic faces stored once).
 *   2D node array: entry (i,j) is the node at the low-x, low-y corner.
 *   3D edge arrays, order xy, xz, yz: entry (i,j,k) of the xy array is the
 *       edge at the low-x, low-y corner, centred in z (likewise xz, yz).
 * All arrays are FP64 at the boundary.
 *
 * Status codes: 0 = success, > 0 = warning (result usable), < 0 = error.
 */
#ifndef FHD_B200_H
#define FHD_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* status codes                                                        */
/* ------------------------------------------------------------------ */
#define FHD_OK                          0
#define FHD_WARN_NOT_CONVERGED_MAXITER  1  /* gmres.f90:268-274 */
#define FHD_WARN_NOT_CONVERGED_OUTER    2  /* gmres.f90:305-310 */
#define FHD_WARN_TRUE_RESID             3  /* gmres.f90:286-289 */
#define FHD_ERR_BAD_ARG                -1
#define FHD_ERR_BAD_GHOSTS             -2  /* apply_matrix.f90:54-68 */
#define FHD_ERR_DX_NOT_ISOTROPIC       -3  /* stag_applyop.f90:118-128 */
#define FHD_ERR_ORTHO_BREAKDOWN        -4  /* gmres.f90:391 */
#define FHD_ERR_UNSUPPORTED            -5  /* apply_precon.f90:426 */
#define FHD_ERR_NONFINITE              -6
#define FHD_ERR_OOM                    -7
#define FHD_ERR_CUDA                   -8
#define FHD_ERR_NO_DEVICE              -9

/* precision modes of a context */
#define FHD_PREC_FP64   0  /* everything in FP64 */
#define FHD_PREC_MIXED  1  /* FP32 multigrid preconditioner and stochastic
                              fluxes; FP64 outer residual, Arnoldi/Givens,
                              mean-zero projection */

/* ------------------------------------------------------------------ */
/* parameters: mirror of namelist probin_gmres (probin_gmres.f90:12-163)*/
/* ------------------------------------------------------------------ */
typedef struct fhd_gmres_params {
    int    precon_type;            /* 1..5 and negatives */
    int    visc_schur_approx;      /* 0 simple Schur complements; 1 BFBt (|visc_type| 1, 2) */
    double p_norm_weight;
    double scale_factor;
    int    mg_verbose, cg_verbose;
    int    mg_max_vcycles, mg_minwidth, mg_bottom_solver;
    int    mg_nsmooths_down, mg_nsmooths_up, mg_nsmooths_bottom;
    int    mg_max_bottom_nlevels;
    double mg_rel_tol, mg_abs_tol;
    int    stag_mg_verbosity, stag_mg_max_vcycles, stag_mg_minwidth;
    int    stag_mg_bottom_solver;
    int    stag_mg_nsmooths_down, stag_mg_nsmooths_up, stag_mg_nsmooths_bottom;
    int    stag_mg_max_bottom_nlevels;
    double stag_mg_omega;
    int    stag_mg_smoother;       /* 0 = Jacobi, 1 = 2*dim-colour Gauss-Seidel */
    double stag_mg_rel_tol;
    double gmres_rel_tol, gmres_abs_tol;
    int    gmres_verbose, gmres_max_outer, gmres_max_inner;
    int    gmres_max_iter, gmres_min_iter;
    int    gmres_spatial_order;    /* 2, or 4 with visc_type 1 (apply_matrix only) */
} fhd_gmres_params;

/* Fills the defaults of probin_gmres_init (probin_gmres.f90:122-163). */
void fhd_gmres_params_default(fhd_gmres_params* p);

/* Stochastic momentum flux parameters (probin_common: k_B,
 * variance_coef_mom, stoch_stress_form, filtering_width;
 * stochastic_m_fluxdiv.f90:137).  dV is the cell volume product(dx)
 * (in 2D: dx*dy*cell_depth). */
typedef struct fhd_stoch_params {
    double k_B;
    double variance_coef_mom;
    double dV;
    int    stoch_stress_form;      /* 0 non-symmetric, 1 symmetric */
    int    filtering_width;        /* 0 off; 1, 2 or 4: the stress filter of
                                      filter_stoch_m_flux (stochastic_m_fluxdiv.f90:
                                      604-778), periodic boxes only (walls:
                                      FHD_ERR_UNSUPPORTED); another width, or one
                                      above a domain side: FHD_ERR_BAD_ARG */
} fhd_stoch_params;

/* Multispecies mixture parameters (namelist probin_multispecies,
 * probin_multispecies.f90:100-140): ideal isothermal mixture, constant
 * Maxwell-Stefan coefficients (mixture_type 0).  Dbar holds the
 * nspecies*(nspecies-1)/2 off-diagonal entries in the order
 * (2,1),(3,1),(3,2),(4,1),... of compute_D_bar_local
 * (compute_mixture_properties.f90:217-273). */
#define FHD_MAX_SPECIES 8
typedef struct fhd_mixture_params {
    int    nspecies;
    double molmass[FHD_MAX_SPECIES];
    double Dbar[FHD_MAX_SPECIES * (FHD_MAX_SPECIES - 1) / 2];
    double rhobar[FHD_MAX_SPECIES];
    double variance_coef_mass;
    int    chi_iterations;         /* Dbar2chi_iterative iterations (10) */
    double fraction_tolerance;     /* trace-species threshold (1e-14) */
    int    correct_flux;           /* last species = -sum of the others */
    int    avg_type;               /* compute_nonnegative_rho_av: 1,2,3,10 */
} fhd_mixture_params;

/* Per-solve diagnostics (gmres.f90:72-85 locals, vcycle_counter.f90). */
typedef struct fhd_solve_stats {
    int    outer_iters;            /* gmres 'iter' */
    int    total_iters;            /* gmres 'total_iter' */
    int    vcycles;                /* vcycle_counter */
    int    status;
    double norm_b, norm_pre_b, norm_init_resid, norm_resid;
    double norm_resid_Stokes, norm_init_Stokes, norm_resid_est;
} fhd_solve_stats;

/* ------------------------------------------------------------------ */
/* context                                                             */
/* ------------------------------------------------------------------ */
typedef struct fhd_ctx fhd_ctx;

/* Builds the solver for one periodic box: multigrid hierarchy
 * (stag_mg_layout_build + compute_nlevs_mg, stag_mg_layout.f90:21-222;
 * mgt_macproj_precon_build, macproject.f90:364-421), Krylov storage and a
 * CUDA stream.  dim = 2 or 3; dx must be equal in all directions
 * (stag_applyop.f90:118-128).  visc_type in {-3,-2,-1,1,2,3}
 * (probin_common visc_type). */
int  fhd_ctx_create(int dim, const int n_cells[3], const double dx[3],
                    int visc_type, const fhd_gmres_params* params,
                    int precision_mode, fhd_ctx** out);
/* The same context with the layout arguments of the driver's set-up
 * (probin_common max_grid_size, bc_lo, bc_hi; main_driver.f90:392-393).
 * bc codes (bc.f90:24-44): FHD_BC_PERIODIC (-1), FHD_BC_NO_SLIP_WALL (100)
 * and FHD_BC_SLIP_WALL (200); a direction is periodic on both sides or on
 * neither.  The Stokes solve sees homogeneous walls (zero wall velocity)
 * through the ghost rules of multifab_physbc_domainvel /
 * multifab_physbc_macvel (multifab_physbc_stag.f90:91-1116); moving no-slip
 * walls enter the timesteps only (fhd_ctx_set_wall_speed).  Walls are
 * built for visc_type 1, 2 or 3, precon_type 1 without the BFBt Schur complement,
 * the colour smoother, gmres_spatial_order 2 and one box; the device and
 * host-fab flux entries and the timesteps carry the wall rules of their
 * parts.  Reservoir codes 101 and 201 are walls here
 * (FHD_BC_NO_SLIP_RESERVOIR).  In a wall
 * direction a face array keeps n faces: face 0 is the low wall face (held at
 * zero) and the high wall face is not stored.  Reservoirs and other codes
 * return FHD_ERR_UNSUPPORTED.
 * max_grid_size[d] (>= 1; below n_cells[d] it must divide it) sets the box
 * layout the reference's staggered multigrid follows: with several boxes
 * its hierarchy stops at the boxes' depth (compute_nlevs_mg over the boxes,
 * stag_mg_layout.f90:179-222), and with stag_mg_bottom_solver 4 and
 * n_cells/max_grid_size >= 2 in every direction its bottom is the "fancy"
 * nested solve over the deeper levels of the domain (stag_mg_solver.f90:
 * 447-555).  The pressure multigrid is FBoxLib's in the reference and keeps
 * the whole-domain hierarchy here. */
#define FHD_BC_PERIODIC (-1)
#define FHD_BC_NO_SLIP_WALL 100
#define FHD_BC_SLIP_WALL 200
/* Reservoirs (bc.f90): walls for the velocity, the pressure and the
 * stochastic momentum flux, as the reference's bc tower and mflux_bc treat
 * them; their mass exchange is not built, so the mass-flux entries and the
 * multispecies steps return FHD_ERR_UNSUPPORTED on such a context. */
#define FHD_BC_NO_SLIP_RESERVOIR 101
#define FHD_BC_SLIP_RESERVOIR 201
int  fhd_ctx_create_bc(int dim, const int n_cells[3], const int max_grid_size[3],
                       const int bc_lo[3], const int bc_hi[3], const double dx[3],
                       int visc_type, const fhd_gmres_params* params,
                       int precision_mode, fhd_ctx** out);
int  fhd_ctx_destroy(fhd_ctx* ctx);
/* CUDA stream (cudaStream_t) the context launches on; may be set by the
 * caller before any call (NULL = the context's own stream). */
void* fhd_ctx_stream(fhd_ctx* ctx);
int  fhd_ctx_set_stream(fhd_ctx* ctx, void* stream);
/* Preconditioner applications inside GMRES as CUDA graphs: the first
 * application for given operands and prepared coefficients is captured, later
 * ones replay it (mode 1 on, 0 off, -1 default: on unless a multigrid
 * runs more than one V-cycle per application).  Mode 2 also replays each
 * GMRES inner iteration (matrix apply, preconditioner, Gram-Schmidt passes,
 * normalisation, Hessenberg column copy) as one graph per iteration index:
 * one launch per iteration, worth its capture cost when a context runs many
 * solves of small problems.  fhd_ctx_profile timing works in every mode. */
int fhd_ctx_set_graphs(fhd_ctx* ctx, int mode);
/* The coarse end of both multigrid V-cycles (every level from the first
 * whose unknowns, right-hand sides and residuals fit in one SM's shared
 * memory down to the bottom) as one single-block kernel per V-cycle instead
 * of one launch per smoother colour and transfer (mode 1 or -1 default: on,
 * 0: per-level launches).  Same arithmetic either way.  Replaces no
 * reference routine: the levels are those of stag_mg_solver.f90:301-599 and
 * of the pressure multigrid behind macproject.f90:294-298. */
int fhd_ctx_set_coarse(fhd_ctx* ctx, int mode);
/* Whole smooths (both colours of every component) of the large FP32 levels
 * of a visc_type 1 staggered multigrid as one row-tile launch each, staged
 * by the bulk-copy engine, instead of one launch per colour (mode 1 or -1
 * default: on where the level allows, 0: colour launches).  The colour
 * sweeps of stag_mg_solver.f90:360-396, evaluated in the same order. */
int fhd_ctx_set_fused(fhd_ctx* ctx, int mode);
/* Moving no-slip walls: the namelist arrays wallspeed_lo / wallspeed_hi of
 * probin_common, in their Fortran layout (MAX_SPACEDIM-1, MAX_SPACEDIM):
 * element [t + 2 d] is the speed of the t-th tangential velocity component
 * (the components other than d, ascending) on the wall normal to direction d
 * -- the constant values of inhomogeneous_bc_val_2d / _3d
 * (src_lowMach/inhomogeneous_bc_val.f90:84-145, 274-372; not the prob_type
 * 12 profiles).  The timesteps (fhd_dev_advance_overdamped, _inertial,
 * _inertial_multispecies) then take each diffusive_m_fluxdiv of their
 * velocity with the tangential ghost 2 v_bc - u behind those walls
 * (physbc_macvel_*_inhomogeneous, multifab_physbc_stag.f90:1118-1160),
 * which puts their solves in delta form with homogeneous walls
 * (advance_timestep_inertial.f90:408-440).  The Stokes-solve entries stay
 * homogeneous, as gmres and apply_matrix are in the reference.  A speed on
 * a periodic side is ignored; a nonzero speed on a slip wall (where the
 * reference reads a traction) returns FHD_ERR_UNSUPPORTED.  Zero speeds
 * (the default) are the standing walls. */
int fhd_ctx_set_wall_speed(fhd_ctx* ctx, const double wallspeed_lo[6], const double wallspeed_hi[6]);
/* Smoother autotuner.  Each multigrid level that smooths through launches
 * (staggered and pressure multigrids, above the single-block coarse end) can
 * smooth as colour launches with one of four thread-block shapes, as the
 * tiled fused smooth with one of several tile sizes (3D), or as the row-tile
 * smooth with one of the tile heights that fit, one CTA per SM with a deep
 * copy ring (256 or 512 compute threads) or two with a short one (3D FP32
 * visc_type 1).  With
 * the tuner on (mode 1 or -1 default), the first solve call that meets a
 * level shape times every candidate on scratch unknowns with the level's
 * coefficients and keeps the fastest for the process (per device,
 * precision, visc_type and shape); later calls and contexts reuse it.
 * Mode 0: the fixed size rules of fhd_ctx_set_fused.  Mode 2 + k: candidate
 * k of every level (its first where it has fewer), untimed, for tests.
 * Every candidate evaluates the update expression of the colour sweeps of
 * stag_mg_solver.f90:360-396 (pressure: the red-black Gauss-Seidel of the
 * macproject multigrid) in the same order; the choice changes time only. */
int fhd_ctx_set_tune(fhd_ctx* ctx, int mode);
/* Plan of staggered (which 0) or pressure (which 1) multigrid level `level`
 * after the last solve call: kind -1 fixed rules, 0 colour launches, 1 tiled
 * fused, 2 row-tile; ncand candidates considered; pair_us the measured time
 * of one smooth pair (0 when not timed); shape = {block x, block y, 0, 1,
 * threads} for colour launches, {tile x, tile y, z-runs, CTAs per SM,
 * compute threads} for fused smooths.  Any output pointer may be NULL.  No
 * reference counterpart. */
int fhd_ctx_tune_info(fhd_ctx* ctx, int which, int level, int* kind, int* ncand, double* pair_us,
                      int shape[5]);
/* The candidate list the tuner would time for one level (host only, no
 * device): staggered (which 0) or pressure (1) multigrid, extents, precision
 * mode, visc_type, and the device's SM count and shared-memory limits (per
 * block opt-in, per SM).  Writes up to max_out records of 7 ints {kind (as
 * fhd_ctx_tune_info), block x | tile x | nx, block y | tile y, z-runs, CTAs
 * per SM, row-tile shared-memory bytes, threads} and returns the number of
 * candidates.  No reference counterpart. */
int fhd_tune_candidates(int which, int dim, const int n_cells[3], int precision_mode, int visc_type, int sms,
                        int smem_optin, int smem_sm, int* out, int max_out);
/* The autotuner's table as text, so that a long-running host (a server)
 * can start with the plans an earlier process measured: one line per level
 * shape, "<key> <candidate index>".  The key names the candidate-list
 * version, device ordinal, multigrid, element size, dimension, visc_type,
 * extents, and the device's SM count and shared-memory limits (per block
 * opt-in, per SM) -- everything the candidate list depends on, so a table
 * from another GPU model or library version matches no level.  export
 * writes the table (measured and imported plans) into buf (len bytes,
 * NUL-terminated, truncated if short) and returns the bytes the whole text
 * needs; import reads such text, returns the number of lines taken (lines of
 * another candidate-list version are skipped), or FHD_ERR_BAD_ARG (nothing
 * taken) on a malformed line.  An imported choice is used, untimed, by the
 * first solve that meets its shape; an index beyond that level's candidate
 * list is ignored and the level is timed.  fhd_tune_key writes the key of
 * one level shape for the given device figures (host only) and returns the
 * bytes it needs, or FHD_ERR_BAD_ARG.  No reference counterpart. */
long long fhd_tune_export(char* buf, long long len);
int fhd_tune_import(const char* text);
long long fhd_tune_key(int which, int dim, const int n_cells[3], int precision_mode, int visc_type, int sms,
                       int smem_optin, int smem_sm, int device, char* buf, long long len);
/* Number of this library's kernels launched through ctx so far. */
long long fhd_ctx_kernel_launches(fhd_ctx* ctx);
const char* fhd_status_string(int status);

/* ------------------------------------------------------------------ */
/* device-pointer entry points (canonical layout)                      */
/* u-type arguments are arrays of dim device pointers to face arrays;  */
/* beta_ed has 1 (2D node) or 3 (3D edge) device pointers.             */
/* ------------------------------------------------------------------ */

/* apply_matrix (apply_matrix.f90:24-157):
 *   b_u = theta_alpha*alpha_fc*x_u - L x_u + G x_p ;  b_p = -D x_u */
int fhd_dev_apply_matrix(fhd_ctx* ctx,
                         double* const b_u[], double* b_p,
                         const double* const x_u[], const double* x_p,
                         const double* const alpha_fc[], const double* beta,
                         const double* const beta_ed[], const double* gamma,
                         double theta_alpha);

/* apply_precon (apply_precon.f90:29-475): x = M^{-1} b for precon_type
 * 1..5, including the null-space mean removal; visc_schur_approx = 1 takes
 * the BFBt Schur complement of visc_schur_complement (538-685). */
int fhd_dev_apply_precon(fhd_ctx* ctx,
                         const double* const b_u[], const double* b_p,
                         double* const x_u[], double* x_p,
                         const double* const alpha_fc[], const double* beta,
                         const double* const beta_ed[], const double* gamma,
                         double theta_alpha);

/* stag_mg_solver (stag_mg_solver.f90:37-863): V-cycles on
 * (theta_alpha*alpha - L) phi = rhs; phi is the initial guess on entry. */
int fhd_dev_stag_mg_solver(fhd_ctx* ctx,
                           const double* const alpha_fc[], const double* beta,
                           const double* const beta_ed[], const double* gamma,
                           double theta_alpha,
                           double* const phi[], const double* const rhs[]);

/* gmres (gmres.f90:32-491): restarted left-preconditioned GMRES on the
 * saddle-point system.  x_u, x_p: initial guess in, solution out.
 * norm_pre_rhs (nullable) receives |M^{-1} b|. */
int fhd_dev_gmres(fhd_ctx* ctx,
                  const double* const b_u[], const double* b_p,
                  double* const x_u[], double* x_p,
                  const double* const alpha_fc[], const double* beta,
                  const double* const beta_ed[], const double* gamma,
                  double theta_alpha, double* norm_pre_rhs,
                  fhd_solve_stats* stats);

/* stochastic_m_fluxdiv (stochastic_m_fluxdiv.f90:42-602), periodic box:
 *   force (+)= div( sqrt(variance_coef_mom*2 k_B/(dV dt)) * sqrt(eta T) *
 *                   sum_r weights[r] W_r )
 * W_cc: n_rngs*dim cell arrays (rng r, component c at index r*dim+c).
 * W_ed: 2D: n_rngs*2 node arrays (index r*2+comp); 3D: n_rngs*6 edge arrays
 *       (index r*6 + 2*edge_set + comp, edge sets xy, xz, yz).
 * The random arrays follow fill_m_stochastic (stochastic_m_fluxdiv.f90:
 * 781-860): for the symmetric form the cell entries carry variance 2 and
 * comp 1 of every edge entry equals comp 0.
 * Walls (fhd_ctx_create_bc codes 100, 200): an edge set that contains a
 * wall direction d (2D: the nodes contain x and y; 3D: xy, xz, yz) has
 * n[d] + 1 planes in d, the last one on the high wall; the arrays W_ed,
 * eta_ed and temperature_ed of that set have these extents (x fastest).
 * The edges on a no-slip wall are multiplied by sqrt(2), those on a slip
 * wall set to zero (mflux_bc_2d / _3d, stochastic_m_fluxdiv.f90:363-451),
 * and the normal component of force on a wall face is set to zero
 * (multifab_physbc_domainvel), with or without increment.  The host-fab
 * entry fhd_stochastic_m_fluxdiv takes these planes from the nodal fabs'
 * plane hi+1 (one whole-domain fab per edge multifab). */
int fhd_dev_stochastic_m_fluxdiv(fhd_ctx* ctx, const fhd_stoch_params* sp,
                                 double* const force[], int increment,
                                 const double* eta, const double* const eta_ed[],
                                 const double* temperature,
                                 const double* const temperature_ed[],
                                 double dt, const double* weights, int n_rngs,
                                 const double* const W_cc[],
                                 const double* const W_ed[]);

/* advance_timestep_inertial (advance_timestep_inertial.f90:45-923) for a
 * single-species fluid (nspecies = 1, centred advection, no gravity,
 * periodic box): the Crank-Nicolson predictor-corrector with two GMRES
 * solves (theta_alpha = 1/dt, eta/2 and kappa/2 as in lines 467-474 and
 * 777-784).  umac, rho, pi are advanced in place.  W_cc/W_ed hold this
 * step's random fields as for fhd_dev_stochastic_m_fluxdiv with n_rngs = 1;
 * predictor and corrector use the same fields, as the reference does.
 * stats (nullable) receives the two solves' diagnostics.
 * Walls (fhd_ctx_create_bc codes 100, 200, visc_type 1, 2 or 3): as for
 * fhd_dev_advance_overdamped, and the momentum advection's update is zero
 * on a wall face (mk_advective_m_fluxdiv.f90:80-85). */
int fhd_dev_advance_inertial(fhd_ctx* ctx, const fhd_stoch_params* sp,
                             double dt, double* const umac[], double* rho,
                             double* pi, const double* eta,
                             const double* const eta_ed[], const double* kappa,
                             const double* temperature,
                             const double* const temperature_ed[],
                             const double* const W_cc[],
                             const double* const W_ed[],
                             fhd_solve_stats* stats2);

/* compute_mass_fluxdiv (compute_mass_fluxdiv.f90:29-183) for an ideal
 * isothermal mixture: mass_fluxdiv[i] = div of the corrected diffusive
 * (diffusive_mass_fluxdiv.f90) plus stochastic (stochastic_mass_fluxdiv.f90:
 * 37-116, compute_sqrtLonsager_fc mass_flux_utilities.f90:1096-1522) flux
 * of species i.  rho: nspecies cell arrays.  W_fc[(r*dim+d)*nspecies+i]:
 * N(0,1) field of rng r on the faces of direction d for species i
 * (fill_mass_stochastic, stochastic_mass_fluxdiv.f90:182-214).  Uses k_B
 * and dV of sp.  nspecies 2..5.
 * Walls (fhd_ctx_create_bc codes 100, 200): no flux through a wall face
 * (first-order extrapolated concentrations, scalar_bc in
 * inhomogeneous_bc_val.f90:21-54, and stoch_mass_bc). */
int fhd_dev_compute_mass_fluxdiv(fhd_ctx* ctx, const fhd_mixture_params* mp,
                                 const fhd_stoch_params* sp,
                                 const double* const rho[], double dt,
                                 const double* weights, int n_rngs,
                                 const double* const W_fc[],
                                 double* const mass_fluxdiv[]);

/* compute_sqrtLonsager_fc (mass_flux_utilities.f90:1096-1229): on every
 * face of direction d, the Cholesky factor of the Onsager matrix at the
 * face-averaged density (compute_nonnegative_rho_av, avg_type of mp;
 * compute_sqrtLonsager_local, trace species through the non-trace
 * subsystem).  rho: nspecies cell arrays.  sqrtLonsager_fc: dim*ns*ns face
 * arrays, entry (r, c) of direction d at index d*ns*ns + r + ns*c (the
 * column-major component order of the reference's ns^2-component
 * multifab).  FP64.  nspecies 2..5.
 * Walls (fhd_ctx_create_bc codes 100, 200): on a wall face the ghost cell is
 * the first-order extrapolation of the interior cell (scalar_bc,
 * inhomogeneous_bc_val.f90:21-54).  The high wall face is not stored; the
 * host-fab entry fhd_compute_sqrtLonsager_fc writes it (the last cell with
 * its extrapolated ghost) into the face fab's nodal plane hi+1. */
int fhd_dev_compute_sqrtLonsager_fc(fhd_ctx* ctx, const fhd_mixture_params* mp,
                                    const fhd_stoch_params* sp,
                                    const double* const rho[],
                                    double* const sqrtLonsager_fc[]);

/* stochastic_mass_fluxdiv (stochastic_mass_fluxdiv.f90:37-116) with the
 * face factors of fhd_dev_compute_sqrtLonsager_fc: per face the flux
 * sqrt(2 k_B variance_coef_mass/(dV dt)) * sqrtL * sum_r weights[r] W_r,
 * corrected to a zero species sum when mp->correct_flux
 * (correction_flux.f90:17-226), and its divergence (compute_div), written
 * to stoch_mass_fluxdiv[i] or added to it when increment (increment_in).
 * W_fc[(r*dim+d)*nspecies+i] as in fhd_dev_compute_mass_fluxdiv.
 * stoch_mass_flux (nullable): dim*nspecies face arrays [d*ns+i] receiving the
 * flux.  FP64.  nspecies 2..5, n_rngs 1..4.
 * Walls (fhd_ctx_create_bc codes 100, 200): the flux through a wall face is
 * zero (stoch_mass_bc, stochastic_mass_fluxdiv.f90:216-368); the face
 * arrays keep the periodic layout (face 0 of a wall direction is the low
 * wall, the high wall face is not stored).  The host-fab entry
 * fhd_stochastic_mass_fluxdiv takes walls too: the high wall face of a
 * flux fab, zero, is written from face 0. */
int fhd_dev_stochastic_mass_fluxdiv(fhd_ctx* ctx, const fhd_mixture_params* mp,
                                    const fhd_stoch_params* sp,
                                    const double* const sqrtLonsager_fc[],
                                    double dt, const double* weights, int n_rngs,
                                    const double* const W_fc[], int increment,
                                    double* const stoch_mass_fluxdiv[],
                                    double* const stoch_mass_flux[]);

/* advance_timestep_inertial (advance_timestep_inertial.f90:45-923) for an
 * ideal isothermal mixture of mp->nspecies species (centred advection,
 * periodic box).  rho (nspecies cell arrays), umac, pi advanced in place;
 * mass_fluxdiv holds F^n = div(diffusive + stochastic mass flux) on entry
 * (from the previous step or compute_mass_fluxdiv at start-up) and F^{n+1}
 * on exit.  W_mass: 2*dim*nspecies face arrays, first the fields of the
 * previous corrector (the predictor reuses them, as the reference does
 * between fill_mass_stochastic calls), then this step's new fields.
 * Walls: as for fhd_dev_advance_inertial. */
int fhd_dev_advance_inertial_multispecies(fhd_ctx* ctx, const fhd_stoch_params* sp,
                                          const fhd_mixture_params* mp, double dt,
                                          double* const umac[], double* const rho[],
                                          double* pi, double* const mass_fluxdiv[],
                                          const double* eta,
                                          const double* const eta_ed[],
                                          const double* kappa,
                                          const double* temperature,
                                          const double* const temperature_ed[],
                                          const double* const W_cc[],
                                          const double* const W_ed[],
                                          const double* const W_mass[],
                                          fhd_solve_stats* stats2);

/* advance_timestep_overdamped (advance_timestep_overdamped.f90:135-734):
 * the two-stage overdamped step (theta_alpha = 0) of a single fluid
 * (mp = NULL, rho one array) or an ideal isothermal mixture (rho nspecies
 * arrays), periodic box, centred advection, midpoint_stoch_mass_flux_type
 * 1.  umac, rho, pi advanced in place.  The step draws two random stages
 * once (n_rngs = 2, main_driver.f90:534-536): W_cc 2*dim cell arrays,
 * W_ed 2*2*nE node/edge arrays (indexing as fhd_dev_stochastic_m_fluxdiv
 * with n_rngs = 2), W_mass 2*dim*nspecies face arrays
 * (W_mass[(r*dim+d)*nspecies+i]; NULL without a mixture).  The predictor
 * weighs the stages (1, 0) over dt/2, the corrector (1/sqrt2, 1/sqrt2)
 * over dt.  stats (nullable) receives the two solves' diagnostics.
 * Walls (fhd_ctx_create_bc codes 100, 200, visc_type 1, 2 or 3): the Stokes solve,
 * the stochastic and mass fluxes carry their wall rules (W_ed, eta_ed and
 * temperature_ed then have the high wall's edge planes, as for
 * fhd_dev_stochastic_m_fluxdiv), the pressure gradient is zero on a wall
 * face, and umac's wall faces (zero on entry) stay zero. */
int fhd_dev_advance_overdamped(fhd_ctx* ctx, const fhd_stoch_params* sp,
                               const fhd_mixture_params* mp, double dt,
                               double* const umac[], double* const rho[], double* pi,
                               const double* eta, const double* const eta_ed[],
                               const double* kappa, const double* temperature,
                               const double* const temperature_ed[],
                               const double* const W_cc[], const double* const W_ed[],
                               const double* const W_mass[], fhd_solve_stats* stats2);

/* ------------------------------------------------------------------ */
/* device random numbers (fill_m_stochastic / fill_mass_stochastic,     */
/* stochastic_m_fluxdiv.f90:781-860, stochastic_mass_fluxdiv.f90:182-214*/
/* draw from the host RNG; this is the device-side replacement)         */
/* ------------------------------------------------------------------ */
/* out[0..n) = scale * N(0,1) from Philox-4x32-10 (Salmon et al., SC 2011)
 * keyed by seed; element pair (2j, 2j+1) is the Box-Muller transform of
 * the block at counter (j, field, stream_a, stream_b).  Launched on
 * stream (cudaStream_t, NULL = legacy default stream). */
int fhd_dev_fill_normal(double* out, long long n, unsigned long long seed,
                        unsigned field, unsigned stream_a, unsigned stream_b,
                        double scale, void* stream);
/* The Philox-4x32-10 block function on the host (the same code as the
 * device generator). */
void fhd_philox4x32_10(const unsigned ctr[4], const unsigned key[2],
                       unsigned out[4]);

/* ------------------------------------------------------------------ */
/* serving: many device-resident problems on one GPU (no counterpart in */
/* the reference, whose driver runs one problem per process)           */
/* ------------------------------------------------------------------ */
#define FHD_REQ_OVERDAMPED 0   /* advance_timestep_overdamped steps */
#define FHD_REQ_INERTIAL   1   /* advance_timestep_inertial steps   */
/* One problem: a periodic box, a fluid (nspecies = 1) or an ideal
 * mixture (2..5), uniform eta, k_B T and total density rho0 (mass
 * fractions 1/nspecies), zero initial velocity and pressure, `steps`
 * timesteps of `kind` with device-drawn noise from `seed`.  The final
 * velocity (dim*Nc) and densities (nspecies*Nc) are copied to the host
 * buffers out_umac / out_rho when those are not NULL. */
typedef struct fhd_request {
    int    kind;
    int    dim;
    int    n_cells[3];
    double dx;
    double cell_depth;             /* 2D: dV = dx*dx*cell_depth */
    int    visc_type;
    int    precision;              /* FHD_PREC_FP64 / FHD_PREC_MIXED */
    int    nspecies;
    fhd_mixture_params mix;        /* used when nspecies > 1 */
    double rho0, eta, kT, dt;
    int    steps;
    unsigned long long seed;
    fhd_gmres_params params;
    double* out_umac;
    double* out_rho;
} fhd_request;
typedef struct fhd_request_result {
    long long id;
    int    status;                 /* worst step status, or an error */
    int    gmres_iters;            /* total over all solves */
    long long launches;            /* kernels launched for the request */
    double t_submit, t_start, t_end;   /* seconds on the server's clock */
    double u_sumsq;                /* sum over faces of |u|^2 at the end */
    unsigned long long bytes;      /* device bytes reserved at admission */
} fhd_request_result;
void fhd_request_default(fhd_request* r);
/* Device bytes the server reserves for a request (an upper estimate). */
unsigned long long fhd_request_bytes(const fhd_request* r);
/* A server with `slots` worker threads (one CUDA stream each) on the
 * current device.  Requests start in arrival order as soon as a slot is
 * free and their bytes fit in hbm_budget_bytes beside the running ones;
 * each result depends only on its request. */
typedef struct fhd_server fhd_server;
int fhd_server_create(int slots, unsigned long long hbm_budget_bytes, fhd_server** out);
/* Queues a copy of *req; *id identifies it for fhd_server_wait.  A request
 * larger than the whole budget is refused with FHD_ERR_OOM. */
int fhd_server_submit(fhd_server* srv, const fhd_request* req, long long* id);
/* Blocks until request id has finished. */
int fhd_server_wait(fhd_server* srv, long long id, fhd_request_result* res);
/* Seconds since the server was created (the clock of the results). */
double fhd_server_clock(fhd_server* srv);
/* Finishes the queued requests and joins the workers. */
int fhd_server_destroy(fhd_server* srv);
/* The admission policy on a synthetic trace without a GPU: n requests
 * (arrival time, bytes, run time) on `slots` workers and a byte budget;
 * writes each start time. */
int fhd_sched_simulate(int slots, unsigned long long budget, int n,
                       const double* arrive, const unsigned long long* bytes,
                       const double* runtime, double* start);

/* Text of the last CUDA error seen by the calling thread. */
const char* fhd_last_error(void);
/* Bytes of device memory a context holds. */
unsigned long long fhd_ctx_device_bytes(fhd_ctx* ctx);
/* ------------------------------------------------------------------ */
/* static structure factors on the device                              */
/* ------------------------------------------------------------------ */
/* Replaces HydroGrid's updateStructureFactors (HydroGrid/
 * HydroGridModule.f90:1077-1180) and the normalisation of
 * writeStructureFactors (1862-1868) for periodic boxes: per sample, the
 * unnormalised forward DFT of each of nvars device fields (canonical layout,
 * x fastest), the staggered-velocity phase shift exp(i s k_d pi / N_d) of
 * variable d < dim when shift[d] = s is +1 or -1 (HydroGridModule.f90:
 * 1119-1141; shift may be NULL), and for each of npairs pairs (a, b) =
 * (pairs[2p], pairs[2p+1]) the running mean of Ua conj(Ub).  fhd_sk_read
 * returns pair p times dV / N_cells (structFactMultiplier 1) on the half
 * spectrum kx = 0 .. nx/2, index (kz, ky, kx) with kx fastest, in host
 * arrays of fhd_sk_modes() doubles (re or im may be NULL).  update orders
 * itself after the caller's stream (NULL: none) and makes that stream wait
 * for it.  nvars <= 8, npairs <= 16. */
typedef struct fhd_sk fhd_sk;
int fhd_sk_create(int dim, const int n_cells[3], double dV, int nvars, const int* shift, int npairs,
                  const int* pairs, fhd_sk** out);
int fhd_sk_update(fhd_sk* sk, const double* const vars[], void* stream);
int fhd_sk_read(fhd_sk* sk, int pair, double* re, double* im, long long* samples);
long long fhd_sk_modes(fhd_sk* sk);
int fhd_sk_destroy(fhd_sk* sk);

/* Timing of the finest-level colour smoother (the dominant kernel; the
 * smooths of stag_mg_solver.f90:360-396): while enabled, CUDA events on the
 * context stream bracket each launch.  read returns the launches, their
 * summed device time (ms) and their algorithmic bytes since enable. */
int fhd_ctx_profile(fhd_ctx* ctx, int enable);
int fhd_ctx_profile_read(fhd_ctx* ctx, long long* launches, double* ms,
                         double* bytes);

/* stag_mg_solver without device allocation -- no counterpart in the
 * reference; a variant of fhd_dev_stag_mg_solver for callers that cannot
 * call cudaMalloc (device memory owned by another runtime such as an OpenACC
 * or CUDA Fortran data region, a fixed job pool, or code where an allocation
 * must not synchronise the device).  It needs no context: every work array
 * of the V-cycles comes from one static device array of
 * FHD_NOALLOC_SCRATCH_BYTES that each device loading the library keeps until
 * exit.  Grids whose work arrays do not fit (larger than about 64^3 cells in
 * 3D or 512^2 in 2D) are rejected with FHD_ERR_BAD_ARG and a message in
 * fhd_last_error().  FP64 only; arguments as fhd_dev_stag_mg_solver plus the
 * grid, the parameters and the stream (NULL = legacy default stream).
 * Every call looks up the array's device address on the current device
 * (cudaGetSymbolAddress), so no address outlives a device reset.  All calls
 * share the array: calls whose work overlaps on the GPU race with each
 * other; serialise them (one stream, or synchronise between calls). */
#define FHD_NOALLOC_SCRATCH_BYTES (16ll * 1024 * 1024)
int fhd_dev_stag_mg_solver_noalloc(int dim, const int n_cells[3], double dx,
                                   int visc_type,
                                   const fhd_gmres_params* params,
                                   const double* const alpha_fc[],
                                   const double* beta,
                                   const double* const beta_ed[],
                                   const double* gamma, double theta_alpha,
                                   double* const phi[],
                                   const double* const rhs[], void* stream);

/* ------------------------------------------------------------------ */
/* host BoxLib-fab entry points (drop-in boundary)                     */
/* ------------------------------------------------------------------ */
/* One fab: data(lo(1)-ng : hi(1)+nodal(1)+ng, ..., 1:ncomp) in Fortran
 * column-major order, lo/hi the cell-centred box, nodal[d] = 1 for a face
 * (or node/edge) direction.  Component 0 is used. */
typedef struct fhd_fab {
    double* data;
    int lo[3], hi[3];
    int nodal[3];
    int ng;
    int ncomp;
} fhd_fab;

/* A single-level multifab: the boxes of the level in BoxLib order. */
typedef struct fhd_multifab {
    int nfabs;
    const fhd_fab* fabs;
} fhd_multifab;

/* gmres(mla,the_bc_tower,dx,b_u,b_p,x_u,x_p,alpha_fc,beta,beta_ed,gamma,
 *       theta_alpha,norm_pre_rhs)  (gmres.f90:32-47).
 * x_u/x_p are read as the initial guess and overwritten with the solution
 * in the valid region and ghost cells (periodic fill).  Ghost-cell counts
 * are checked as apply_matrix.f90:54-68 does (x_u, x_p need >= 1). */
int fhd_gmres(fhd_ctx* ctx,
              const fhd_multifab* b_u, const fhd_multifab* b_p,
              const fhd_multifab* x_u, const fhd_multifab* x_p,
              const fhd_multifab* alpha_fc, const fhd_multifab* beta,
              const fhd_multifab* beta_ed, const fhd_multifab* gamma,
              double* theta_alpha, double* norm_pre_rhs,
              fhd_solve_stats* stats);

/* apply_precon(mla,b_u,b_p,x_u,x_p,alpha_fc,beta,beta_ed,gamma,
 *              theta_alpha,dx,the_bc_tower)  (apply_precon.f90:29-43) */
int fhd_apply_precon(fhd_ctx* ctx,
                     const fhd_multifab* b_u, const fhd_multifab* b_p,
                     const fhd_multifab* x_u, const fhd_multifab* x_p,
                     const fhd_multifab* alpha_fc, const fhd_multifab* beta,
                     const fhd_multifab* beta_ed, const fhd_multifab* gamma,
                     double theta_alpha);

/* apply_matrix(mla,b_u,b_p,x_u,x_p,alpha_fc,beta,beta_ed,gamma,
 *              theta_alpha,dx,the_bc_tower)  (apply_matrix.f90:24-40) */
int fhd_apply_matrix(fhd_ctx* ctx,
                     const fhd_multifab* b_u, const fhd_multifab* b_p,
                     const fhd_multifab* x_u, const fhd_multifab* x_p,
                     const fhd_multifab* alpha_fc, const fhd_multifab* beta,
                     const fhd_multifab* beta_ed, const fhd_multifab* gamma,
                     double theta_alpha);

/* stochastic_m_fluxdiv(mla,the_bc_level,stoch_m_force,increment,eta,
 *   eta_ed,temperature,temperature_ed,dx,dt,weights)
 *   (stochastic_m_fluxdiv.f90:42-53).  The module-global random storage
 *   mflux_cc/mflux_nd/mflux_ed of the reference is passed explicitly:
 *   W_cc[r] is a dim-component cell multifab, W_ed[r*nE+e] a 2-component
 *   node (2D, nE=1) or edge (3D, nE=3) multifab.  With walls every edge
 *   multifab (eta_ed, temperature_ed, W_ed) is one whole-domain fab, nodal
 *   in its edge set's directions; its plane hi+1 in a wall direction is the
 *   high wall's (FHD_ERR_BAD_ARG otherwise). */
int fhd_stochastic_m_fluxdiv(fhd_ctx* ctx, const fhd_stoch_params* sp,
                             const fhd_multifab* stoch_m_force, int increment,
                             const fhd_multifab* eta,
                             const fhd_multifab* eta_ed,
                             const fhd_multifab* temperature,
                             const fhd_multifab* temperature_ed,
                             double dt, const double* weights, int n_rngs,
                             const fhd_multifab* W_cc,
                             const fhd_multifab* W_ed);

/* stag_mg_solver(mla,la_mg,alpha_fc,beta_cc,beta_ed,gamma_cc,theta_alpha,
 *                phi_fc,rhs_fc,dx,the_bc_tower)  (stag_mg_solver.f90:37-50):
 * staggered multigrid V-cycles on (theta_alpha alpha - L) phi = rhs.  phi_fc
 * is read as the initial guess and overwritten (valid region and ghost
 * cells, periodic fill); it needs >= 1 ghost cell. */
int fhd_stag_mg_solve(fhd_ctx* ctx,
                      const fhd_multifab* alpha_fc, const fhd_multifab* beta_cc,
                      const fhd_multifab* beta_ed, const fhd_multifab* gamma_cc,
                      double theta_alpha,
                      const fhd_multifab* phi_fc, const fhd_multifab* rhs_fc);

/* compute_sqrtLonsager_fc(mla,rho,rhotot,sqrtLonsager_fc,dx)
 * (mass_flux_utilities.f90:1096-1229): rho an nspecies-component cell
 * multifab with >= 1 ghost cell; rhotot (nullable; the reference does not
 * read it here); sqrtLonsager_fc[d] an nspecies^2-component face multifab of
 * direction d, component r + ns*c = entry (r, c) of the lower Cholesky
 * factor, written over the whole fab (periodic fill). */
int fhd_compute_sqrtLonsager_fc(fhd_ctx* ctx, const fhd_mixture_params* mp,
                                const fhd_stoch_params* sp,
                                const fhd_multifab* rho, const fhd_multifab* rhotot,
                                const fhd_multifab* sqrtLonsager_fc);

/* stochastic_mass_fluxdiv(mla,rho,rhotot,sqrtLonsager_fc,stoch_mass_fluxdiv,
 *   stoch_mass_flux,dx,dt,weights,the_bc_level,increment_in)
 *   (stochastic_mass_fluxdiv.f90:37-51).  The module-global random storage
 *   stoch_W_fc of the reference is passed explicitly: W_fc[r*dim+d] is an
 *   nspecies-component face multifab of stage r, direction d.
 *   stoch_mass_fluxdiv: nspecies-component cell multifab (read too when
 *   increment); stoch_mass_flux (nullable): dim nspecies-component face
 *   multifabs.  rho, rhotot (nullable) are the correction_flux arguments of
 *   the reference, whose correction reads only the fluxes. */
int fhd_stochastic_mass_fluxdiv(fhd_ctx* ctx, const fhd_mixture_params* mp,
                                const fhd_stoch_params* sp,
                                const fhd_multifab* rho, const fhd_multifab* rhotot,
                                const fhd_multifab* sqrtLonsager_fc,
                                const fhd_multifab* stoch_mass_fluxdiv,
                                const fhd_multifab* stoch_mass_flux,
                                double dt, const double* weights, int n_rngs,
                                const fhd_multifab* W_fc, int increment);

/* ------------------------------------------------------------------ */
/* batched realizations: many independent 2D periodic boxes of uneven  */
/* size solved together (no counterpart in the reference, whose driver */
/* runs one problem per process)                                      */
/* ------------------------------------------------------------------ */
/* A batch of nboxes 2D periodic boxes, box b of n_cells[2b] x n_cells[2b+1]
 * cells of side dx, with one multigrid hierarchy per box (compute_nlevs_mg
 * each) packed level by level: every launch of a multigrid level or a
 * Krylov pass covers all boxes, the coarse end of each box's V-cycles runs
 * in one CTA per box, and GMRES's scalar control (Arnoldi coefficients,
 * Givens rotations, stopping tests) runs on the device, one thread per box.
 * Operator: visc_type 1 with a constant viscosity per box, density 1,
 * precon_type 1 (apply_precon.f90:103-195), one V-cycle per multigrid call;
 * precision_mode as fhd_ctx_create (FP32 multigrid in FP64 GMRES, or FP64).
 * Vectors are device arrays of all boxes' cells concatenated in box order,
 * each box in the canonical layout; fhd_batch_box_offset(B, b) is the first
 * element of box b (b = nboxes: the total). */
typedef struct fhd_batch fhd_batch;
int fhd_batch_create(int nboxes, const int* n_cells, double dx,
                     const fhd_gmres_params* params, int precision_mode,
                     fhd_batch** out);
int fhd_batch_destroy(fhd_batch* batch);
long long fhd_batch_box_offset(fhd_batch* batch, int box);
long long fhd_batch_kernel_launches(fhd_batch* batch);
/* gmres (gmres.f90:32-491) of every box: b = (b_u x, b_u y, b_p), x the
 * initial guess in and the solution out, eta[nboxes] (host) the boxes'
 * viscosities, theta_alpha shared.  Each box follows exactly the steps it
 * would take alone.  stats (nullable): nboxes records.  Returns the worst
 * status of the boxes. */
int fhd_batch_gmres(fhd_batch* batch, const double* const b[3],
                    double* const x[3], const double* eta,
                    double theta_alpha, fhd_solve_stats* stats);
/* `steps` overdamped steps (advance_timestep_overdamped.f90:135-734) of
 * every box, one species of density 1 (its density does not change): umac
 * (2 face arrays) and pi in place; eta[nboxes], kT[nboxes] (host) per box;
 * the two random stages of each step drawn on the device from Philox keyed
 * by (seed, box) and counted by (element, field, step0 + step).
 * gmres_iters (nullable): nboxes totals over the steps.  Returns the worst
 * GMRES status. */
int fhd_batch_overdamped(fhd_batch* batch, double* const umac[2], double* pi,
                         const double* eta, const double* kT, double dt,
                         int steps, unsigned long long seed, int step0,
                         int* gmres_iters);

#ifdef __cplusplus
}
#endif
#endif /* FHD_B200_H */
