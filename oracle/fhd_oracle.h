/*
 * fhd_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU FP64 restatement of LowMachFHD's staggered Stokes solve and stochastic
 * momentum flux (periodic single box), used as the parity checker of the
 * CUDA library and as the timed CPU baseline.  Nothing in the product
 * links or calls it; only tests/, __graft_entry__.smoke() and bench.py's
 * CPU baseline leg load it.
 *
 * Arrays use the canonical layout of include/fhd_b200.h.  Vector arguments
 * (u-type, beta_ed) are arrays of `dim` (or nE) host pointers.
 */
#ifndef FHD_ORACLE_H
#define FHD_ORACLE_H

#include "../include/fhd_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* number of staggered MG levels (stag_mg_layout.f90:179-222) */
/* max_grid_size of the level's box layout for the staggered multigrid
 * (module state); NULL or zeros: one box */
void or_set_max_grid_size(const int mgs[3]);
int or_compute_nlevs_mg(int dim, const int n[3], int minwidth);

/* stag_applyop_level with colour (stag_applyop.f90:70-1075); alpha_fc is
 * used as given (already multiplied by theta_alpha). */
void or_stag_applyop(int dim, const int n[3], double dx, int visc_type,
                     const double* const phi[], double* const Lphi[],
                     const double* const alpha_fc[], const double* beta,
                     const double* const beta_ed[], const double* gamma,
                     int color);

int or_stag_mg_solver(int dim, const int n[3], double dx, int visc_type,
                      const fhd_gmres_params* p,
                      const double* const alpha_fc[], const double* beta,
                      const double* const beta_ed[], const double* gamma,
                      double theta_alpha, double* const phi[],
                      const double* const rhs[]);

/* as or_stag_mg_solver, also recording the L2 residual ratio |r|/|r0|
 * after every V-cycle into hist[0 .. stag_mg_max_vcycles-1] (the history
 * stag_mg_verbosity >= 1 prints, stag_mg_solver.f90:782-785) */
int or_stag_mg_history(int dim, const int n[3], double dx, int visc_type,
                       const fhd_gmres_params* p,
                       const double* const alpha_fc[], const double* beta,
                       const double* const beta_ed[], const double* gamma,
                       double theta_alpha, double* const phi[],
                       const double* const rhs[], double* hist);

/* macproject (macproject.f90:34-316) with the pressure multigrid restated
 * from PreconditionerNotes.tex:484-575: solves D (alphainv) G phi = rhs. */
int or_macproject(int dim, const int n[3], double dx,
                  const fhd_gmres_params* p,
                  double* phi, const double* const alphainv_fc[],
                  const double* rhs);
/* the same with the L2 residual ratio after each of mg_max_vcycles
 * V-cycles (no stopping test) in hist */
int or_macproject_history(int dim, const int n[3], double dx, const fhd_gmres_params* p, double* phi,
                          const double* const alphainv_fc[], const double* rhs, double* hist);

int or_apply_matrix(int dim, const int n[3], double dx, int visc_type,
                    double* const b_u[], double* b_p,
                    const double* const x_u[], const double* x_p,
                    const double* const alpha_fc[], const double* beta,
                    const double* const beta_ed[], const double* gamma,
                    double theta_alpha);

/* apply_matrix with gmres_spatial_order = order (2, or 4 with visc_type 1:
 * stag_applyop_4o and compute_grad_4o); nonzero for an unsupported pair */
int or_apply_matrix_order(int dim, const int n[3], double dx, int visc_type,
                          double* const b_u[], double* b_p,
                          const double* const x_u[], const double* x_p,
                          const double* const alpha_fc[], const double* beta,
                          const double* const beta_ed[], const double* gamma,
                          double theta_alpha, int order);

int or_apply_precon(int dim, const int n[3], double dx, int visc_type,
                    const fhd_gmres_params* p,
                    const double* const b_u[], const double* b_p,
                    double* const x_u[], double* x_p,
                    const double* const alpha_fc[], const double* beta,
                    const double* const beta_ed[], const double* gamma,
                    double theta_alpha);

int or_gmres(int dim, const int n[3], double dx, int visc_type,
             const fhd_gmres_params* p,
             const double* const b_u[], const double* b_p,
             double* const x_u[], double* x_p,
             const double* const alpha_fc[], const double* beta,
             const double* const beta_ed[], const double* gamma,
             double theta_alpha, double* norm_pre_rhs,
             fhd_solve_stats* stats);

int or_stochastic_m_fluxdiv(int dim, const int n[3], double dx,
                            const fhd_stoch_params* sp,
                            double* const force[], int increment,
                            const double* eta, const double* const eta_ed[],
                            const double* temperature,
                            const double* const temperature_ed[],
                            double dt, const double* weights, int n_rngs,
                            const double* const W_cc[],
                            const double* const W_ed[]);

/* average_cc_to_node (2D) / average_cc_to_edge (3D) (convert_stag.f90:
 * 395-864) and average_cc_to_face (convert_stag.f90:132-391). */
void or_average_cc_to_edge(int dim, const int n[3], const double* cc,
                           double* const ed[]);
void or_average_cc_to_face(int dim, const int n[3], const double* cc,
                           double* const fc[]);

/* One inertial predictor-corrector step of a single-species fluid with
 * centred advection (advance_timestep_inertial.f90:45-923 with
 * nspecies=1, no mass diffusion, no gravity, periodic).  State umac, rho,
 * pi is advanced in place.  W_cc/W_ed: the step's random fields (one set,
 * n_rngs=1, weights=1), used by predictor and corrector as the reference
 * does.  kappa plays the role of gamma in the solver. */
int or_advance_inertial(int dim, const int n[3], double dx, int visc_type,
                        const fhd_gmres_params* p, const fhd_stoch_params* sp,
                        double dt, double* const umac[], double* rho,
                        double* pi, const double* eta,
                        const double* const eta_ed[], const double* kappa,
                        const double* temperature,
                        const double* const temperature_ed[],
                        const double* const W_cc[], const double* const W_ed[],
                        fhd_solve_stats* stats2);

/* The inertial step for ns species (advance_timestep_inertial.f90 with
 * compute_mass_fluxdiv, ideal isothermal mixture).  rho[ns] and
 * fluxdiv[ns] (F^n in, F^{n+1} out) advanced in place; W_mass holds
 * 2*dim*ns face arrays: the previous corrector's fields (reused by this
 * predictor) then this corrector's new fields. */
/* advance_timestep_overdamped (advance_timestep_overdamped.f90:135-734);
 * mp = NULL for a single fluid (rho: one array, W_mass unused).  W_cc:
 * 2*dim, W_ed: 2*2*nE, W_mass: 2*dim*ns (two random stages). */
int or_advance_overdamped(int dim, const int n[3], double dx, int visc_type,
                          const fhd_gmres_params* p, const fhd_stoch_params* sp,
                          const fhd_mixture_params* mp, double dt, double* const umac[],
                          double* const rho[], double* pi, const double* eta,
                          const double* const eta_ed[], const double* kappa,
                          const double* temperature, const double* const temperature_ed[],
                          const double* const W_cc[], const double* const W_ed[],
                          const double* const W_mass[], fhd_solve_stats* stats2);
int or_advance_inertial_ms(int dim, const int n[3], double dx, int visc_type,
                           const fhd_gmres_params* p, const fhd_stoch_params* sp,
                           const fhd_mixture_params* mp, double dt,
                           double* const umac[], double* const rho[], double* pi,
                           double* const fluxdiv[], const double* eta,
                           const double* const eta_ed[], const double* kappa,
                           const double* temperature,
                           const double* const temperature_ed[],
                           const double* const W_cc[], const double* const W_ed[],
                           const double* const W_mass[], fhd_solve_stats* stats2);

/* compute_mass_fluxdiv (compute_mass_fluxdiv.f90:29-183): divergence of the
 * corrected diffusive + stochastic mass flux; W_fc[(r*dim+d)*ns+i] is the
 * random field of rng r on faces of direction d for species i; flux
 * (nullable) receives the dim*ns face fluxes. */
int or_mass_fluxdiv(int dim, const int n[3], double dx, const fhd_stoch_params* sp,
                    const fhd_mixture_params* mp, const double* const rho[],
                    double dt, const double* weights, int n_rngs,
                    const double* const W_fc[], double* const fluxdiv[],
                    double* const flux[]);

/* chi (Dbar2chi_iterative) and chol(L) at one state rho[ns] (row-major) */
int or_mixture_local(const fhd_mixture_params* mp, double k_B, const double* rho,
                     double* chi, double* sqrtL);
/* compute_sqrtLonsager_fc: per face of direction d the Onsager Cholesky
 * factor at the face-averaged density; sqrtL[d*ns*ns + r + ns*c] */
void or_sqrtLonsager_fc(int dim, const int n[3], const fhd_stoch_params* sp,
                        const fhd_mixture_params* mp, const double* const rho[],
                        double* const sqrtL[]);
/* stochastic_mass_fluxdiv with given face factors; W_fc[(r*dim+d)*ns+s],
 * flux (nullable) [d*ns+s]; div overwritten or, if increment, added to */
void or_stochastic_mass_fluxdiv(int dim, const int n[3], double dx,
                                const fhd_stoch_params* sp,
                                const fhd_mixture_params* mp,
                                const double* const sqrtL[], double dt,
                                const double* weights, int n_rngs,
                                const double* const W_fc[], int increment,
                                double* const div[], double* const flux[]);
/* rho W chi and the Onsager Cholesky factor at one state, trace species
 * included (compute_rhoWchi_local, compute_sqrtLonsager_local) */
void or_mixture_trace_local(const fhd_mixture_params* mp, double k_B, const double* rho,
                            double* rhowchi_out, double* sqrtL_out);

/* Discretisation-accuracy harness of exec/stokes_preconditioner
 * (main_driver.f90:354-387, test_type=0): on [0,1]^dim with n cells per
 * direction returns max|f - A x_exact| per velocity component (err[0..dim-1])
 * and for the pressure row (err[dim]).  prob_coeff in {1,5}, prob_sol in
 * {1,31}. */
int or_accuracy_test(int dim, int n, int prob_coeff, int prob_sol,
                     int visc_type, double* err);
/* the same with apply_matrix of spatial order `order` (2 or 4) */
int or_accuracy_test_order(int dim, int n, int prob_coeff, int prob_sol,
                           int visc_type, int order, double* err);

/* Domain boundaries of the grids the following calls build: per direction
 * bc codes -1 (periodic), 100 (no-slip wall), 200 (slip wall), as in bc.f90;
 * a direction is periodic on both sides or on neither.  Walls are
 * homogeneous (zero wall velocity) and need visc_type 1. */
int or_set_walls(const int bc_lo[3], const int bc_hi[3]);
void or_set_wall_speed(const double wallspeed_lo[6], const double wallspeed_hi[6]);

/* number of OpenMP threads the oracle uses */
int or_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
