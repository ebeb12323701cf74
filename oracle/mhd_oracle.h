/*
 * mhd_oracle.h -- CPU restatement of the reference's per-stage DG update for 2D ideal MHD.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the correctness oracle and the timed CPU
 * baseline.  Only tests/, __graft_entry__.smoke() and bench.py (cpu_baseline leg and
 * --impl reference) may load it.  The product path (pp-es-dg-mhd_b200/) never links it.
 *
 * It restates, in the reference's operation order and with its clamps, the Fortran
 * routines of YueWu2002/PP-ES-DG-MHD:
 *   DG_solver.f90:47-107   init_DG_solver (geometry, NaN-filled state)
 *   DG_solver.f90:125-661  macros _macro_prs_/_macro_ent_ and post_process
 *   DG_solver.f90:663-892  DG_semidiscretize
 *   DG_solver.f90:894-1071 ESPP_HLL_flux_x
 *   DG_solver.f90:1556-1681 swap_xy, ec_flux_x/y, log_avg_divisor
 *   LDF.f90:114-250        LDF_projector init/apply (SVD by one-sided Jacobi in place of DGESDD)
 *   gauss.f90:17-71,134-331,436-475  GLL and Legendre tables (computed, not tabulated)
 *   drive.f90:32-343       solve_execute (SSP-RK(1,1),(2,2),(3,3),(5,4), CFL dt, retry)
 *   problems.f90:312-423,597-654     BC_periodic, BC_BrioWu, BC_YeeSjogreen, BC_rotor
 *
 * Parity status: the reference cannot be compiled here (no Fortran compiler), so no run of
 * the reference pins this restatement.  What pins it: the reference's own self-checks
 * (gauss.f90:73-132,365-388,477-502 quadrature/SBP/nilpotency; LDF.f90:83-87 projector
 * identities), closed-form table values from the reference, conservation, positivity and
 * entropy invariants.  Full-step parity against the reference is therefore "parity unpinned"
 * beyond those known answers.
 *
 * All arrays use the reference's Fortran (column-major) layouts:
 *   u      (8, px+1, py+1, 0:nx+1, 0:ny+1)
 *   ut     (8, px+1, py+1, nx, ny)
 *   u_avg  (8, 0:nx+1, 0:ny+1)
 */
#ifndef MHD_ORACLE_H
#define MHD_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct ora_solver ora_solver;

/* boundary-condition kinds (problems.f90) */
enum {
  ORA_BC_PERIODIC = 0,      /* BC_periodic      problems.f90:312-348 */
  ORA_BC_EXTRAPOLATE = 1,   /* BC_YeeSjogreen   problems.f90:386-423 */
  ORA_BC_FIXED = 2,         /* BC_rotor pattern problems.f90:597-654 (state given) */
  ORA_BC_XEXTRAP_YPER = 3,  /* BC_BrioWu        problems.f90:350-384 */
  ORA_BC_CLOUD_SHOCK = 4,   /* BC_cloud_shock   problems.f90:425-472 (state = right inflow) */
  ORA_BC_JET = 5            /* BC_jet1_cell_ext problems.f90:474-595 (state = bottom nozzle) */
};

/* status codes returned by ora_solve */
enum {
  ORA_OK = 0,
  ORA_ERR_DT_COLLAPSE = 1,     /* drive.f90:97-100  error stop 1 */
  ORA_ERR_INIT_NEG_AVG = 2,    /* drive.f90:70 */
  ORA_ERR_PP_RELIMIT = 3,      /* DG_solver.f90:582-586 error stop 123456789 */
  ORA_ERR_BAD_ARG = 4
};

ora_solver *ora_create(int nx, int ny, int px, int py, int rknstg, double left, double right,
                       double bottom, double top, double gamma, int bc_kind,
                       const double *bc_state8);
void ora_destroy(ora_solver *s);

/* number of doubles of each array */
long ora_size_u(const ora_solver *s);
long ora_size_ut(const ora_solver *s);
long ora_size_avg(const ora_solver *s);

/* direct access to the module-level arrays (solver owns them) */
double *ora_u_con(ora_solver *s);
double *ora_ut_con(ora_solver *s, int stage);  /* stage 1..rknstg */
double *ora_urk_con(ora_solver *s, int stage); /* stage 1..rknstg */
double *ora_u_avg(ora_solver *s);

/* node coordinates xx(px+1,nx), yy(py+1,ny) */
void ora_nodes(const ora_solver *s, double *xx, double *yy);

/* 1-D tables for degree p (p<=6), column-major (p+1)x(p+1):
 * x, w: GLL nodes/weights; M, Minv, D, Pmn, Pnm: nodal matrices (gauss.f90:134-331). */
int ora_gll_tables(int p, double *x, double *w, double *M, double *Minv, double *D,
                   double *Pmn, double *Pnm);
/* Legendre modal tables (gauss.f90:436-475): m, minv, tl, tr (p+1), D (p+1)^2 */
int ora_legendre_tables(int p, double *m, double *minv, double *D, double *tl, double *tr);
/* LDF projector tables (LDF.f90:114-217): Lx(px+1), Ux(px+1)^2, Ly, Uy, Ldagger(px+1,py+1) */
int ora_ldf_tables(int px, int py, double *Lx, double *Ux, double *Ly, double *Uy,
                   double *Ldagger);
/* LDF projector apply on Legendre coefficients uu(px+1,py+1,2) in place (LDF.f90:219-250) */
int ora_ldf_apply(int px, int py, double *uu);
/* divergence of modal coefficients (LDF.f90:252-260) */
int ora_ldf_div(int px, int py, const double *uu, double *udiv);

/* two-point fluxes (unit-level checks) */
void ora_hll_flux_x(const double *wl, const double *wr, double gamma, double *nflux,
                    double *nBn, double *sl, double *sr);
void ora_ec_flux_x(const double *pl, const double *pr, double gamma, double *flux);
void ora_ec_flux_y(const double *pl, const double *pr, double gamma, double *flux);
double ora_log_avg_divisor(double a, double b);

/* ghost-cell fill of u according to the solver's BC kind */
void ora_apply_bc(ora_solver *s, double *u);

/* post_process (DG_solver.f90:128-661); pp_relimit_fail reports the error-stop condition */
void ora_post_process(ora_solver *s, double *u, double *u_avg, int *neg_avg, int *num_negcell,
                      int apply_oedg, int apply_ldf, double oedg_dt, int ent_offset,
                      int comput_ent, double *tot_ent, int *pp_relimit_fail);

/* DG_semidiscretize (DG_solver.f90:663-892) */
void ora_semidiscretize(ora_solver *s, double *ut, double *dt_lim, const double *u);

/* RK stage combination (drive.f90:130-275), writes uRK(:,stage) interior; returns t_RK(stage) */
double ora_rk_combine(ora_solver *s, int stage, double dt, double t, double *t_rk);

/* solve_execute (drive.f90:32-343) starting from the interior values already in u_con.
 * Runs until t reaches final_T or max_steps accepted steps (max_steps<=0: no limit).
 * out_stats (may be NULL) receives: [0]=t, [1]=dt_lim, [2]=tot_ent, [3]=steps,
 * [4]=retries, [5]=last dt, [6]=total num_negcell over all stages. */
int ora_solve(ora_solver *s, double final_T, double cfl, int use_oedg, int use_ldf,
              int ent_offset, int max_steps, double *out_stats);

/* as ora_solve; resume != 0 continues from the driver scalars (t, dt, dt_lim) and ut(:,1) left by
 * the previous call instead of running the prologue again */
int ora_solve_resume(ora_solver *s, double final_T, double cfl, int use_oedg, int use_ldf,
                     int ent_offset, int max_steps, int resume, double *out_stats);

/* set OpenMP threads used by the oracle (<=0: leave default) */
void ora_set_threads(int n);
int ora_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
