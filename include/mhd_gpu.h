/*
 * mhd_gpu.h -- C ABI of the B200 (sm_100a) per-stage DG update for 2D ideal MHD.
 *
 * This is the drop-in boundary for the reference YueWu2002/PP-ES-DG-MHD.  The reference's
 * Fortran driver (drive.f90), set-ups (problems.f90) and output (io.f90) call the hot path
 * through Fortran module procedures and module-level arrays (DG_solver.f90:6-43).  Each entry
 * point below replaces one of those procedures; a Fortran caller binds them with
 * ISO_C_BINDING (interface blocks with bind(C), type(c_ptr), value handles).
 *
 * Conventions
 *   - Every function returns int: 0 = OK, > 0 = sticky solver flag bits (MHD_FLAG_*),
 *     < 0 = API error (MHD_ERR_*).  Nothing aborts the process (the reference's
 *     `error stop` conditions become flags).
 *   - All arrays are FP64 in the reference's Fortran (column-major) layouts:
 *         u      (8, px+1, py+1, 0:nx+1, 0:ny+1)   state with one ghost layer
 *         ut     (8, px+1, py+1, nx, ny)           time derivative
 *         u_avg  (8, 0:nx+1, 0:ny+1)               cell averages
 *         xx     (px+1, nx),  yy (py+1, ny)        GLL node coordinates
 *     The library keeps its own element-blocked device layout and transposes on the GPU at
 *     upload/download.  Host pointers may be pageable or pinned (pinned is faster).
 *   - One handle is used by one host thread at a time.  Handles are independent (no
 *     module-level state), so many solver instances may coexist in one process.
 *   - Supported: px == py in {1,2,3}; rknstg in {1,2,3,5}; nx, ny >= 2.
 */
#ifndef MHD_GPU_H
#define MHD_GPU_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct mhd_gpu mhd_gpu_t;

/* ---- status codes ---------------------------------------------------------------------- */
#define MHD_OK 0
#define MHD_FLAG_NEG_AVG 1        /* inadmissible cell average (DG_solver.f90:189-193)       */
#define MHD_FLAG_PP_RELIMIT 2     /* PP re-limit failed (DG_solver.f90:582-586, error stop)  */
#define MHD_FLAG_DT_COLLAPSE 4    /* dt collapse / too many retries (drive.f90:97-100)       */
#define MHD_FLAG_INIT_NEG_AVG 8   /* initial value inadmissible (drive.f90:70)               */
#define MHD_FLAG_DEVICE_WAIT 16   /* a kernel's bounded wait for its own asynchronous tile copy
                                     ran out; the affected results are invalid (no reference
                                     counterpart; not expected in normal operation)          */
#define MHD_ERR_INVALID -1        /* bad argument                                            */
#define MHD_ERR_UNSUPPORTED -2    /* configuration not supported by the kernels              */
#define MHD_ERR_CUDA -3           /* a CUDA runtime call failed                              */
#define MHD_ERR_NO_DEVICE -4      /* no CUDA device visible                                  */
#define MHD_ERR_STATE -5          /* call out of order (e.g. step before solve_begin)        */

/* ---- boundary-condition kinds (replace the BC_handle procedure pointer, drive.f90:25) --- */
#define MHD_BC_PERIODIC 0         /* BC_periodic     problems.f90:312-348 */
#define MHD_BC_EXTRAPOLATE 1      /* BC_YeeSjogreen  problems.f90:386-423 (outflow) */
#define MHD_BC_FIXED 2            /* BC_rotor        problems.f90:597-654 (bc_state8 = conserved state) */
#define MHD_BC_XEXTRAP_YPER 3     /* BC_BrioWu       problems.f90:350-384 */
#define MHD_BC_CLOUD_SHOCK 4      /* BC_cloud_shock  problems.f90:425-472 (bc_state8 = right inflow state) */
#define MHD_BC_JET 5              /* BC_jet1_cell_ext problems.f90:474-595 (bc_state8 = nozzle state,
                                     below the first nx/10 elements of the bottom side) */

/* status of the device-resident driver (the scalars solve_execute keeps, drive.f90:39-48) */
typedef struct mhd_gpu_status {
  double t;            /* simulated time after the last accepted step              */
  double dt;           /* dt of the last try                                        */
  double dt_lim;       /* dt limit of the last residual (DG_semidiscretize out)     */
  double tot_ent;      /* total entropy of the last final stage                     */
  long long steps;     /* accepted time steps                                       */
  long long retries;   /* re-tries (drive.f90:102)                                  */
  long long num_negcell_total; /* PP-limited cells summed over all accepted stages  */
  int num_negcell_last;/* PP-limited cells of the last stage                        */
  int done;            /* t reached final_T                                         */
  int flags;           /* MHD_FLAG_* bits                                           */
  int pad_;
} mhd_gpu_status;

/* ---- life cycle ------------------------------------------------------------------------- */

/* init_DG_solver(nx,ny,px,py,rknstg,l,r,b,t) (DG_solver.f90:47-107) + set_gamma (MHD_PDE.f90:5)
 * + the choice of BC_handle (drive.f90:25).  Allocates every device array NaN-filled
 * (DG_solver.f90:56,68-85).  bc_state8 is required for MHD_BC_FIXED, MHD_BC_CLOUD_SHOCK and
 * MHD_BC_JET, else may be NULL. */
int mhd_gpu_create(int nx, int ny, int px, int py, int rknstg, double left, double right,
                   double bottom, double top, double gamma, int bc_kind, const double *bc_state8,
                   mhd_gpu_t **out);

/* finalize_DG_solver (DG_solver.f90:109-123) */
int mhd_gpu_destroy(mhd_gpu_t *h);

/* Run all later work of this handle on the given cudaStream_t (NULL = the handle's own). */
int mhd_gpu_set_stream(mhd_gpu_t *h, void *cuda_stream);

/* Device bytes held by this handle (state, stages, scratch); no reference counterpart —
 * used by a caller that admits many solver instances into a fixed HBM budget. */
int mhd_gpu_device_bytes(const mhd_gpu_t *h, size_t *bytes);

/* Block the host until all work queued on the handle's stream is finished. */
int mhd_gpu_synchronize(mhd_gpu_t *h);

/* Human-readable text of a status code. */
const char *mhd_gpu_status_string(int code);

/* ---- geometry and tables ---------------------------------------------------------------- */

/* module variables xx(px+1,nx), yy(py+1,ny) (DG_solver.f90:24,101-106): the node
 * coordinates that Init_type callbacks receive (drive.f90:6-12). */
int mhd_gpu_nodes(const mhd_gpu_t *h, double *xx, double *yy);

/* gauss_lobatto (gauss.f90:17-71) + gauss_lobatto_matrix (gauss.f90:134-331) for degree p<=6:
 * x,w (p+1); M, Minv, D, Pmn, Pnm ((p+1)x(p+1), column-major).  Any pointer may be NULL. */
int mhd_gpu_gll_tables(int p, double *x, double *w, double *M, double *Minv, double *D,
                       double *Pmn, double *Pnm);

/* The locally divergence-free projection that post_process applies to (Bx,By) on an hx x hy
 * element of degree p (DG_solver.f90:231-266 with LDF.f90:114-250), folded into one dense nodal
 * operator A of size (2n^2)x(2n^2), n = p+1, column-major:
 *     [Bx;By]_new - avg = A ([Bx;By] - avg),   node index k + n*l, Bx block first.
 * Host-only (no GPU needed); the kernels apply exactly this matrix.  p in 1..6. */
int mhd_gpu_ldf_operator(int p, double hx, double hy, double *A);

/* ---- state transfer (Fortran layouts) --------------------------------------------------- */

/* slot 0 = u_con, slot s in 1..rknstg = uRK_con(:,:,:,:,:,s) (DG_solver.f90:12,14) */
int mhd_gpu_upload_state(mhd_gpu_t *h, int slot, const double *u);
int mhd_gpu_download_state(mhd_gpu_t *h, int slot, double *u);
/* ut_con(:,:,:,:,:,stage), stage in 1..rknstg (DG_solver.f90:13) */
int mhd_gpu_upload_ut(mhd_gpu_t *h, int stage, const double *ut);
int mhd_gpu_download_ut(mhd_gpu_t *h, int stage, double *ut);
/* u_avg (DG_solver.f90:11), the input of save_tecbin_finite_volume (io.f90:4) */
int mhd_gpu_download_avg(mhd_gpu_t *h, double *u_avg);

/* The cell-average output of save_tecbin_finite_volume (io.f90:75-86): MHD_con2pri
 * (MHD_PDE.f90:44-56) of every interior u_avg, rounded to single precision, in the reference's
 * buffer_var(nx+1, ny, 8) layout (Fortran order; the column nx+1, which the reference leaves
 * unset, is zero), and the per-variable min/max of the rounded values (var_min, var_max: 8 each,
 * may be NULL).  The Tecplot file itself is written by the host, as before. */
int mhd_gpu_download_avg_primitive(mhd_gpu_t *h, float *buffer_var, double *var_min, double *var_max);

/* ---- initial state on the device ---------------------------------------------------------- */

/* init_by_fun_pri (problems.f90:25-51) for the set-ups of the package's problems module,
 * evaluated at the GLL nodes on the GPU into slot 0 (u_con); the ghost ring is set to NaN.
 * params (may be NULL / nparams 0 for the defaults):
 *   MHD_IC_OT2PI, MHD_IC_OT_UNIT, MHD_IC_ROTOR, MHD_IC_ALFVEN: {amp}            (default 1)
 *   MHD_IC_VORTEX: {kappa, mu, p_inf, bulk_vx, bulk_vy}                         (default 1,1,1,1,1)
 *   MHD_IC_BLAST:  {centre_x, centre_y}                                         (default 0,0)
 * Rotor: problems.f90:170-199; OT on [0,1]^2: :155-168; blast: :201-218; smooth Alfven: :74-98;
 * OT on [0,2pi]^2 and the vortex are not in the reference (see the problems module). */
#define MHD_IC_OT2PI 0
#define MHD_IC_OT_UNIT 1
#define MHD_IC_VORTEX 2
#define MHD_IC_BLAST 3
#define MHD_IC_ROTOR 4
#define MHD_IC_ALFVEN 5
#define MHD_IC_CLOUD_SHOCK 6  /* cloud_shock_init_pri (problems.f90:220-247), no parameters */
#define MHD_IC_JET 7          /* jet1_init_pri (problems.f90:249-257), no parameters */
int mhd_gpu_init_problem(mhd_gpu_t *h, int problem, const double *params, int nparams);

/* ---- the reference's per-call interface -------------------------------------------------- */

/* BC_handle(u_con or uRK_con(:,s), ...) (drive.f90:68,71,277,291) */
int mhd_gpu_apply_bc(mhd_gpu_t *h, int slot);

/* post_process(u, u_avg, neg_avg, num_negcell, apply_oedg, apply_LDF, oedg_dt, ent_offset,
 *              comput_ent, tot_ent) (DG_solver.f90:128-661) on state slot `slot`.
 * neg_avg/num_negcell/tot_ent may be NULL.  Returns MHD_FLAG_PP_RELIMIT where the reference
 * would `error stop 123456789`. */
int mhd_gpu_post_process(mhd_gpu_t *h, int slot, int apply_oedg, int apply_ldf, double oedg_dt,
                         int ent_offset, int comput_ent, int *neg_avg, int *num_negcell,
                         double *tot_ent);

/* DG_semidiscretize(ut_con(:,:,:,:,:,ut_stage), dt_lim, u) (DG_solver.f90:663-892) where u is
 * state slot `slot`.  dt_lim may be NULL. */
int mhd_gpu_semidiscretize(mhd_gpu_t *h, int ut_stage, int slot, double *dt_lim);

/* The convex stage update of stage `stage` of SSP-RK(rknstg) with step dt
 * (drive.f90:130-275): writes the interior of uRK_con(:,stage). */
int mhd_gpu_rk_combine(mhd_gpu_t *h, int stage, double dt);

/* The acceptance of a step (drive.f90:304-311): u_con = uRK_con(:,rknstg) on the interior
 * elements; u_con's ghost ring is left as it was, as in the reference. */
int mhd_gpu_rk_accept(mhd_gpu_t *h);

/* ---- device-resident solve_execute (drive.f90:32-343) ----------------------------------- */

/* Prologue of solve_execute after Init_handle filled u_con (drive.f90:67-75): BC,
 * post_process (no OEDG, comput_ent), BC, DG_semidiscretize(ut(:,1)).  Also records
 * final_T, CFL and the limiter switches for the following steps.  tot_ent/dt_lim may be NULL. */
int mhd_gpu_solve_begin(mhd_gpu_t *h, double final_T, double cfl, int use_oedg, int use_ldf,
                        int ent_offset, double *tot_ent, double *dt_lim);

/* One time step of the solving loop (drive.f90:83-320) including its re-tries, entirely on the
 * device; blocks until the step is done and fills *st (may be NULL).  The result is in slot 0
 * (u_con, interior; its ghost ring is left as it was, as in the reference).  The stage slots
 * 1..rknstg are the driver's scratch: unlike the reference's uRK_con(:,rknstg), slot rknstg does
 * not hold a copy of the accepted interior afterwards (the final limiter writes u_con only). */
int mhd_gpu_step(mhd_gpu_t *h, mhd_gpu_status *st);

/* Up to max_steps time steps (<= 0: until final_T), queued without host round trips;
 * the host checks progress every `check_every` steps (<= 0: a default). */
int mhd_gpu_advance(mhd_gpu_t *h, long long max_steps, int check_every, mhd_gpu_status *st);

/* Current driver status without advancing. */
int mhd_gpu_get_status(mhd_gpu_t *h, mhd_gpu_status *st);

/* ---- driver log ------------------------------------------------------------------------- */

/* What solve_execute reports while it runs, recorded on the device by the device-resident driver so
 * that a host that polls only every few steps still sees every stage: per stage the PP-limited
 * cell count it prints (drive.f90:292-294) or the inadmissible average that abandons the try
 * (drive.f90:285-289), per accepted step the (t, tot_ent) pair it appends to its entropy log
 * (drive.f90:314), and the initial state's pair (drive.f90:74). */
#define MHD_LOG_STAGE 1
#define MHD_LOG_STEP 2
typedef struct mhd_log_entry {
  long long seq;        /* running record number, from 0 at solve_begin                       */
  long long step;       /* time step (time_step_num, 1-based; 0 = the initial state)          */
  int kind;             /* MHD_LOG_STAGE or MHD_LOG_STEP                                      */
  int stage;            /* RK stage (stage records; step records: rknstg)                     */
  int try_num;          /* try of the step (1 = first; the stage records of a re-try carry 2+) */
  int num_negcell;      /* PP-limited cells of the stage                                      */
  int neg_avg;          /* 1: inadmissible average, the try was abandoned                      */
  int flags;            /* MHD_FLAG_* bits after the record                                   */
  double t;             /* stage: its pseudo-time t_RK(s); step: the time reached             */
  double dt;            /* dt of the try                                                      */
  double dt_lim;        /* step records: dt_lim of the last residual; stage records: NaN      */
  double tot_ent;       /* step records: total entropy of the accepted state                  */
  double rho_min, p_min;/* diagnostics: min nodal density and pressure of the stage state      */
  double total[8];      /* diagnostics: sum over interior nodes of (hx*hy/4)*w_k*w_l*u, i.e. the
                           domain integrals of rho, m, B, E by the quadrature of the cell
                           averages (DG_solver.f90:177-184); NaN without diagnostics          */
} mhd_log_entry;

/* Keep a log of `capacity` records on the device (0 = no log, the default), drained to the host at
 * every poll of mhd_gpu_advance.  diagnostics != 0 adds, after every completed stage, one kernel
 * that fills rho_min, p_min and total[] of the stage record (and of the step record from its final
 * stage): the invariants the method promises (positivity after every stage, conservation) can
 * then be checked on the device's own output.  Without it the log costs one thread's writes per
 * stage.  Takes effect from the next mhd_gpu_solve_begin or advance (the step graph is
 * re-captured).  Members of a batch log stage and step records, without diagnostics. */
int mhd_gpu_set_log(mhd_gpu_t *h, int capacity, int diagnostics);

/* Up to `cap` of the oldest records not yet read, removed from the log; *n = how many were copied
 * (out == NULL: how many are waiting).  *dropped (may be NULL) = records lost because the device
 * ring filled between two drains.  MHD_ERR_STATE without a log.  For a batch member, call between
 * batch rounds. */
int mhd_gpu_read_log(mhd_gpu_t *h, mhd_log_entry *out, int cap, int *n, long long *dropped);

/* Device address of a state slot in the library's element-blocked layout
 * [ (ny+2) rows ][ (nx+2) elements ][ 8 variables ][ (px+1)*(py+1) nodes ]  (for callers that
 * keep data on the GPU, e.g. a PyTorch tensor view).  No reference counterpart. */
int mhd_gpu_state_device_ptr(mhd_gpu_t *h, int slot, double **dptr);

/* Number of kernel launches in one try of a time step: the kernel nodes of the CUDA graph that
 * mhd_gpu_advance captured (launches that a device-side gate turns into no-ops included).
 * MHD_ERR_STATE before the first advance.  No reference counterpart (diagnostics). */
int mhd_gpu_step_graph_kernels(const mhd_gpu_t *h, int *n);

/* ---- batches of independent instances ---------------------------------------------------- */

/* No reference counterpart (the reference runs one instance per process).  A batch advances many
 * independent solver instances together: one CUDA graph per SSP-RK try runs the batched kernels
 * (persistent grids over a flattened work list of every member's tiles), grouped by (p, rknstg).
 * Each member computes exactly what mhd_gpu_advance would compute for it alone.
 * Members must be on the batch's device and past mhd_gpu_solve_begin; while in a batch a member is
 * driven only by the batch (its status is still readable); remove it before destroying it. */
typedef struct mhd_batch mhd_batch_t;
int mhd_batch_create(mhd_batch_t **out);
int mhd_batch_destroy(mhd_batch_t *b);
int mhd_batch_add(mhd_batch_t *b, mhd_gpu_t *h);
int mhd_batch_remove(mhd_batch_t *b, mhd_gpu_t *h);
int mhd_batch_size(const mhd_batch_t *b, int *n);
/* `tries` graph launches (each member takes one try of a time step per launch: an accepted step,
 * a re-try, or nothing once done), then a refresh of every member's status; *n_active (may be
 * NULL) = members neither done nor failed. */
int mhd_batch_advance(mhd_batch_t *b, int tries, int *n_active);
/* mhd_batch_advance in two halves, so that the host can work while a round runs: _launch queues
 * the round and returns; _wait blocks until it has finished and refreshes the statuses.  Between
 * the two, members can be neither added nor removed (MHD_ERR_STATE). */
int mhd_batch_launch(mhd_batch_t *b, int tries);
int mhd_batch_wait(mhd_batch_t *b, int *n_active);
/* a member's status as of the last completed round */
int mhd_batch_member_status(mhd_batch_t *b, mhd_gpu_t *h, mhd_gpu_status *st);

/* ---- serving ------------------------------------------------------------------------------ */

/* No reference counterpart.  Device bytes mhd_gpu_create would allocate for one instance (the
 * admission price of a run). */
int mhd_gpu_footprint(int nx, int ny, int p, int rknstg, size_t *bytes);

/* One run = one solve_execute: configuration, initial state and an arrival time (seconds on the
 * server clock, which starts at the first mhd_server_run). */
typedef struct mhd_request {
  long long id;
  int nx, ny, p, rknstg;
  double left, right, bottom, top, gamma;
  int bc_kind;
  int pad_;
  double bc_state8[8];
  double final_T, cfl;
  int use_oedg, use_ldf, ent_offset;
  int pad2_;
  double arrival;
  const double *u0;   /* host, Fortran layout u(8,p+1,p+1,0:nx+1,0:ny+1); valid until finished */
  double *u_avg_out;  /* host, receives u_avg (8,0:nx+1,0:ny+1) at the end; may be NULL */
} mhd_request;

typedef struct mhd_request_result {
  long long id;
  double arrival, admitted, finished;  /* server clock, seconds */
  double t;                            /* simulated time reached */
  long long steps, retries;
  int done, flags, error, pad_;
} mhd_request_result;

/* A request loop with continuous batching: runs are admitted when they have arrived and their
 * footprint fits the HBM budget (at most max_active at once), all active runs advance together in
 * one batch (tries_per_round batched tries between polls), finished runs retire and free their
 * memory.  batched = 0 serves the same queue one plain run at a time (the comparison point).
 * The budget is reserved on the device when the server is created (one allocation; a budget the
 * device cannot hold returns MHD_ERR_UNSUPPORTED) and every run's buffers are carved from it, so
 * the loop itself makes no device allocation call.  Admissions overlap the round in flight. */
typedef struct mhd_server mhd_server_t;
int mhd_server_create(size_t hbm_budget_bytes, int max_active, int tries_per_round, int batched,
                      mhd_server_t **out);
int mhd_server_submit(mhd_server_t *s, const mhd_request *r);
/* serve until every submitted run has finished, or max_seconds (<= 0: no limit) of wall time */
int mhd_server_run(mhd_server_t *s, double max_seconds);
int mhd_server_pending(const mhd_server_t *s, int *queued, int *active, size_t *used_bytes);
int mhd_server_results(const mhd_server_t *s, mhd_request_result *out, int cap, int *n);
/* where the loop's host time went (wall seconds, summed over every mhd_server_run) */
typedef struct mhd_server_stats {
  long long rounds;          /* batched rounds launched (plain mode: runs executed) */
  long long admitted, retired;
  long long graph_captures;  /* batch graph (re)captures */
  double admit_s;            /* creating instances, uploading, solve_begin */
  double launch_s;           /* queueing rounds */
  double wait_s;             /* blocked on the device */
  double retire_s;           /* downloading results, freeing instances, batch membership */
  double idle_s;             /* nothing active and nothing arrived */
} mhd_server_stats;
int mhd_server_get_stats(const mhd_server_t *s, mhd_server_stats *out);
int mhd_server_destroy(mhd_server_t *s);

/* ---- allocation-free residual ------------------------------------------------------------ */

/* No counterpart in the reference: an extra entry point of this library.
 *
 * ut = L(u) and dt_lim, the same computation as mhd_gpu_semidiscretize, for callers that must
 * not allocate device memory: hosts whose device-memory budget is fully reserved up front by
 * their own pool or memory manager, hosts running on a device whose allocations are capped by an
 * external manager, and time-critical loops that cannot afford the implicit device-wide
 * synchronisation a cudaMalloc/cudaFree may cause.  The caller owns and passes both arrays:
 *   u   device pointer, state in the library's element-blocked layout with the ghost ring filled
 *       ([ny+2][nx+2][8][(p+1)^2] doubles, the layout mhd_gpu_state_device_ptr exposes);
 *   ut  device pointer, [ny][nx][8][(p+1)^2] doubles, written;
 *   dt_lim  host pointer (may be NULL); when given, the call waits for the stream.
 * u and ut must both start on a 16-byte boundary (the kernel moves whole element blocks with
 * 16-byte loads and stores) and must not overlap; a pointer that breaks either rule is rejected
 * with MHD_ERR_INVALID before the GPU is touched.
 * The call allocates nothing: its only scratch (the dt_lim reduction cell and status words) is a
 * 4 KiB static device array inside the library, which every GPU that loads the library holds
 * until the process exits.  All calls share that array and it keeps the last call's contents;
 * the reduction cell is reset at the start of every call, and calls that overlap on the GPU
 * (different streams or host threads at the same time) race on it.
 * The first call on a device sets that device up (constant tables, kernel attributes and the
 * address of the static array); make that first call before any stream capture.  That set-up is
 * kept for the life of the process, like every handle's device set-up: the library must not be
 * used across a cudaDeviceReset of its device.
 * Limits: px = py = p in 1..3, 2 <= nx, ny <= 4096; anything larger or any other argument out of
 * range is rejected with MHD_ERR_UNSUPPORTED / MHD_ERR_INVALID before touching the GPU.
 * stream: a cudaStream_t (NULL = the legacy default stream). */
int mhd_gpu_semidiscretize_noalloc(int p, int nx, int ny, double hx, double hy, double gamma,
                                   const double *u, double *ut, double *dt_lim, void *stream);

#ifdef __cplusplus
}
#endif
#endif
