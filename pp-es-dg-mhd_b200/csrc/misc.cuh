// misc.cuh -- boundary fill, SSP-RK stage combination, layout transposes and the device-side
// step control of solve_execute.
#pragma once
#include "common.cuh"

namespace mhd {

enum BcKind : int {
  BC_PERIODIC = 0, BC_EXTRAPOLATE = 1, BC_FIXED = 2, BC_XEXTRAP_YPER = 3, BC_CLOUD_SHOCK = 4, BC_JET = 5
};

// Where a ghost value comes from (problems.f90:312-423,597-654): node sq of variable v of interior
// element (si, sj), negated if neg, or the fixed state bc_state[v] if fixed.  (i, j) is a ghost
// element off the corners, q its node.
struct BcSrc {
  int si, sj, sq;
  bool fixed, neg;
};

template <int P>
__device__ __forceinline__ BcSrc bc_source(const Geo& g, int i, int j, int v, int q) {
  constexpr int N = P + 1;
  const int nx = g.nx, ny = g.ny, k = q % N, l = q / N;
  const bool xside = (i == 0 || i == nx + 1);  // left/right ghost column
  BcSrc s{i, j, q, false, false};
  int kind = g.bc_kind;
  if (kind == BC_CLOUD_SHOCK || kind == BC_JET) {
    // BC_cloud_shock (problems.f90:449-471): element copies, inflow state on the right.
    // BC_jet1_cell_ext (problems.f90:502-593): mirror of element 1 on the left (k <- n-1-k, normal
    // momentum and field negated), copies elsewhere, the nozzle state below i <= nx/10.
    if ((kind == BC_CLOUD_SHOCK && i == nx + 1) || (kind == BC_JET && j == 0 && i <= nx / 10)) {
      s.fixed = true;
      return s;
    }
    s.si = (i == 0) ? 1 : (i == nx + 1 ? nx : i);
    s.sj = (j == 0) ? 1 : (j == ny + 1 ? ny : j);
    if (kind == BC_JET && i == 0) {
      s.sq = (N - 1 - k) + N * l;
      s.neg = (v == 1 || v == 4);
    }
    return s;
  }
  if (kind == BC_XEXTRAP_YPER) kind = xside ? BC_EXTRAPOLATE : BC_PERIODIC;
  if (kind == BC_FIXED) {
    s.fixed = true;
  } else if (kind == BC_PERIODIC) {
    s.si = (i == 0) ? nx : (i == nx + 1 ? 1 : i);
    s.sj = (j == 0) ? ny : (j == ny + 1 ? 1 : j);
  } else if (xside) {  // extrapolation of the adjacent interior trace
    s.si = (i == 0) ? 1 : nx;
    s.sq = ((i == 0) ? 0 : N - 1) + N * l;
  } else {
    s.sj = (j == 0) ? 1 : ny;
    s.sq = k + N * ((j == 0) ? 0 : N - 1);
  }
  return s;
}

// Ghost-ring fill of dst from the interior of src (the same array, or an array whose interior holds
// the same values).  One thread per ghost value; corners untouched.
template <int P>
__device__ __forceinline__ void bc_value(const double* src, double* dst_u, const Geo& g, long long it) {
  constexpr int N = P + 1, NN = N * N, EB = 8 * NN;
  const int nx = g.nx, ny = g.ny, NXG = nx + 2;
  const long long nghost = 2LL * (nx + ny);
  if (it >= nghost * EB) return;
  const int ge = (int)(it / EB), vi = (int)(it - (long long)ge * EB);
  const int v = vi / NN, q = vi - v * NN;
  int i, j;  // ghost element
  if (ge < ny) { i = 0; j = 1 + ge; }
  else if (ge < 2 * ny) { i = nx + 1; j = 1 + ge - ny; }
  else if (ge < 2 * ny + nx) { i = 1 + ge - 2 * ny; j = 0; }
  else { i = 1 + ge - 2 * ny - nx; j = ny + 1; }
  const long long dst = ((long long)j * NXG + i) * EB + vi;
  const BcSrc s = bc_source<P>(g, i, j, v, q);
  if (s.fixed) {
    dst_u[dst] = g.bc_state[v];
    return;
  }
  const double x = src[((long long)s.sj * NXG + s.si) * EB + v * NN + s.sq];
  dst_u[dst] = s.neg ? -x : x;
}

template <int P>
__global__ void __launch_bounds__(256) bc_kernel(double* __restrict__ u, Geo g, const Ctrl* ctrl, int gate) {
  if (!gate_open(ctrl, gate)) return;
  bc_value<P>(u, u, g, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// many instances: items = every member's blocks of 256 ghost values
template <int P>
__global__ void __launch_bounds__(256) bc_batched(const InstDesc* __restrict__ insts, const int* __restrict__ pref,
                                                  const int* __restrict__ nwork, const int* __restrict__ ninst,
                                                  int slot, int gate) {
  const int nw = *nwork, n = *ninst;
  for (BatchWalk it(pref, n, nw); it.more(); it.next()) {
    const int m = it.m, chunk = it.local();
    const InstDesc& d = insts[m];
    if (!gate_open(d.ctrl, gate)) continue;
    bc_value<P>(d.u[slot], d.u[slot], d.g, (long long)chunk * 256 + threadIdx.x);
  }
}

// SSP-RK stage update (drive.f90:130-275) on interior elements, rounded exactly as written
// (explicit _rn intrinsics: no fused multiply-add contraction).
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }

// the weight of dt in the stage-1 update u0 + (weight*dt)*k1
__host__ __device__ constexpr double stage1_coef(int R) { return R == 5 ? 0.391752226571890 : 1.0; }

template <int EB>
__device__ __forceinline__ void combine_value(
    const double* __restrict__ u0, const double* __restrict__ r1, const double* __restrict__ r2,
    const double* __restrict__ r3, const double* __restrict__ r4, const double* __restrict__ k1,
    const double* __restrict__ k2, const double* __restrict__ k3, const double* __restrict__ k4,
    const double* __restrict__ k5, double* __restrict__ out, int nx, int ny, int R, int stage, double dt,
    long long it) {
  const long long n = (long long)nx * ny * EB;
  if (it >= n) return;
  const long long e = it / EB;
  const int c = (int)(it - e * EB);
  const int j = 1 + (int)(e / nx), i = 1 + (int)(e - (long long)(j - 1) * nx);
  const long long gi = ((long long)j * (nx + 2) + i) * EB + c;  // ghosted index
  const long long ki = it;                                       // interior index
  double val;
  if (R == 1 || (stage == 1 && R <= 3)) {
    val = add(u0[gi], mul(dt, k1[ki]));
  } else if (R == 2) {
    val = add(mul(0.5, u0[gi]), mul(0.5, add(r1[gi], mul(dt, k2[ki]))));
  } else if (R == 3) {
    if (stage == 2)
      val = add(mul(0.75, u0[gi]), mul(0.25, add(r1[gi], mul(dt, k2[ki]))));
    else
      val = add(mul(1.0 / 3.0, u0[gi]), mul(2.0 / 3.0, add(r2[gi], mul(dt, k3[ki]))));
  } else {  // SSP-RK(5,4)
    switch (stage) {
      case 1: val = add(u0[gi], mul(mul(stage1_coef(5), dt), k1[ki])); break;
      case 2: val = add(add(mul(0.444370493651235, u0[gi]), mul(0.555629506348765, r1[gi])), mul(mul(0.368410593050371, dt), k2[ki])); break;
      case 3: val = add(add(mul(0.620101851488403, u0[gi]), mul(0.379898148511597, r2[gi])), mul(mul(0.251891774271694, dt), k3[ki])); break;
      case 4: val = add(add(mul(0.178079954393132, u0[gi]), mul(0.821920045606868, r3[gi])), mul(mul(0.544974750228521, dt), k4[ki])); break;
      default:
        val = add(add(add(add(mul(0.517231671970585, r2[gi]), mul(0.096059710526147, r3[gi])), mul(mul(0.063692468666290, dt), k4[ki])),
                      mul(0.386708617503269, r4[gi])), mul(mul(0.226007483236906, dt), k5[ki]));
        break;
    }
  }
  out[gi] = val;
}

template <int EB>
__global__ void __launch_bounds__(256)
    combine_kernel(const double* __restrict__ u0, const double* __restrict__ r1, const double* __restrict__ r2,
                   const double* __restrict__ r3, const double* __restrict__ r4,
                   const double* __restrict__ k1, const double* __restrict__ k2, const double* __restrict__ k3,
                   const double* __restrict__ k4, const double* __restrict__ k5, double* __restrict__ out,
                   int nx, int ny, int R, int stage, const double* __restrict__ dt_ptr, double dt_arg,
                   const Ctrl* ctrl, int gate) {
  if (!gate_open(ctrl, gate)) return;
  const double dt = dt_ptr ? *dt_ptr : dt_arg;
  combine_value<EB>(u0, r1, r2, r3, r4, k1, k2, k3, k4, k5, out, nx, ny, R, stage, dt,
                    (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// many instances: items = every member's blocks of 256 values; dt from each member's control block
template <int EB>
__global__ void __launch_bounds__(256) combine_batched(const InstDesc* __restrict__ insts, const int* __restrict__ pref,
                                                       const int* __restrict__ nwork, const int* __restrict__ ninst,
                                                       int stage, int gate) {
  const int nw = *nwork, n = *ninst;
  for (BatchWalk it(pref, n, nw); it.more(); it.next()) {
    const int m = it.m, chunk = it.local();
    const InstDesc& d = insts[m];
    if (!gate_open(d.ctrl, gate)) continue;
    combine_value<EB>(d.u[0], d.u[1], d.u[2], d.u[3], d.u[4], d.ut[1], d.ut[2], d.ut[3], d.ut[4], d.ut[5],
                      d.u[stage], d.g.nx, d.g.ny, d.R, stage, d.ctrl->dt, (long long)chunk * 256 + threadIdx.x);
  }
}

// Fortran layout (8, n, n, E) <-> element-blocked layout [E][8][n*n].  E = element count.
__global__ void __launch_bounds__(256) to_blocked_kernel(const double* __restrict__ src, double* __restrict__ dst,
                                                        long long nelem, int NN) {
  const long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = nelem * 8 * NN;
  if (it >= n) return;
  const int EB = 8 * NN;
  const long long e = it / EB;
  const int c = (int)(it - e * EB);
  const int v = c / NN, q = c - v * NN;
  dst[it] = src[e * EB + q * 8 + v];
}
__global__ void __launch_bounds__(256) to_fortran_kernel(const double* __restrict__ src, double* __restrict__ dst,
                                                        long long nelem, int NN) {
  const long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = nelem * 8 * NN;
  if (it >= n) return;
  const int EB = 8 * NN;
  const long long e = it / EB;
  const int c = (int)(it - e * EB);
  const int q = c / 8, v = c - q * 8;
  dst[it] = src[e * EB + v * NN + q];
}

// ---- device-side control of solve_execute (drive.f90:83-320) ---------------------------------

__device__ __forceinline__ double dec_dtlim(unsigned long long b) { return __longlong_as_double((long long)b); }

// reset the per-call outputs of post_process
__global__ void ctl_pp_reset(Ctrl* c, int gate) {
  if (!gate_open(c, gate)) return;
  c->neg_avg = 0;
  c->num_negcell = 0;
  c->pp_relimit = 0;
  for (int v = 0; v < 8; ++v) {
    c->umax_bits[v] = 0ULL;
    c->umin_bits[v] = ~0ULL;
  }
}

// Fortran x**n for integer n >= 1 (binary exponentiation, as libgcc's __powidf2)
__device__ __forceinline__ double powi_d(double x, int n) {
  double r = (n & 1) ? x : 1.0;
  while (n >>= 1) {
    x = __dmul_rn(x, x);
    if (n & 1) r = __dmul_rn(r, x);
  }
  return r;
}

// Start of one try of a time step (drive.f90:93-105).  Decodes the last residual's dt_lim.
__device__ __forceinline__ void ctl_step_begin_body(Ctrl* c) {
  if (c->pending_dtlim) {
    c->dt_lim = dec_dtlim(c->dt_lim_bits);
    c->pending_dtlim = 0;
  }
  if (c->done || (c->flags & FLAGS_FATAL) || c->steps >= c->step_limit) {  // finished, error, or step budget used
    c->state = ST_IDLE;
    return;
  }
  c->try_num += 1;
  if (c->try_num > 10 || c->dt_lim < 1e-14) {
    c->flags |= 4;  // MHD_FLAG_DT_COLLAPSE
    c->state = ST_IDLE;
    return;
  }
  if (c->try_num > 1) {
    c->retries += 1;
    c->state = ST_RECOMPUTE;  // re-compute ut(:,1) from u_con (drive.f90:104)
    c->dt_lim_bits = ~0ULL;
    c->pending_dtlim = 1;
  } else {
    c->state = ST_RUN;
  }
}

// dt of this try (drive.f90:107-120)
__device__ __forceinline__ void ctl_dt_body(Ctrl* c) {
  if (c->pending_dtlim) {
    c->dt_lim = dec_dtlim(c->dt_lim_bits);
    c->pending_dtlim = 0;
  }
  if (c->state == ST_IDLE) return;
  double dt;
  if (c->try_num <= 1)
    dt = __dmul_rn(c->cfl_total, c->dt_lim);
  else
    dt = __dmul_rn(powi_d(__dadd_rn(__dsqrt_rn(1.25), -0.5), c->try_num - 1), c->dt);
  if (__dadd_rn(c->t, dt) >= c->final_T) {
    dt = __dadd_rn(c->final_T, -c->t);
    c->last_step = 1;
  } else {
    c->last_step = 0;
  }
  c->dt = dt;
  c->state = ST_RUN;
}

// pseudo-time of stage s (drive.f90:142-267), computed before the stage's combine
__device__ __forceinline__ void ctl_stage_time_body(Ctrl* c, int R, int s) {
  if (c->state != ST_RUN) return;
  const double t = c->t, dt = c->dt;
  double* tr = c->t_rk;
  double v;
  if (R == 1 || (s == 1 && R <= 3)) v = __dadd_rn(t, __dmul_rn(dt, 1.0));
  else if (R == 2) v = __dadd_rn(__dmul_rn(0.5, t), __dmul_rn(0.5, __dadd_rn(tr[1], __dmul_rn(dt, 1.0))));
  else if (R == 3)
    v = (s == 2) ? __dadd_rn(__dmul_rn(0.75, t), __dmul_rn(0.25, __dadd_rn(tr[1], __dmul_rn(dt, 1.0))))
                 : __dadd_rn(__dmul_rn(1.0 / 3.0, t), __dmul_rn(2.0 / 3.0, __dadd_rn(tr[2], __dmul_rn(dt, 1.0))));
  else {
    switch (s) {
      case 1: v = __dadd_rn(t, __dmul_rn(__dmul_rn(0.391752226571890, dt), 1.0)); break;
      case 2: v = __dadd_rn(__dadd_rn(__dmul_rn(0.444370493651235, t), __dmul_rn(0.555629506348765, tr[1])), __dmul_rn(__dmul_rn(0.368410593050371, dt), 1.0)); break;
      case 3: v = __dadd_rn(__dadd_rn(__dmul_rn(0.620101851488403, t), __dmul_rn(0.379898148511597, tr[2])), __dmul_rn(__dmul_rn(0.251891774271694, dt), 1.0)); break;
      case 4: v = __dadd_rn(__dadd_rn(__dmul_rn(0.178079954393132, t), __dmul_rn(0.821920045606868, tr[3])), __dmul_rn(__dmul_rn(0.544974750228521, dt), 1.0)); break;
      default:
        v = __dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(0.517231671970585, tr[2]), __dmul_rn(0.096059710526147, tr[3])),
                                          __dmul_rn(__dmul_rn(0.063692468666290, dt), 1.0)),
                                __dmul_rn(0.386708617503269, tr[4])),
                      __dmul_rn(__dmul_rn(0.226007483236906, dt), 1.0));
        break;
    }
  }
  tr[s] = v;
  // reset the post_process outputs of this stage
  c->neg_avg = 0;
  c->num_negcell = 0;
  c->pp_relimit = 0;
  for (int v8 = 0; v8 < 8; ++v8) {
    c->umax_bits[v8] = 0ULL;
    c->umin_bits[v8] = ~0ULL;
  }
}

// after post_process of a stage (drive.f90:285-298): inadmissible average -> abandon the try;
// otherwise account the limiter count and arm the dt_lim reduction of the coming residual.
__device__ __forceinline__ void ctl_stage_end_body(Ctrl* c) {
  if (c->state != ST_RUN) return;
  if (c->neg_avg) {  // checked first: a stage whose loops 1 and 3 ran fused may also hold a
    c->state = ST_FAILED;  // re-limit failure that the reference, skipping loop 3, never reaches
    return;
  }
  if (c->pp_relimit) {
    c->flags |= 2;  // MHD_FLAG_PP_RELIMIT (the reference stops the program)
    c->state = ST_IDLE;
    return;
  }
  c->num_negcell_last = c->num_negcell;
  c->num_negcell_total += c->num_negcell;
  c->dt_lim_bits = ~0ULL;
  c->pending_dtlim = 1;
}

// end of a try: accept (drive.f90:304-312) or prepare the re-try.  dt_lim is the value of the
// last residual that ran, as in the reference, where every DG_semidiscretize overwrites it.
// An accepted step appends its record to the log (drive.f90:314 log_append(t, tot_ent)); the
// stage diagnostics of its final stage, which is the accepted state, are carried over.
__device__ __forceinline__ void ctl_step_end_body(Ctrl* c, int R, LogEntry* log = nullptr, int log_cap = 0) {
  if (c->pending_dtlim) {
    c->dt_lim = dec_dtlim(c->dt_lim_bits);
    c->pending_dtlim = 0;
  }
  if (c->state == ST_FAILED) {  // re-try with a smaller dt
    c->state = ST_IDLE;
    return;
  }
  if (c->state != ST_RUN) return;
  c->t = c->t_rk[R];
  c->steps += 1;
  const LogEntry* last = (log && log_cap > 0 && c->log_seq > 0) ? log + ((c->log_seq - 1) % log_cap) : nullptr;
  if (LogEntry* e = log_next(log, log_cap, c)) {
    e->step = c->steps;
    e->kind = LOG_STEP;
    e->stage = R;
    e->try_num = c->try_num;
    e->num_negcell = 0;
    e->neg_avg = 0;
    e->flags = c->flags;
    e->t = c->t;
    e->dt = c->dt;
    e->dt_lim = c->dt_lim;
    e->tot_ent = c->tot_ent;
    if (last && last->kind == LOG_STAGE && last->step == c->steps && last->stage == R) {
      e->rho_min = last->rho_min;
      e->p_min = last->p_min;
      for (int v = 0; v < 8; ++v) e->total[v] = last->total[v];
    }
  }
  c->try_num = 0;
  if (c->last_step) c->done = 1;
  c->state = ST_IDLE;
}

// The record of a stage that reached its end (drive.f90:285-294): the PP-limited cell count, or
// the inadmissible average that abandons the try.  Called right after ctl_stage_end_body by the
// thread that ran it, for a stage that was running when its end was reached.
__device__ __forceinline__ void ctl_log_stage(Ctrl* c, int stage, LogEntry* log, int log_cap) {
  LogEntry* e = log_next(log, log_cap, c);
  if (!e) return;
  e->step = c->steps + 1;
  e->kind = LOG_STAGE;
  e->stage = stage;
  e->try_num = c->try_num;
  e->neg_avg = c->neg_avg;
  e->num_negcell = c->neg_avg ? 0 : c->num_negcell;
  e->flags = c->flags;
  e->t = c->t_rk[stage];
  e->dt = c->dt;
  e->dt_lim = __longlong_as_double(0x7ff8000000000000LL);
  e->tot_ent = c->tot_ent;
}

// the record of the initial state (drive.f90:74 log_append(0, tot_ent)), written by solve_begin
__global__ void ctl_log_initial(Ctrl* c, LogEntry* log, int log_cap) {
  LogEntry* e = log_next(log, log_cap, c);
  if (!e) return;
  e->step = 0;
  e->kind = LOG_STEP;
  e->stage = 0;
  e->try_num = 0;
  e->num_negcell = 0;
  e->neg_avg = 0;
  e->flags = c->flags;
  e->t = c->t;
  e->dt = 0.0;
  e->dt_lim = c->dt_lim;
  e->tot_ent = c->tot_ent;
}

__global__ void ctl_step_begin(Ctrl* c) { ctl_step_begin_body(c); }
__global__ void ctl_step_end(Ctrl* c, int R, LogEntry* log, int log_cap) { ctl_step_end_body(c, R, log, log_cap); }
// the dt of the try and the pseudo-time of its first stage, in one launch
__global__ void ctl_dt_stage1(Ctrl* c, int R) {
  ctl_dt_body(c);
  ctl_stage_time_body(c, R, 1);
}

// The starting control block of solve_execute (drive.f90:67-73) without a host round trip: the
// initial post_process and residual ran just before on this stream, and their outputs (neg_avg,
// tot_ent, the dt_lim reduction cell) become the first step's inputs.  An inadmissible initial
// value sets MHD_FLAG_INIT_NEG_AVG, which every later try treats as a failed run.
__global__ void ctl_solve_begin(Ctrl* c, double final_T, double cfl_total) {
  const int neg = c->neg_avg;
  const double te = c->tot_ent;
  const unsigned long long bits = c->dt_lim_bits;
  Ctrl z;
  memset(&z, 0, sizeof(z));
  z.final_T = final_T;
  z.cfl_total = cfl_total;
  z.state = ST_IDLE;
  z.step_limit = 0x7fffffffffffffffLL;
  if (neg) {
    z.flags = 8;  // MHD_FLAG_INIT_NEG_AVG
  } else {
    z.dt_lim = dec_dtlim(bits);
    z.tot_ent = te;
  }
  *c = z;
}

// the same decisions for every instance of a batch, one thread each
enum CtlOp : int { CTL_STEP_BEGIN = 0, CTL_DT_STAGE1 = 1, CTL_STEP_END = 2 };
__global__ void ctl_batched(const InstDesc* __restrict__ insts, const int* __restrict__ ninst, int op, int R, int s) {
  const int n = *ninst;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    Ctrl* c = insts[i].ctrl;
    switch (op) {
      case CTL_STEP_BEGIN: ctl_step_begin_body(c); break;
      case CTL_DT_STAGE1:
        ctl_dt_body(c);
        ctl_stage_time_body(c, R, 1);
        break;
      default: ctl_step_end_body(c, R, insts[i].log, insts[i].log_cap); break;
    }
  }
}

// status of every instance of a batch into one contiguous array (one copy to the host)
__global__ void ctl_gather_batched(const InstDesc* __restrict__ insts, const int* __restrict__ ninst,
                                   Ctrl* __restrict__ out) {
  const int n = *ninst;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = *insts[i].ctrl;
}

}  // namespace mhd
