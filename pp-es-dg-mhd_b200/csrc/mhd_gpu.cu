// mhd_gpu.cu -- C ABI (include/mhd_gpu.h) of the sm_100a DG-MHD stage pipeline.
//
// The handle replaces the reference's module-level state (DG_solver.f90:6-43) with device
// allocations; every entry point maps onto one reference procedure (see mhd_gpu.h).  The
// device-resident driver replays solve_execute's try/stage sequence (drive.f90:83-320) as one
// captured CUDA graph per time-step try: control decisions (dt, retry, acceptance) are made by
// single-thread control kernels on the device, so the host only polls a status block.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstddef>
#include <cstdlib>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/mhd_gpu.h"
#include "common.cuh"
#include "misc.cuh"
#include "post.cuh"
#include "residual.cuh"
#include "setup.cuh"
#include "tables.h"

using namespace mhd;

struct mhd_gpu {
  int nx, ny, p, n, nn, eb, R, bc_kind;
  double left, right, bottom, top, hx, hy, gamma, bc_state[8];
  int device;
  cudaStream_t stream;
  cudaStream_t own_stream;
  cudaStream_t side_stream;  // the OEDG global sums run here beside the face indicators
  cudaEvent_t ev_fork, ev_join;
  double* u[6];   // slot 0 = u_con, s = uRK_con(:,s)
  double* ut[6];  // 1..R
  double* u_avg;
  double* staging;
  double* ldfA;
  double* sig_x;
  double* sig_y;
  double* partial;
  double* ent_partial;
  double* cell_ent_DG;
  double* cell_ent_FV;
  unsigned char* cell_ent_nan;
  Ctrl* ctrl;
  Ctrl* ctrl_host;  // pinned mirror
  size_t bytes;
  void* block;      // the one device allocation every buffer above is carved from
  bool owns_block;  // false: the block was lent by a server and goes back to it
  Geo geo;
  // device-resident driver
  int solve_ready;
  int graph_kernels;  // kernel nodes of the captured step graph (0 before the first capture)
  double final_T, cfl;
  int use_oedg, use_ldf, ent_offset;
  cudaGraphExec_t step_exec;
  // driver log (mhd_gpu_set_log): a device ring of log_cap records, drained into log_host
  LogEntry* log;
  int log_cap;
  int diag;                    // run the stage diagnostics kernel after every stage
  double* diag_part;           // its block partials, followed by its ticket counter
  void* log_block;
  long long log_host_seq;      // records copied to the host so far
  long long log_dropped;       // records overwritten in the ring before they were copied
  std::vector<LogEntry>* log_host;
};

namespace {

const int kMaxDevices = 64;
std::mutex g_init_mutex;
bool g_dev_init[kMaxDevices];

#define CK(call)                                  \
  do {                                            \
    cudaError_t e_ = (call);                      \
    if (e_ != cudaSuccess) return MHD_ERR_CUDA;   \
  } while (0)

// Where each buffer of an instance sits in its one device block (256-byte aligned pieces).
struct InstLayout {
  size_t u[6], ut[6], u_avg, staging, ldfA, sig_x, sig_y, partial, ent_partial, cell_ent_DG, cell_ent_FV,
      cell_ent_nan, ctrl, total;
};

InstLayout inst_layout(int nx, int ny, int p, int R) {
  InstLayout L;
  std::memset(&L, 0, sizeof(L));
  size_t off = 0;
  auto take = [&off](size_t bytes) {
    const size_t at = off;
    off += (bytes + 255) / 256 * 256;
    return at;
  };
  const size_t eb = 8 * (size_t)(p + 1) * (p + 1);
  const size_t nelg = (size_t)(nx + 2) * (ny + 2);
  const size_t sb = sizeof(double) * nelg * eb, tb = sizeof(double) * (size_t)nx * ny * eb;
  for (int s = 0; s <= R; ++s) L.u[s] = take(sb);
  for (int s = 1; s <= R; ++s) L.ut[s] = take(tb);
  L.u_avg = take(sizeof(double) * 8 * nelg);
  L.staging = take(sb);
  const size_t n2 = 2 * (size_t)(p + 1) * (p + 1);
  L.ldfA = take(sizeof(double) * n2 * n2);
  L.sig_x = take(sizeof(double) * 8 * (size_t)(nx + 1) * ny);
  L.sig_y = take(sizeof(double) * 8 * (size_t)nx * (ny + 1));
  const size_t te_min = pp_min_chunk();  // the smallest elements-per-CTA of the post-process kernels
  L.partial = take(sizeof(double) * 8 * ((nelg + te_min - 1) / te_min + 1));
  L.ent_partial = take(sizeof(double) * (((size_t)nx + te_min - 1) / te_min + 1) * ny);
  L.cell_ent_DG = take(sizeof(double) * nelg);
  L.cell_ent_FV = take(sizeof(double) * nelg);
  L.cell_ent_nan = take(nelg);
  L.ctrl = take(sizeof(Ctrl));
  L.total = off;
  return L;
}

long long n_state(const mhd_gpu* h) { return (long long)(h->nx + 2) * (h->ny + 2) * h->eb; }
long long n_ut(const mhd_gpu* h) { return (long long)h->nx * h->ny * h->eb; }
int grid1d(long long n, int bs) { return (int)((n + bs - 1) / bs); }

template <int P>
int pp_nblk_avg(const mhd_gpu* h) { return grid1d((long long)(h->nx + 2) * (h->ny + 2), PPCfg<P>::TE); }
template <int P>
dim3 pp_grid_limit(const mhd_gpu* h) { return dim3((h->nx + PPCfg<P>::TEL - 1) / PPCfg<P>::TEL, h->ny); }

// CTAs of pp_avg_ldf_kernel<P> the device holds at once (its grid walks the chunks)
template <int P, bool NEEDG>
int pp_resident_ctas(int dev) {
  static int cached[kMaxDevices];
  if (dev < 0 || dev >= kMaxDevices) return 1;
  if (!cached[dev]) {
    int nsm = 0, per_sm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pp_avg_ldf_kernel<P, NEEDG>, PPCfg<P>::NT, 0);
    cached[dev] = std::max(1, nsm) * std::max(1, per_sm);
  }
  return cached[dev];
}

int init_device_tables(int dev) {
  std::lock_guard<std::mutex> lk(g_init_mutex);
  if (dev < 0 || dev >= kMaxDevices) return MHD_ERR_INVALID;
  if (g_dev_init[dev]) return MHD_OK;
  DegConst tabs[MAXP + 1];
  std::memset(tabs, 0, sizeof(tabs));
  for (int p = 1; p <= MAXP; ++p) {
    const int n = p + 1;
    double x[8], w[8], D[64], R0[64], RN[64];
    if (tables::gll(p, x, w, nullptr, nullptr, D, nullptr, nullptr)) return MHD_ERR_INVALID;
    if (tables::dpow_rows(p, R0, RN)) return MHD_ERR_INVALID;
    for (int i = 0; i < n; ++i) {
      tabs[p].qx[i] = x[i];
      tabs[p].qw[i] = w[i];
      tabs[p].iqw[i] = 1.0 / w[i];
    }
    for (int i = 0; i < n * n; ++i) tabs[p].D[i] = D[i];
    for (int kk = 0; kk <= p; ++kk)
      for (int k = 0; k < n; ++k) {
        tabs[p].R0[kk][k] = R0[kk * n + k];
        tabs[p].RN[kk][k] = RN[kk * n + k];
      }
  }
  CK(cudaMemcpyToSymbol(c_deg, tabs, sizeof(tabs)));
  CK(cudaFuncSetAttribute(residual2_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Res2Layout<1>::BYTES));
  CK(cudaFuncSetAttribute(residual2_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Res2Layout<2>::BYTES));
  CK(cudaFuncSetAttribute(residual2_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Res2Layout<3>::BYTES));
  CK(cudaFuncSetAttribute(residual2_batched<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Res2Layout<1>::BYTES));
  CK(cudaFuncSetAttribute(residual2_batched<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Res2Layout<2>::BYTES));
  CK(cudaFuncSetAttribute(residual2_batched<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Res2Layout<3>::BYTES));
  CK(cudaFuncSetAttribute(residual2_persistent<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Res2Layout<1>::BYTES));
  CK(cudaFuncSetAttribute(residual2_persistent<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Res2Layout<2>::BYTES));
  CK(cudaFuncSetAttribute(residual2_persistent<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Res2Layout<3>::BYTES));
  g_dev_init[dev] = true;
  return MHD_OK;
}

// Instance buffers come from one memory pool per device that keeps freed memory reserved
// (release threshold = all), so creating and destroying instances in a serving loop neither
// pays cudaMalloc/cudaFree nor synchronises the device.
cudaMemPool_t g_pool[kMaxDevices];
bool g_pool_ready[kMaxDevices];

int device_pool(int dev, cudaMemPool_t* pool) {
  std::lock_guard<std::mutex> lk(g_init_mutex);
  if (!g_pool_ready[dev]) {
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    CK(cudaMemPoolCreate(&g_pool[dev], &props));
    unsigned long long thr = ~0ULL;
    CK(cudaMemPoolSetAttribute(g_pool[dev], cudaMemPoolAttrReleaseThreshold, &thr));
    g_pool_ready[dev] = true;
  }
  *pool = g_pool[dev];
  return MHD_OK;
}

int enter(const mhd_gpu* h) {
  if (!h) return MHD_ERR_INVALID;
  CK(cudaSetDevice(h->device));
  return MHD_OK;
}

// ---- launchers ---------------------------------------------------------------------------
template <int P>
void launch_bc(mhd_gpu* h, double* u, int gate) {
  constexpr int EB = 8 * (P + 1) * (P + 1);
  const long long n = 2LL * (h->nx + h->ny) * EB;
  bc_kernel<P><<<grid1d(n, 256), 256, 0, h->stream>>>(u, h->geo, h->ctrl, gate);
}

// ug: the array whose ghost ring the boundary halos come from (nullptr: u's own)
template <int P>
void launch_residual(mhd_gpu* h, const double* u, double* ut, int gate, StageCombine sc = StageCombine{},
                     const double* ug = nullptr) {
  using L = Res2Layout<P>;
  dim3 grid((h->nx + L::TX - 1) / L::TX, (h->ny + L::TY - 1) / L::TY);
  residual2_kernel<P><<<grid, L::NT, L::BYTES, h->stream>>>(u, ug ? ug : u, ut, h->geo, h->ctrl, gate, sc);
}

// the re-try residual of a try (gate ST_RECOMPUTE, usually closed): a persistent grid of the CTAs
// the device holds at once
template <int P>
int res_resident_ctas(int dev) {
  static int cached[kMaxDevices];
  if (dev < 0 || dev >= kMaxDevices) return 1;
  if (!cached[dev]) {
    int nsm = 0, per_sm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, residual2_persistent<P>, Res2Layout<P>::NT,
                                                  Res2Layout<P>::BYTES);
    cached[dev] = std::max(1, nsm) * std::max(1, per_sm);
  }
  return cached[dev];
}
template <int P>
void launch_residual_retry(mhd_gpu* h, const double* u, double* ut) {
  using L = Res2Layout<P>;
  const int ntx = (h->nx + L::TX - 1) / L::TX, ntiles = ntx * ((h->ny + L::TY - 1) / L::TY);
  residual2_persistent<P><<<std::min(ntiles, res_resident_ctas<P>(h->device)), L::NT, L::BYTES, h->stream>>>(
      u, ut, h->geo, h->ctrl, ST_RECOMPUTE, ntx, ntiles);
}

template <int P>
void launch_combine(mhd_gpu* h, int stage, const double* dt_ptr, double dt, int gate) {
  constexpr int EB = 8 * (P + 1) * (P + 1);
  const long long n = (long long)h->nx * h->ny * EB;
  combine_kernel<EB><<<grid1d(n, 256), 256, 0, h->stream>>>(
      h->u[0], h->u[1], h->R >= 2 ? h->u[2] : nullptr, h->R >= 3 ? h->u[3] : nullptr, h->R >= 4 ? h->u[4] : nullptr,
      h->ut[1], h->R >= 2 ? h->ut[2] : nullptr, h->R >= 3 ? h->ut[3] : nullptr, h->R >= 4 ? h->ut[4] : nullptr,
      h->R >= 5 ? h->ut[5] : nullptr, h->u[stage], h->nx, h->ny, h->R, stage, dt_ptr, dt, h->ctrl, gate);
}

// post_process on slot `slot` (everything but the control-block reset and the host read-back)
template <int P>
// fuse = 1 (time-step pipeline only): a stage without OEDG, entropy or acceptance copy runs loops
// 1 and 3 in one kernel (the stage result is discarded if an average is inadmissible)
// s1 (time-step pipeline, stage 1 only): loop 1 forms the stage state from u0 and the stage-1
// residual, with its ghost ring, in place of the combination and boundary-fill launches
// entsum_later (time-step pipeline): the entropy sum is left to the stage-end launch
// accept_only (with accept_dst): the limiter writes its result to accept_dst only, leaving slot's
// interior as loop 1 left it
void launch_post(mhd_gpu* h, int slot, int apply_oedg, int apply_ldf, const double* dt_ptr, double oedg_dt,
                 int ent_offset, int comput_ent, double* accept_dst, int gate, int fuse = 0,
                 Stage1Src s1 = Stage1Src{}, bool entsum_later = false, int accept_only = 0) {
  const int nb1 = pp_nblk_avg<P>(h);
  const int limit_in_loop1 = fuse && !apply_oedg && !comput_ent && !accept_dst;
  if (apply_oedg) {
    const int grid1 = std::min(nb1, pp_resident_ctas<P, true>(h->device));
    pp_avg_ldf_kernel<P, true><<<grid1, PPCfg<P>::NT, 0, h->stream>>>(h->u[slot], h->u_avg, h->geo, h->ctrl, gate, apply_ldf,
                                                                1, ent_offset, h->partial, h->cell_ent_DG,
                                                                h->cell_ent_FV, h->cell_ent_nan, limit_in_loop1, nb1, s1);
  } else {
    const int grid1 = std::min(nb1, pp_resident_ctas<P, false>(h->device));
    pp_avg_ldf_kernel<P, false><<<grid1, PPCfg<P>::NT, 0, h->stream>>>(h->u[slot], h->u_avg, h->geo, h->ctrl, gate, apply_ldf,
                                                                 0, ent_offset, h->partial, h->cell_ent_DG,
                                                                 h->cell_ent_FV, h->cell_ent_nan, limit_in_loop1, nb1, s1);
  }
  if (limit_in_loop1) return;
  if (apply_oedg) {  // the global sums (one CTA) and the face indicators are independent: fork/join
    cudaEventRecord(h->ev_fork, h->stream);
    cudaStreamWaitEvent(h->side_stream, h->ev_fork, 0);
    pp_reduce_kernel<<<1, 256, 0, h->side_stream>>>(h->partial, nb1, h->ctrl, gate);
    cudaEventRecord(h->ev_join, h->side_stream);
    const dim3 gs((h->nx + SigCfg<P>::TX - 1) / SigCfg<P>::TX, (h->ny + SigCfg<P>::TY - 1) / SigCfg<P>::TY);
    pp_sigsum_kernel<P><<<gs, 256, 0, h->stream>>>(h->u[slot], h->geo, h->ctrl, gate, h->sig_x, h->sig_y);
    cudaStreamWaitEvent(h->stream, h->ev_join, 0);
  }
  dim3 g3 = pp_grid_limit<P>(h);
  pp_limit_kernel<P><<<g3, PPCfg<P>::NT, 0, h->stream>>>(h->u[slot], h->u_avg, h->geo, h->ctrl, gate, apply_oedg, dt_ptr,
                                                   oedg_dt, ent_offset, comput_ent, h->sig_x, h->sig_y,
                                                   h->cell_ent_DG, h->cell_ent_FV, h->cell_ent_nan,
                                                   h->ent_partial, accept_dst, accept_only);
  if (comput_ent && !entsum_later)
    pp_entsum_kernel<<<1, 256, 0, h->stream>>>(h->ent_partial, (int)(g3.x * g3.y), h->ctrl, gate);
}

// stage diagnostics of state u into the newest log record
template <int P>
void launch_diag(mhd_gpu* h, const double* u, int gate) {
  const long long E = (long long)h->nx * h->ny;
  const int nb = (int)std::min<long long>(DIAG_MAX_BLOCKS, std::max<long long>(1, E / 16));
  stage_diag_kernel<P><<<nb, 256, 0, h->stream>>>(u, h->geo, h->ctrl, gate, h->diag_part,
                                                   reinterpret_cast<unsigned int*>(h->diag_part + DIAG_VALS * DIAG_MAX_BLOCKS),
                                                   h->log, h->log_cap);
}

#define DISPATCH_P(h, fn, ...)              \
  do {                                      \
    switch ((h)->p) {                       \
      case 1: fn<1>(__VA_ARGS__); break;    \
      case 2: fn<2>(__VA_ARGS__); break;    \
      default: fn<3>(__VA_ARGS__); break;   \
    }                                       \
  } while (0)

int read_ctrl(mhd_gpu* h) {
  CK(cudaMemcpyAsync(h->ctrl_host, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return MHD_OK;
}

// Copy the log records written since the last drain from the device ring to the host buffer.
// Needs a fresh ctrl_host (read_ctrl) and an idle stream.  Records the ring overwrote before they
// could be copied are counted in log_dropped.
int drain_log(mhd_gpu* h) {
  if (!h->log) return MHD_OK;
  const long long dev_seq = h->ctrl_host->log_seq;
  long long from = h->log_host_seq;
  if (dev_seq <= from) return MHD_OK;
  if (dev_seq - from > h->log_cap) {
    h->log_dropped += dev_seq - from - h->log_cap;
    from = dev_seq - h->log_cap;
  }
  const long long cnt = dev_seq - from;
  std::vector<LogEntry>& out = *h->log_host;
  const size_t at = out.size();
  out.resize(at + (size_t)cnt);
  const long long first = from % h->log_cap;
  const long long run1 = std::min<long long>(cnt, h->log_cap - first);
  CK(cudaMemcpyAsync(out.data() + at, h->log + first, sizeof(LogEntry) * run1, cudaMemcpyDeviceToHost, h->stream));
  if (cnt > run1)
    CK(cudaMemcpyAsync(out.data() + at + run1, h->log, sizeof(LogEntry) * (cnt - run1), cudaMemcpyDeviceToHost,
                       h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->log_host_seq = dev_seq;
  return MHD_OK;
}

void fill_status(const mhd_gpu* h, mhd_gpu_status* st) {
  if (!st) return;
  const Ctrl* c = h->ctrl_host;
  st->t = c->t;
  st->dt = c->dt;
  st->dt_lim = c->dt_lim;
  st->tot_ent = c->tot_ent;
  st->steps = c->steps;
  st->retries = c->retries;
  st->num_negcell_total = c->num_negcell_total;
  st->num_negcell_last = c->num_negcell_last;
  st->done = c->done;
  st->flags = c->flags;
  st->pad_ = 0;
}

// one try of a time step (drive.f90:93-300), recorded into the capturing stream
// the combination of stage `stage` (SSP-RK(2,2) stage 2, SSP-RK(3,3) stages 2 and 3; the
// coefficients of combine_value) folded into the previous residual; none otherwise
StageCombine next_stage_combine(const mhd_gpu* h, int stage) {
  StageCombine sc{};
  if (h->R == 2 && stage == 2) {
    sc = StageCombine{h->u[0], h->u[2], 0.5, 0.5, &h->ctrl->dt};
  } else if (h->R == 3 && (stage == 2 || stage == 3)) {
    sc = StageCombine{h->u[0], h->u[stage], stage == 2 ? 0.75 : 1.0 / 3.0, stage == 2 ? 0.25 : 2.0 / 3.0, &h->ctrl->dt};
  }
  return sc;
}

template <int P>
void enqueue_try(mhd_gpu* h) {
  const int R = h->R;
  ctl_step_begin<<<1, 1, 0, h->stream>>>(h->ctrl);
  launch_residual_retry<P>(h, h->u[0], h->ut[1]);
  ctl_dt_stage1<<<1, 1, 0, h->stream>>>(h->ctrl, R);  // dt, and the pseudo-time of stage 1
  // SSP-RK(2,2) and (3,3): stages after the first take their combination from the previous
  // stage's residual (next_stage_combine); SSP-RK(1,1) and (5,4) keep the separate combine
  constexpr int EB = 8 * (P + 1) * (P + 1);
  const long long nghost = 2LL * (h->nx + h->ny) * EB;
  const int nseg = (int)(pp_grid_limit<P>(h).x * pp_grid_limit<P>(h).y);
  for (int s = 1; s <= R; ++s) {
    const int fin = (s == R);
    // stage 1: loop 1 forms the stage state and its ghost ring (Stage1Src)
    if (s > 1 && R > 3) launch_combine<P>(h, s, &h->ctrl->dt, 0.0, ST_RUN);
    if (s > 1) launch_bc<P>(h, h->u[s], ST_RUN);
    const Stage1Src s1 = s == 1 ? Stage1Src{h->u[0], h->ut[1], &h->ctrl->dt, stage1_coef(R)} : Stage1Src{};
    // the final stage's limiter writes the accepted interior to u_con only (drive.f90:304-311); the
    // stage array's ghost ring is then filled from u_con, and the next step's stage-1 residual reads
    // u_con's interior with that ring.  u_con keeps its own ghost ring, which only the re-try
    // residual reads (drive.f90:104 takes u_con as it is).
    launch_post<P>(h, s, h->use_oedg && fin, h->use_ldf, &h->ctrl->dt, 0.0, h->ent_offset, fin,
                   fin ? h->u[0] : nullptr, ST_RUN, 1, s1, /*entsum_later=*/true, /*accept_only=*/fin);
    const double* cur = fin ? h->u[0] : h->u[s];  // the stage result's interior
    // entropy sum (final stage), stage-end decision, next stage's pseudo-time and the ghost ring
    stage_end_bc_kernel<P><<<grid1d(nghost, 256), 256, 0, h->stream>>>(
        cur, h->u[s], h->geo, h->ctrl, R, s, fin ? 0 : s + 1, fin ? h->ent_partial : nullptr, nseg, h->log,
        h->log_cap);
    if (h->diag) launch_diag<P>(h, cur, ST_RUN);
    launch_residual<P>(h, cur, h->ut[(s % R) + 1], ST_RUN, fin ? StageCombine{} : next_stage_combine(h, s + 1),
                       h->u[s]);
  }
  ctl_step_end<<<1, 1, 0, h->stream>>>(h->ctrl, R, h->log, h->log_cap);
}

// kernel nodes of a graph (every launch of the captured try, gated ones included)
int count_kernel_nodes(cudaGraph_t graph) {
  size_t n = 0;
  if (cudaGraphGetNodes(graph, nullptr, &n) != cudaSuccess || n == 0) return 0;
  std::vector<cudaGraphNode_t> nodes(n);
  if (cudaGraphGetNodes(graph, nodes.data(), &n) != cudaSuccess) return 0;
  int k = 0;
  for (size_t i = 0; i < n; ++i) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++k;
  }
  return k;
}

int build_step_graph(mhd_gpu* h) {
  if (h->step_exec) {
    cudaGraphExecDestroy(h->step_exec);
    h->step_exec = nullptr;
  }
  cudaGraph_t graph;
  CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  DISPATCH_P(h, enqueue_try, h);
  cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
  if (e != cudaSuccess) return MHD_ERR_CUDA;
  h->graph_kernels = count_kernel_nodes(graph);
  e = cudaGraphInstantiate(&h->step_exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return MHD_ERR_CUDA;
  return MHD_OK;
}

void free_all(mhd_gpu* h) {
  if (!h) return;
  if (h->step_exec) cudaGraphExecDestroy(h->step_exec);
  if (h->side_stream) {
    cudaStreamSynchronize(h->side_stream);
    cudaStreamDestroy(h->side_stream);
  }
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->ev_join) cudaEventDestroy(h->ev_join);
  cudaStream_t fs = h->own_stream;  // a stream-ordered free back into the device pool
  if (h->block && h->owns_block) cudaFreeAsync(h->block, fs);
  if (h->log_block) cudaFreeAsync(h->log_block, fs);
  delete h->log_host;
  h->log_host = nullptr;
  if (fs) {
    cudaStreamSynchronize(fs);
    cudaStreamDestroy(fs);
  }
  std::free(h->ctrl_host);
}

}  // namespace

// =============================================================================================
extern "C" {

const char* mhd_gpu_status_string(int code) {
  switch (code) {
    case MHD_OK: return "ok";
    case MHD_FLAG_NEG_AVG: return "inadmissible cell average";
    case MHD_FLAG_PP_RELIMIT: return "positivity re-limit failed";
    case MHD_FLAG_DT_COLLAPSE: return "time step collapsed (too many re-tries or dt_lim < 1e-14)";
    case MHD_FLAG_INIT_NEG_AVG: return "initial value has an inadmissible cell average";
    case MHD_FLAG_DEVICE_WAIT: return "a kernel's wait for its asynchronous copy ran out";
    case MHD_ERR_INVALID: return "invalid argument";
    case MHD_ERR_UNSUPPORTED: return "unsupported configuration";
    case MHD_ERR_CUDA: return "CUDA runtime error";
    case MHD_ERR_NO_DEVICE: return "no CUDA device";
    case MHD_ERR_STATE: return "call out of order";
    default: return "solver flags set";
  }
}

int mhd_gpu_gll_tables(int p, double* x, double* w, double* M, double* Minv, double* D, double* Pmn, double* Pnm) {
  if (p < 0 || p > 6) return MHD_ERR_INVALID;
  return tables::gll(p, x, w, M, Minv, D, Pmn, Pnm) ? MHD_ERR_INVALID : MHD_OK;
}

}  // extern "C"

namespace {

// mhd_gpu_create.  With sync = false the set-up work stays queued on the instance's own stream.
// u0 (may be NULL): an initial state in the Fortran layout, uploaded into slot 0.  Its host-to-device
// copy and the LDF table's are queued before any kernel, so that (from pageable memory, where the
// copy first waits for the stream's earlier work) the host never waits for the device.
// block (may be NULL): device memory of at least inst_layout(...).total bytes lent by the caller,
// which takes it back after mhd_gpu_destroy; NULL: one allocation from the device pool.
int create_instance(int nx, int ny, int px, int py, int rknstg, double left, double right, double bottom,
                    double top, double gamma, int bc_kind, const double* bc_state8, const double* u0, bool sync,
                    void* block, mhd_gpu_t** out) {
  if (!out) return MHD_ERR_INVALID;
  *out = nullptr;
  if (nx < 2 || ny < 2 || !(right > left) || !(top > bottom) || !(gamma > 1.0)) return MHD_ERR_INVALID;
  if (px != py || px < 1 || px > MAXP) return MHD_ERR_UNSUPPORTED;
  if (!(rknstg == 1 || rknstg == 2 || rknstg == 3 || rknstg == 5)) return MHD_ERR_UNSUPPORTED;
  if (bc_kind < 0 || bc_kind > 5) return MHD_ERR_INVALID;
  if ((bc_kind == MHD_BC_FIXED || bc_kind == MHD_BC_CLOUD_SHOCK || bc_kind == MHD_BC_JET) && !bc_state8)
    return MHD_ERR_INVALID;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MHD_ERR_NO_DEVICE;
  mhd_gpu* h = new (std::nothrow) mhd_gpu;
  if (!h) return MHD_ERR_INVALID;
  std::memset(h, 0, sizeof(*h));
  if (cudaGetDevice(&h->device) != cudaSuccess) {
    delete h;
    return MHD_ERR_CUDA;
  }
  int rc = init_device_tables(h->device);
  if (rc) {
    delete h;
    return rc;
  }
  h->nx = nx;
  h->ny = ny;
  h->p = px;
  h->n = px + 1;
  h->nn = h->n * h->n;
  h->eb = 8 * h->nn;
  h->R = rknstg;
  h->bc_kind = bc_kind;
  h->left = left;
  h->right = right;
  h->bottom = bottom;
  h->top = top;
  h->gamma = gamma;
  h->hx = (right - left) / nx;  // DG_solver.f90:93-94
  h->hy = (top - bottom) / ny;
  for (int v = 0; v < 8; ++v) h->bc_state[v] = bc_state8 ? bc_state8[v] : 0.0;
  cudaMemPool_t pool;
  if (device_pool(h->device, &pool) || cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->side_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming) != cudaSuccess) {
    free_all(h);
    delete h;
    return MHD_ERR_CUDA;
  }
  h->stream = h->own_stream;
  const InstLayout L = inst_layout(nx, ny, px, rknstg);
  if (block) {
    h->block = block;
    h->owns_block = false;
  } else {
    if (cudaMallocFromPoolAsync(&h->block, L.total, pool, h->own_stream) != cudaSuccess) {
      h->block = nullptr;
      free_all(h);
      delete h;
      return MHD_ERR_CUDA;
    }
    h->owns_block = true;
  }
  h->bytes = L.total;
  char* base = static_cast<char*>(h->block);
  for (int s = 0; s <= rknstg; ++s) h->u[s] = reinterpret_cast<double*>(base + L.u[s]);
  for (int s = 1; s <= rknstg; ++s) h->ut[s] = reinterpret_cast<double*>(base + L.ut[s]);
  h->u_avg = reinterpret_cast<double*>(base + L.u_avg);
  h->staging = reinterpret_cast<double*>(base + L.staging);
  h->ldfA = reinterpret_cast<double*>(base + L.ldfA);
  h->sig_x = reinterpret_cast<double*>(base + L.sig_x);
  h->sig_y = reinterpret_cast<double*>(base + L.sig_y);
  h->partial = reinterpret_cast<double*>(base + L.partial);
  h->ent_partial = reinterpret_cast<double*>(base + L.ent_partial);
  h->cell_ent_DG = reinterpret_cast<double*>(base + L.cell_ent_DG);
  h->cell_ent_FV = reinterpret_cast<double*>(base + L.cell_ent_FV);
  h->cell_ent_nan = reinterpret_cast<unsigned char*>(base + L.cell_ent_nan);
  h->ctrl = reinterpret_cast<Ctrl*>(base + L.ctrl);
  const size_t sb = sizeof(double) * (size_t)n_state(h), tb = sizeof(double) * (size_t)n_ut(h);
  const long long nelg = (long long)(nx + 2) * (ny + 2);
  const int n2 = 2 * h->nn;
  h->ctrl_host = static_cast<Ctrl*>(std::calloc(1, sizeof(Ctrl)));
  if (!h->ctrl_host) {
    free_all(h);
    delete h;
    return MHD_ERR_CUDA;
  }
  if (u0) cudaMemcpyAsync(h->staging, u0, sb, cudaMemcpyHostToDevice, h->stream);
  double A[32 * 32];
  tables::ldf_nodal_operator(px, h->hx, h->hy, A);
  cudaMemcpyAsync(h->ldfA, A, sizeof(double) * n2 * n2, cudaMemcpyHostToDevice, h->stream);
  // NaN-filled state, as the reference allocates with ieee_signaling_nan (DG_solver.f90:56,68-71)
  for (int s = 0; s <= rknstg; ++s) cudaMemsetAsync(h->u[s], 0xFF, sb, h->stream);
  for (int s = 1; s <= rknstg; ++s) cudaMemsetAsync(h->ut[s], 0xFF, tb, h->stream);
  cudaMemsetAsync(h->u_avg, 0xFF, sizeof(double) * 8 * nelg, h->stream);
  cudaMemsetAsync(h->ctrl, 0, sizeof(Ctrl), h->stream);
  if (u0) to_blocked_kernel<<<grid1d(nelg * h->eb, 256), 256, 0, h->stream>>>(h->staging, h->u[0], nelg, h->nn);
  h->geo.nx = nx;
  h->geo.ny = ny;
  h->geo.hx = h->hx;
  h->geo.hy = h->hy;
  h->geo.gamma = gamma;
  h->geo.bc_kind = bc_kind;
  for (int v = 0; v < 8; ++v) h->geo.bc_state[v] = h->bc_state[v];
  h->geo.ldfA = h->ldfA;
  if ((sync ? cudaStreamSynchronize(h->stream) : cudaGetLastError()) != cudaSuccess) {
    free_all(h);
    delete h;
    return MHD_ERR_CUDA;
  }
  *out = h;
  return MHD_OK;
}

}  // namespace

extern "C" {

int mhd_gpu_create(int nx, int ny, int px, int py, int rknstg, double left, double right, double bottom,
                   double top, double gamma, int bc_kind, const double* bc_state8, mhd_gpu_t** out) {
  return create_instance(nx, ny, px, py, rknstg, left, right, bottom, top, gamma, bc_kind, bc_state8, nullptr, true,
                         nullptr, out);
}

int mhd_gpu_destroy(mhd_gpu_t* h) {
  if (!h) return MHD_ERR_INVALID;
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->stream);
  free_all(h);
  delete h;
  return MHD_OK;
}

int mhd_gpu_set_stream(mhd_gpu_t* h, void* stream) {
  int rc = enter(h);
  if (rc) return rc;
  CK(cudaStreamSynchronize(h->stream));
  h->stream = stream ? (cudaStream_t)stream : h->own_stream;
  if (h->step_exec) {  // recaptured on the new stream by the next advance
    cudaGraphExecDestroy(h->step_exec);
    h->step_exec = nullptr;
  }
  return MHD_OK;
}

int mhd_gpu_device_bytes(const mhd_gpu_t* h, size_t* bytes) {
  if (!h || !bytes) return MHD_ERR_INVALID;
  *bytes = h->bytes;
  return MHD_OK;
}

int mhd_gpu_synchronize(mhd_gpu_t* h) {
  int rc = enter(h);
  if (rc) return rc;
  CK(cudaStreamSynchronize(h->stream));
  return MHD_OK;
}

int mhd_gpu_nodes(const mhd_gpu_t* h, double* xx, double* yy) {
  if (!h) return MHD_ERR_INVALID;
  double x[8], w[8];
  tables::gll(h->p, x, w, nullptr, nullptr, nullptr, nullptr, nullptr);
  const int n = h->n;
  if (xx)  // DG_solver.f90:101-103
    for (int i = 1; i <= h->nx; ++i)
      for (int k = 0; k < n; ++k) xx[k + n * (i - 1)] = (0.5 * h->hx) * x[k] + (h->left + (i - 0.5) * h->hx);
  if (yy)
    for (int j = 1; j <= h->ny; ++j)
      for (int l = 0; l < n; ++l) yy[l + n * (j - 1)] = (0.5 * h->hy) * x[l] + (h->bottom + (j - 0.5) * h->hy);
  return MHD_OK;
}

int mhd_gpu_ldf_operator(int p, double hx, double hy, double* A) {
  if (!A || p < 1 || p > 6 || !(hx > 0.0) || !(hy > 0.0)) return MHD_ERR_INVALID;
  return tables::ldf_nodal_operator(p, hx, hy, A) ? MHD_ERR_INVALID : MHD_OK;
}

static int transfer_in(mhd_gpu* h, const double* src, double* dst, long long nelem, bool sync = true) {
  const long long n = nelem * h->eb;
  CK(cudaMemcpyAsync(h->staging, src, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
  to_blocked_kernel<<<grid1d(n, 256), 256, 0, h->stream>>>(h->staging, dst, nelem, h->nn);
  CK(cudaGetLastError());
  if (sync) CK(cudaStreamSynchronize(h->stream));
  return MHD_OK;
}
static int transfer_out(mhd_gpu* h, const double* src, double* dst, long long nelem) {
  const long long n = nelem * h->eb;
  to_fortran_kernel<<<grid1d(n, 256), 256, 0, h->stream>>>(src, h->staging, nelem, h->nn);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(dst, h->staging, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return MHD_OK;
}

int mhd_gpu_upload_state(mhd_gpu_t* h, int slot, const double* u) {
  int rc = enter(h);
  if (rc) return rc;
  if (!u || slot < 0 || slot > h->R) return MHD_ERR_INVALID;
  return transfer_in(h, u, h->u[slot], (long long)(h->nx + 2) * (h->ny + 2));
}
int mhd_gpu_download_state(mhd_gpu_t* h, int slot, double* u) {
  int rc = enter(h);
  if (rc) return rc;
  if (!u || slot < 0 || slot > h->R) return MHD_ERR_INVALID;
  return transfer_out(h, h->u[slot], u, (long long)(h->nx + 2) * (h->ny + 2));
}
int mhd_gpu_upload_ut(mhd_gpu_t* h, int stage, const double* ut) {
  int rc = enter(h);
  if (rc) return rc;
  if (!ut || stage < 1 || stage > h->R) return MHD_ERR_INVALID;
  return transfer_in(h, ut, h->ut[stage], (long long)h->nx * h->ny);
}
int mhd_gpu_download_ut(mhd_gpu_t* h, int stage, double* ut) {
  int rc = enter(h);
  if (rc) return rc;
  if (!ut || stage < 1 || stage > h->R) return MHD_ERR_INVALID;
  return transfer_out(h, h->ut[stage], ut, (long long)h->nx * h->ny);
}
int mhd_gpu_download_avg(mhd_gpu_t* h, double* u_avg) {
  int rc = enter(h);
  if (rc) return rc;
  if (!u_avg) return MHD_ERR_INVALID;
  CK(cudaMemcpyAsync(u_avg, h->u_avg, sizeof(double) * 8 * (size_t)(h->nx + 2) * (h->ny + 2),
                     cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return MHD_OK;
}

int mhd_gpu_download_avg_primitive(mhd_gpu_t* h, float* buffer_var, double* var_min, double* var_max) {
  int rc = enter(h);
  if (rc) return rc;
  if (!buffer_var) return MHD_ERR_INVALID;
  const long long cells = (long long)(h->nx + 1) * h->ny;
  float* dout = reinterpret_cast<float*>(h->staging);  // 8*cells floats fit the staging buffer
  unsigned long long* mm = reinterpret_cast<unsigned long long*>(h->partial);  // 16 words of scratch
  unsigned long long init[16];
  for (int v = 0; v < 8; ++v) {
    init[v] = ~0ULL;
    init[8 + v] = 0ULL;
  }
  CK(cudaMemcpyAsync(mm, init, sizeof(init), cudaMemcpyHostToDevice, h->stream));
  avg_primitive_kernel<<<grid1d(cells, 256), 256, 0, h->stream>>>(h->u_avg, h->geo, dout, mm);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(buffer_var, dout, sizeof(float) * 8 * cells, cudaMemcpyDeviceToHost, h->stream));
  unsigned long long got[16];
  CK(cudaMemcpyAsync(got, mm, sizeof(got), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (int v = 0; v < 8; ++v) {
    if (var_min) var_min[v] = ord_dec_host(got[v]);
    if (var_max) var_max[v] = ord_dec_host(got[8 + v]);
  }
  return MHD_OK;
}

int mhd_gpu_init_problem(mhd_gpu_t* h, int problem, const double* params, int nparams) {
  int rc = enter(h);
  if (rc) return rc;
  if (problem < MHD_IC_OT2PI || problem > MHD_IC_JET || nparams < 0 || (nparams > 0 && !params))
    return MHD_ERR_INVALID;
  ProblemParams pp{};
  pp.id = problem;
  pp.amp = 1.0;
  pp.kappa = pp.mu = pp.p_inf = pp.bx0 = pp.by0 = 1.0;
  pp.cx = pp.cy = 0.0;
  auto arg = [&](int k, double dflt) { return k < nparams ? params[k] : dflt; };
  switch (problem) {
    case MHD_IC_VORTEX:
      pp.kappa = arg(0, 1.0);
      pp.mu = arg(1, 1.0);
      pp.p_inf = arg(2, 1.0);
      pp.bx0 = arg(3, 1.0);
      pp.by0 = arg(4, 1.0);
      if (nparams > 5) return MHD_ERR_INVALID;
      break;
    case MHD_IC_BLAST:
      pp.cx = arg(0, 0.0);
      pp.cy = arg(1, 0.0);
      if (nparams > 2) return MHD_ERR_INVALID;
      break;
    default:
      pp.amp = arg(0, 1.0);
      if (nparams > 1) return MHD_ERR_INVALID;
  }
  const long long n = (long long)(h->nx + 2) * (h->ny + 2) * h->nn;
  switch (h->p) {
    case 1: init_problem_kernel<1><<<grid1d(n, 256), 256, 0, h->stream>>>(h->u[0], h->geo, pp, h->left, h->bottom); break;
    case 2: init_problem_kernel<2><<<grid1d(n, 256), 256, 0, h->stream>>>(h->u[0], h->geo, pp, h->left, h->bottom); break;
    default: init_problem_kernel<3><<<grid1d(n, 256), 256, 0, h->stream>>>(h->u[0], h->geo, pp, h->left, h->bottom); break;
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->stream));
  return MHD_OK;
}

int mhd_gpu_apply_bc(mhd_gpu_t* h, int slot) {
  int rc = enter(h);
  if (rc) return rc;
  if (slot < 0 || slot > h->R) return MHD_ERR_INVALID;
  DISPATCH_P(h, launch_bc, h, h->u[slot], GATE_ALWAYS);
  CK(cudaGetLastError());
  return MHD_OK;
}

int mhd_gpu_post_process(mhd_gpu_t* h, int slot, int apply_oedg, int apply_ldf, double oedg_dt, int ent_offset,
                         int comput_ent, int* neg_avg, int* num_negcell, double* tot_ent) {
  int rc = enter(h);
  if (rc) return rc;
  if (slot < 0 || slot > h->R) return MHD_ERR_INVALID;
  ctl_pp_reset<<<1, 1, 0, h->stream>>>(h->ctrl, GATE_ALWAYS);
  DISPATCH_P(h, launch_post, h, slot, apply_oedg != 0, apply_ldf != 0, nullptr, oedg_dt, ent_offset != 0,
             comput_ent != 0, nullptr, GATE_ALWAYS);
  CK(cudaGetLastError());
  rc = read_ctrl(h);
  if (rc) return rc;
  const Ctrl* c = h->ctrl_host;
  if (neg_avg) *neg_avg = c->neg_avg;
  if (num_negcell) *num_negcell = c->neg_avg ? 0 : c->num_negcell;
  if (tot_ent) *tot_ent = (c->neg_avg || !comput_ent) ? NAN : c->tot_ent;  // DG_solver.f90:660
  return c->pp_relimit ? MHD_FLAG_PP_RELIMIT : MHD_OK;
}

int mhd_gpu_semidiscretize(mhd_gpu_t* h, int ut_stage, int slot, double* dt_lim) {
  int rc = enter(h);
  if (rc) return rc;
  if (slot < 0 || slot > h->R || ut_stage < 1 || ut_stage > h->R) return MHD_ERR_INVALID;
  CK(cudaMemsetAsync(&h->ctrl->dt_lim_bits, 0xFF, sizeof(unsigned long long), h->stream));
  DISPATCH_P(h, launch_residual, h, h->u[slot], h->ut[ut_stage], GATE_ALWAYS);
  CK(cudaGetLastError());
  if (dt_lim) {
    unsigned long long bits;
    CK(cudaMemcpyAsync(&bits, &h->ctrl->dt_lim_bits, sizeof(bits), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    double d;
    std::memcpy(&d, &bits, sizeof(d));
    *dt_lim = d;
  }
  return MHD_OK;
}

int mhd_gpu_rk_combine(mhd_gpu_t* h, int stage, double dt) {
  int rc = enter(h);
  if (rc) return rc;
  if (stage < 1 || stage > h->R) return MHD_ERR_INVALID;
  DISPATCH_P(h, launch_combine, h, stage, nullptr, dt, GATE_ALWAYS);
  CK(cudaGetLastError());
  return MHD_OK;
}

int mhd_gpu_rk_accept(mhd_gpu_t* h) {
  int rc = enter(h);
  if (rc) return rc;
  // the interior rows of uRK(:,rknstg) into u_con, ghost ring untouched (drive.f90:304-311): one
  // strided copy, a row of nx element blocks per grid row
  const size_t row = sizeof(double) * (size_t)h->eb * h->nx, pitch = sizeof(double) * (size_t)h->eb * (h->nx + 2);
  const size_t first = (size_t)h->eb * (h->nx + 2 + 1);  // element (1, 1)
  CK(cudaMemcpy2DAsync(h->u[0] + first, pitch, h->u[h->R] + first, pitch, row, h->ny, cudaMemcpyDeviceToDevice,
                       h->stream));
  return MHD_OK;
}

int mhd_gpu_solve_begin(mhd_gpu_t* h, double final_T, double cfl, int use_oedg, int use_ldf, int ent_offset,
                        double* tot_ent, double* dt_lim) {
  int rc = enter(h);
  if (rc) return rc;
  h->solve_ready = 0;
  // drive.f90:67-73
  rc = mhd_gpu_apply_bc(h, 0);
  if (rc) return rc;
  int neg = 0, nneg = 0;
  double te = 0.0;
  rc = mhd_gpu_post_process(h, 0, 0, use_ldf, 0.0, 0, 1, &neg, &nneg, &te);
  if (rc < 0) return rc;
  if (neg) return MHD_FLAG_INIT_NEG_AVG;
  rc = mhd_gpu_apply_bc(h, 0);
  if (rc) return rc;
  double dl = 0.0;
  rc = mhd_gpu_semidiscretize(h, 1, 0, &dl);
  if (rc) return rc;
  if (tot_ent) *tot_ent = te;
  if (dt_lim) *dt_lim = dl;
  h->final_T = final_T;
  h->cfl = cfl;
  h->use_oedg = use_oedg != 0;
  h->use_ldf = use_ldf != 0;
  h->ent_offset = ent_offset != 0;
  Ctrl c;
  std::memset(&c, 0, sizeof(c));
  c.t = 0.0;
  c.dt_lim = dl;
  c.final_T = final_T;
  c.cfl_total = ((h->R <= 3) ? 1.0 : 1.508) * cfl;  // CFL_RK * CFL (drive.f90:57-63,109)
  c.tot_ent = te;
  c.state = ST_IDLE;
  c.step_limit = 0x7fffffffffffffffLL;
  *h->ctrl_host = c;
  CK(cudaMemcpyAsync(h->ctrl, h->ctrl_host, sizeof(Ctrl), cudaMemcpyHostToDevice, h->stream));
  if (h->log) {  // a new run starts a new log: its first record is the initial state (drive.f90:74)
    h->log_host->clear();
    h->log_host_seq = 0;
    h->log_dropped = 0;
    ctl_log_initial<<<1, 1, 0, h->stream>>>(h->ctrl, h->log, h->log_cap);
    if (h->diag) DISPATCH_P(h, launch_diag, h, h->u[0], GATE_ALWAYS);
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(h->stream));
  if (h->step_exec) {  // the step graph is (re)captured lazily by the first advance
    cudaGraphExecDestroy(h->step_exec);
    h->step_exec = nullptr;
  }
  h->solve_ready = 1;
  return MHD_OK;
}

static int set_step_limit(mhd_gpu* h, long long limit) {
  CK(cudaMemcpyAsync(&h->ctrl->step_limit, &limit, sizeof(limit), cudaMemcpyHostToDevice, h->stream));
  return MHD_OK;
}

int mhd_gpu_get_status(mhd_gpu_t* h, mhd_gpu_status* st) {
  int rc = enter(h);
  if (rc) return rc;
  rc = read_ctrl(h);
  if (rc) return rc;
  fill_status(h, st);
  return h->ctrl_host->flags;
}

int mhd_gpu_advance(mhd_gpu_t* h, long long max_steps, int check_every, mhd_gpu_status* st) {
  int rc = enter(h);
  if (rc) return rc;
  if (!h->solve_ready) return MHD_ERR_STATE;
  if (check_every <= 0) check_every = 16;
  rc = read_ctrl(h);
  if (rc) return rc;
  if (!h->step_exec) {
    rc = build_step_graph(h);
    if (rc) return rc;
  }
  const long long start = h->ctrl_host->steps;
  const long long target = (max_steps > 0) ? start + max_steps : 0x7fffffffffffffffLL;
  rc = set_step_limit(h, target);
  if (rc) return rc;
  for (;;) {
    const Ctrl* c = h->ctrl_host;
    if (c->done || c->flags || c->steps >= target) break;
    // tries left before the target: retries need extra launches, so never queue more than
    // the remaining steps plus a small slack; extra launches past the target are idle.
    long long left = target - c->steps;
    int batch = (int)((left < check_every) ? left : check_every);
    if (batch < 1) batch = 1;
    for (int b = 0; b < batch; ++b) CK(cudaGraphLaunch(h->step_exec, h->stream));
    rc = read_ctrl(h);
    if (rc) return rc;
    rc = drain_log(h);
    if (rc) return rc;
  }
  fill_status(h, st);
  set_step_limit(h, 0x7fffffffffffffffLL);
  CK(cudaStreamSynchronize(h->stream));
  return h->ctrl_host->flags;
}

int mhd_gpu_step(mhd_gpu_t* h, mhd_gpu_status* st) { return mhd_gpu_advance(h, 1, 1, st); }

int mhd_gpu_step_graph_kernels(const mhd_gpu_t* h, int* n) {
  if (!h || !n) return MHD_ERR_INVALID;
  if (!h->step_exec) return MHD_ERR_STATE;
  *n = h->graph_kernels;
  return MHD_OK;
}

static_assert(sizeof(LogEntry) == sizeof(mhd_log_entry), "log record layouts differ");
static_assert(offsetof(LogEntry, total) == offsetof(mhd_log_entry, total), "log record layouts differ");

int mhd_gpu_set_log(mhd_gpu_t* h, int capacity, int diagnostics) {
  int rc = enter(h);
  if (rc) return rc;
  if (capacity < 0 || capacity > (1 << 24)) return MHD_ERR_INVALID;
  CK(cudaStreamSynchronize(h->stream));
  if (h->log_block) {
    CK(cudaFreeAsync(h->log_block, h->stream));
    h->log_block = nullptr;
  }
  h->log = nullptr;
  h->diag_part = nullptr;
  h->log_cap = 0;
  h->diag = 0;
  if (h->step_exec) {  // the step graph is re-captured with (or without) the log by the next advance
    cudaGraphExecDestroy(h->step_exec);
    h->step_exec = nullptr;
  }
  if (capacity == 0) {
    delete h->log_host;
    h->log_host = nullptr;
    return MHD_OK;
  }
  cudaMemPool_t pool;
  rc = device_pool(h->device, &pool);
  if (rc) return rc;
  const size_t ring = (sizeof(LogEntry) * (size_t)capacity + 255) / 256 * 256;
  const size_t part = sizeof(double) * DIAG_VALS * DIAG_MAX_BLOCKS + 256;  // partials, then the ticket
  CK(cudaMallocFromPoolAsync(&h->log_block, ring + part, pool, h->stream));
  CK(cudaMemsetAsync(h->log_block, 0, ring + part, h->stream));
  rc = read_ctrl(h);  // also orders the set-up before the caller's next use
  if (rc) return rc;
  h->log = static_cast<LogEntry*>(h->log_block);
  h->diag_part = reinterpret_cast<double*>(static_cast<char*>(h->log_block) + ring);
  h->log_cap = capacity;
  h->diag = diagnostics != 0;
  if (!h->log_host) h->log_host = new (std::nothrow) std::vector<LogEntry>();
  if (!h->log_host) return MHD_ERR_INVALID;
  h->log_host->clear();
  h->log_host_seq = h->ctrl_host->log_seq;  // records of the past are not in this ring
  h->log_dropped = 0;
  return MHD_OK;
}

int mhd_gpu_read_log(mhd_gpu_t* h, mhd_log_entry* out, int cap, int* n, long long* dropped) {
  int rc = enter(h);
  if (rc) return rc;
  if (!n || cap < 0 || (cap > 0 && !out)) return MHD_ERR_INVALID;
  if (!h->log) return MHD_ERR_STATE;
  rc = read_ctrl(h);
  if (rc) return rc;
  rc = drain_log(h);
  if (rc) return rc;
  std::vector<LogEntry>& v = *h->log_host;
  if (dropped) *dropped = h->log_dropped;
  if (!out) {  // count only
    *n = (int)std::min<size_t>(v.size(), 0x7fffffff);
    return MHD_OK;
  }
  const size_t k = std::min<size_t>(v.size(), (size_t)cap);
  std::memcpy(out, v.data(), sizeof(LogEntry) * k);
  v.erase(v.begin(), v.begin() + (long)k);
  *n = (int)k;
  return MHD_OK;
}

int mhd_gpu_state_device_ptr(mhd_gpu_t* h, int slot, double** dptr) {
  if (!h || !dptr || slot < 0 || slot > h->R) return MHD_ERR_INVALID;
  *dptr = h->u[slot];
  return MHD_OK;
}

}  // extern "C"

// =============================================================================================
// Allocation-free residual.  Its only scratch (the dt_lim reduction cell and the status words of
// the control block that the residual kernel writes) lives in this file-scope static device array;
// host code reaches it through the address cudaGetSymbolAddress returns for the current device.
// =============================================================================================
namespace {

constexpr size_t kNoAllocScratchBytes = 4096;
static_assert(sizeof(Ctrl) <= kNoAllocScratchBytes, "control block must fit the static scratch");
constexpr int kNoAllocMaxCells = 4096;  // per direction

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mutex;
void* g_noalloc_addr[kMaxDevices];  // device address of g_noalloc_scratch, per device

// Once per device, with that device current: tables + kernel attributes, then the symbol address.
int noalloc_setup(int dev, void** addr) {
  int rc = init_device_tables(dev);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(g_noalloc_mutex);
  if (!g_noalloc_addr[dev]) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) return MHD_ERR_CUDA;
    g_noalloc_addr[dev] = ptr;
  }
  *addr = g_noalloc_addr[dev];
  return MHD_OK;
}

}  // namespace

extern "C" int mhd_gpu_semidiscretize_noalloc(int p, int nx, int ny, double hx, double hy, double gamma,
                                              const double* u, double* ut, double* dt_lim, void* stream) {
  if (!u || !ut || !(hx > 0.0) || !(hy > 0.0) || !(gamma > 1.0) || nx < 2 || ny < 2) return MHD_ERR_INVALID;
  if (p < 1 || p > MAXP || nx > kNoAllocMaxCells || ny > kNoAllocMaxCells) return MHD_ERR_UNSUPPORTED;
  // the kernel moves tile rows with 16-byte loads and stores: both arrays must start on a 16-byte
  // boundary (a misaligned access would fault and lose the CUDA context), and ut must not overlap u
  // (tiles read neighbour traces of u while other tiles write ut)
  const uintptr_t ua = reinterpret_cast<uintptr_t>(u), ta = reinterpret_cast<uintptr_t>(ut);
  if ((ua | ta) & 15) return MHD_ERR_INVALID;
  const uintptr_t eb_bytes = sizeof(double) * 8 * (uintptr_t)(p + 1) * (p + 1);
  const uintptr_t u_end = ua + eb_bytes * (uintptr_t)(nx + 2) * (ny + 2), t_end = ta + eb_bytes * (uintptr_t)nx * ny;
  if (ua < t_end && ta < u_end) return MHD_ERR_INVALID;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return MHD_ERR_INVALID;
  void* addr = nullptr;
  int rc = noalloc_setup(dev, &addr);
  if (rc) return rc;
  Ctrl* ctrl = static_cast<Ctrl*>(addr);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the reduction cell must start "empty" (all ones: above every positive double's bit pattern)
  CK(cudaMemsetAsync(&ctrl->dt_lim_bits, 0xFF, sizeof(unsigned long long), s));
  Geo g;
  std::memset(&g, 0, sizeof(g));
  g.nx = nx;
  g.ny = ny;
  g.hx = hx;
  g.hy = hy;
  g.gamma = gamma;
  switch (p) {
    case 1: {
      using L = Res2Layout<1>;
      residual2_kernel<1><<<dim3((nx + L::TX - 1) / L::TX, (ny + L::TY - 1) / L::TY), L::NT, L::BYTES, s>>>(u, u, ut, g, ctrl, GATE_ALWAYS, StageCombine{});
      break;
    }
    case 2: {
      using L = Res2Layout<2>;
      residual2_kernel<2><<<dim3((nx + L::TX - 1) / L::TX, (ny + L::TY - 1) / L::TY), L::NT, L::BYTES, s>>>(u, u, ut, g, ctrl, GATE_ALWAYS, StageCombine{});
      break;
    }
    default: {
      using L = Res2Layout<3>;
      residual2_kernel<3><<<dim3((nx + L::TX - 1) / L::TX, (ny + L::TY - 1) / L::TY), L::NT, L::BYTES, s>>>(u, u, ut, g, ctrl, GATE_ALWAYS, StageCombine{});
      break;
    }
  }
  CK(cudaGetLastError());
  if (dt_lim) {
    unsigned long long bits = 0;
    CK(cudaMemcpyAsync(&bits, &ctrl->dt_lim_bits, sizeof(bits), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    double d;
    std::memcpy(&d, &bits, sizeof(d));
    *dt_lim = d;
  }
  return MHD_OK;
}

#include "batch_impl.cuh"
#include "server_impl.cuh"
