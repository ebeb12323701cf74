// batch_impl.cuh -- many independent solver instances advanced together (included by mhd_gpu.cu).
//
// A batch holds existing handles (each already through mhd_gpu_solve_begin).  Members are grouped
// by (degree p, RK stages R).  Per group the batch keeps a device table of InstDesc entries and one
// flattened work list per kernel kind: residual tiles, average/LDF chunks, OEDG indicator item
// blocks, limiter row segments, combination blocks and ghost blocks, each entry (instance, a, b).
// One SSP-RK try of every member is one CUDA graph: per group the batched kernels of the try
// sequence (the same kernel bodies as the single-instance path, so each member's arithmetic is
// identical alone and in the batch), groups on parallel branches.  The kernels are persistent
// grids that read the list lengths from device memory, so membership changes only rewrite the
// tables; the graph is re-captured only when a table outgrows its buffer.
#pragma once
#include <algorithm>
#include <vector>

namespace {

enum WorkKind { WK_RES = 0, WK_AVG, WK_SIG, WK_LIM, WK_CMB, WK_BC, WK_COUNT };

// One group's device table, one allocation, uploaded with one copy:
//   InstDesc insts[cap] | int total[WK_COUNT] | int ninst | int pref[WK_COUNT][cap + 1]
constexpr int kIdleRounds = 64;  // rounds an empty group is kept in the graph
constexpr int kMinCap = 16;      // members a group's table holds before it first grows

struct BatchGroup {
  int p = 0, R = 0;
  int idle_rounds = 0;  // rounds launched since the group last had a member
  std::vector<mhd_gpu*> members;
  char* d_table = nullptr;
  int cap = 0;
  size_t table_bytes(int c) const { return sizeof(InstDesc) * c + sizeof(int) * (WK_COUNT + 1 + WK_COUNT * (c + 1)); }
  InstDesc* insts() const { return reinterpret_cast<InstDesc*>(d_table); }
  int* total() const { return reinterpret_cast<int*>(d_table + sizeof(InstDesc) * cap); }
  int* ninst() const { return total() + WK_COUNT; }
  int* pref(int k) const { return total() + WK_COUNT + 1 + k * (cap + 1); }
};

int sm_count(int dev) {
  int n = 0;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 148;
}

}  // namespace

struct mhd_batch {
  int device = 0;
  int nsm = 0;
  cudaStream_t stream = nullptr;
  std::vector<BatchGroup> groups;
  std::vector<mhd_gpu*> members;  // in insertion order
  cudaGraphExec_t exec = nullptr;
  bool graph_stale = true;
  bool dirty = true;              // membership changed since the tables were uploaded
  Ctrl* d_status = nullptr;       // gathered control blocks, one per member (group order)
  Ctrl* h_status = nullptr;
  int cap_status = 0;
  char* h_stage = nullptr;        // pinned staging of the table uploads
  size_t cap_stage = 0;
  std::vector<cudaStream_t> branch;
  std::vector<cudaEvent_t> ev;
  cudaEvent_t join_ev = nullptr;  // orders a joining member's queued work before the next round
  bool in_flight = false;         // a round was launched and not yet waited for
  long long captures = 0;         // graph (re)captures so far
};

namespace {

InstDesc make_desc(const mhd_gpu* h) {
  InstDesc d;
  std::memset(&d, 0, sizeof(d));
  d.g = h->geo;
  for (int s = 0; s < 6; ++s) {
    d.u[s] = h->u[s];
    d.ut[s] = h->ut[s];
  }
  d.u_avg = h->u_avg;
  d.log = h->log;
  d.log_cap = h->log_cap;
  d.sig_x = h->sig_x;
  d.sig_y = h->sig_y;
  d.partial = h->partial;
  d.ent_partial = h->ent_partial;
  d.cell_ent_DG = h->cell_ent_DG;
  d.cell_ent_FV = h->cell_ent_FV;
  d.cell_ent_nan = h->cell_ent_nan;
  d.ctrl = h->ctrl;
  d.use_oedg = h->use_oedg;
  d.use_ldf = h->use_ldf;
  d.ent_offset = h->ent_offset;
  d.R = h->R;
  return d;
}

// items of each kind one member contributes (the same decomposition as its single-instance launches)
template <int P>
void member_work(const mhd_gpu* h, long long* cnt, InstDesc& d) {
  using RL = Res2Layout<P>;
  constexpr int EB = 8 * (P + 1) * (P + 1), TE = PPCfg<P>::TE;
  const long long nx = h->nx, ny = h->ny;
  cnt[WK_RES] = ((nx + RL::TX - 1) / RL::TX) * ((ny + RL::TY - 1) / RL::TY);
  const long long nelg = (nx + 2) * (ny + 2);
  d.nblk_avg = (int)((nelg + TE - 1) / TE);
  cnt[WK_AVG] = d.nblk_avg;
  cnt[WK_SIG] = ((nx + SigCfg<P>::TX - 1) / SigCfg<P>::TX) * ((ny + SigCfg<P>::TY - 1) / SigCfg<P>::TY);
  constexpr int TEL = PPCfg<P>::TEL;  // the limiter's row segments
  d.nseg_limit = (int)(((nx + TEL - 1) / TEL) * ny);
  cnt[WK_LIM] = d.nseg_limit;
  cnt[WK_CMB] = (nx * ny * EB + 255) / 256;
  cnt[WK_BC] = (2 * (nx + ny) * EB + 255) / 256;
}

// upload every group's table (one copy per group from pinned staging); grows buffers as needed
int refresh_batch(mhd_batch* b) {
  // an empty group stays in the graph (its launches find no work) until it has idled kIdleRounds
  // rounds, so that runs of one degree coming and going do not re-capture the graph each time
  for (auto& g : b->groups)
    if (g.members.empty() && g.idle_rounds > kIdleRounds) {
      if (g.d_table) cudaFree(g.d_table);
      g.d_table = nullptr;
      b->graph_stale = true;
    }
  b->groups.erase(std::remove_if(b->groups.begin(), b->groups.end(),
                                 [](const BatchGroup& g) { return !g.d_table && g.members.empty() && g.idle_rounds > kIdleRounds; }),
                  b->groups.end());
  size_t stage_need = 0;
  for (auto& g : b->groups) {
    const int n = (int)g.members.size();
    if (n) g.idle_rounds = 0;
    if (n > g.cap || !g.d_table) {
      if (g.d_table) cudaFree(g.d_table);
      g.cap = std::max(std::max(n, kMinCap), 2 * g.cap);
      CK(cudaMalloc((void**)&g.d_table, g.table_bytes(g.cap)));
      b->graph_stale = true;
    }
    stage_need += g.table_bytes(g.cap);
  }
  if (stage_need > b->cap_stage) {
    if (b->h_stage) cudaFreeHost(b->h_stage);
    b->cap_stage = stage_need * 2;
    CK(cudaMallocHost((void**)&b->h_stage, b->cap_stage));
  }
  size_t off = 0;
  for (auto& g : b->groups) {
    const int n = (int)g.members.size();
    char* hs = b->h_stage + off;
    InstDesc* hi = reinterpret_cast<InstDesc*>(hs);
    int* htot = reinterpret_cast<int*>(hs + sizeof(InstDesc) * g.cap);
    int* hpref = htot + WK_COUNT + 1;
    long long run[WK_COUNT] = {0, 0, 0, 0, 0, 0};
    for (int k = 0; k < WK_COUNT; ++k) hpref[k * (g.cap + 1)] = 0;
    for (int m = 0; m < n; ++m) {
      InstDesc d = make_desc(g.members[m]);
      long long cnt[WK_COUNT];
      switch (g.p) {
        case 1: member_work<1>(g.members[m], cnt, d); break;
        case 2: member_work<2>(g.members[m], cnt, d); break;
        default: member_work<3>(g.members[m], cnt, d); break;
      }
      hi[m] = d;
      for (int k = 0; k < WK_COUNT; ++k) {
        run[k] += cnt[k];
        if (run[k] > 0x7fffffffLL) return MHD_ERR_UNSUPPORTED;
        hpref[k * (g.cap + 1) + m + 1] = (int)run[k];
      }
    }
    for (int k = 0; k < WK_COUNT; ++k) htot[k] = (int)run[k];
    htot[WK_COUNT] = n;
    CK(cudaMemcpyAsync(g.d_table, hs, g.table_bytes(g.cap), cudaMemcpyHostToDevice, b->stream));
    off += g.table_bytes(g.cap);
  }
  const int n = (int)b->members.size();
  if (n > b->cap_status) {
    if (b->d_status) cudaFree(b->d_status);
    if (b->h_status) cudaFreeHost(b->h_status);
    b->cap_status = std::max(n, 2 * b->cap_status);
    CK(cudaMalloc((void**)&b->d_status, sizeof(Ctrl) * b->cap_status));
    CK(cudaMallocHost((void**)&b->h_status, sizeof(Ctrl) * b->cap_status));
  }
  b->dirty = false;
  return MHD_OK;
}

// persistent grid: every CTA the SMs can hold at once for this kernel
template <class K>
int full_grid(K kernel, int threads, size_t smem, int nsm) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  return per_sm * nsm;
}

struct BatchGrids {
  int res, cmb, bc, avg, avg_final, sig, lim, seb;
};

// queried before a capture begins (the occupancy calculator is host-only work)
template <int P>
BatchGrids batch_grids(int nsm) {
  constexpr int EB = 8 * (P + 1) * (P + 1);
  BatchGrids gr;
  gr.res = full_grid(residual2_batched<P>, Res2Layout<P>::NT, Res2Layout<P>::BYTES, nsm);
  gr.cmb = full_grid(combine_batched<EB>, 256, 0, nsm);
  gr.bc = full_grid(bc_batched<P>, 256, 0, nsm);
  gr.avg = full_grid(pp_avg_ldf_batched<P, false>, PPCfg<P>::NT, 0, nsm);
  gr.avg_final = full_grid(pp_avg_ldf_batched<P, true>, PPCfg<P>::NT, 0, nsm);
  gr.sig = full_grid(pp_sigsum_batched<P>, 256, 0, nsm);
  gr.lim = full_grid(pp_limit_batched<P>, PPCfg<P>::NT, 0, nsm);
  gr.seb = full_grid(stage_end_bc_batched<P>, 256, 0, nsm);
  return gr;
}

template <int P>
void enqueue_group_try(mhd_batch* b, BatchGroup& g, const BatchGrids& gr, cudaStream_t st) {
  constexpr int EB = 8 * (P + 1) * (P + 1);
  const int R = g.R;
  const int* tot = g.total();
  const int* ninst = g.ninst();
  InstDesc* in = g.insts();
  const size_t smem = Res2Layout<P>::BYTES;
  constexpr int NT_RES = Res2Layout<P>::NT;
  const int grid_res = gr.res, grid_cmb = gr.cmb, grid_bc = gr.bc, grid_avg = gr.avg, grid_sig = gr.sig,
            grid_lim = gr.lim;
  ctl_batched<<<1, 256, 0, st>>>(in, ninst, CTL_STEP_BEGIN, R, 0);
  residual2_batched<P><<<grid_res, NT_RES, smem, st>>>(in, g.pref(WK_RES), tot + WK_RES, ninst, 0, 1, ST_RECOMPUTE,
                                                        0, 0.0, 0.0);
  ctl_batched<<<1, 256, 0, st>>>(in, ninst, CTL_DT_STAGE1, R, 1);  // dt, and the pseudo-time of stage 1
  for (int s = 1; s <= R; ++s) {
    const int fin = (s == R);
    // stage 1: loop 1 forms the stage state and its ghost ring; SSP-RK(2,2)/(3,3): later stages
    // come from the previous residual
    if (s > 1 && R > 3)
      combine_batched<EB><<<grid_cmb, 256, 0, st>>>(in, g.pref(WK_CMB), tot + WK_CMB, ninst, s, ST_RUN);
    if (s > 1) bc_batched<P><<<grid_bc, 256, 0, st>>>(in, g.pref(WK_BC), tot + WK_BC, ninst, s, ST_RUN);
    if (fin)
      pp_avg_ldf_batched<P, true><<<gr.avg_final, PPCfg<P>::NT, 0, st>>>(in, g.pref(WK_AVG), tot + WK_AVG, ninst, s, ST_RUN,
                                                                  s == 1);
    else
      pp_avg_ldf_batched<P, false><<<grid_avg, PPCfg<P>::NT, 0, st>>>(in, g.pref(WK_AVG), tot + WK_AVG, ninst, s, ST_RUN,
                                                                s == 1);
    if (fin) {
      pp_reduce_batched<<<b->nsm, 256, 0, st>>>(in, ninst, fin, ST_RUN);
      pp_sigsum_batched<P><<<grid_sig, 256, 0, st>>>(in, g.pref(WK_SIG), tot + WK_SIG, ninst, s, fin, ST_RUN);
    }
    if (fin) pp_limit_batched<P><<<grid_lim, PPCfg<P>::NT, 0, st>>>(in, g.pref(WK_LIM), tot + WK_LIM, ninst, s, fin, ST_RUN);
    // entropy sum (final stage), stage-end decision, next stage's pseudo-time and the ghost rings
    stage_end_bc_batched<P><<<gr.seb, 256, 0, st>>>(in, g.pref(WK_BC), tot + WK_BC, ninst, s, R, fin ? 0 : s + 1,
                                                     fin);
    // the coefficients of combine_value for SSP-RK(2,2) stage 2 and SSP-RK(3,3) stages 2, 3
    const int nxt = (!fin && (R == 2 || R == 3)) ? s + 1 : 0;
    const double ca = nxt == 0 ? 0.0 : (R == 2 ? 0.5 : (nxt == 2 ? 0.75 : 1.0 / 3.0));
    const double cb = nxt == 0 ? 0.0 : (R == 2 ? 0.5 : (nxt == 2 ? 0.25 : 2.0 / 3.0));
    residual2_batched<P><<<grid_res, NT_RES, smem, st>>>(in, g.pref(WK_RES), tot + WK_RES, ninst, s, (s % R) + 1,
                                                          ST_RUN, nxt, ca, cb);
  }
  ctl_batched<<<1, 256, 0, st>>>(in, ninst, CTL_STEP_END, R, 0);
}

int capture_batch_graph(mhd_batch* b) {
  while (b->branch.size() < b->groups.size()) {
    cudaStream_t s;
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    b->branch.push_back(s);
  }
  while (b->ev.size() < b->groups.size() + 1) {
    cudaEvent_t e;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->ev.push_back(e);
  }
  const BatchGrids grids[3] = {batch_grids<1>(b->nsm), batch_grids<2>(b->nsm), batch_grids<3>(b->nsm)};
  cudaGraph_t graph = nullptr;
  CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  // every call below is recorded, not run; an error invalidates the capture, which still ends
  cudaEventRecord(b->ev[0], b->stream);
  for (size_t gi = 0; gi < b->groups.size(); ++gi) {
    cudaStream_t st = b->branch[gi];
    cudaStreamWaitEvent(st, b->ev[0], 0);
    BatchGroup& g = b->groups[gi];
    switch (g.p) {
      case 1: enqueue_group_try<1>(b, g, grids[0], st); break;
      case 2: enqueue_group_try<2>(b, g, grids[1], st); break;
      default: enqueue_group_try<3>(b, g, grids[2], st); break;
    }
    cudaEventRecord(b->ev[gi + 1], st);
    cudaStreamWaitEvent(b->stream, b->ev[gi + 1], 0);
  }
  cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
  if (e != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return MHD_ERR_CUDA;
  }
  if (b->exec) {  // same groups, new tables: update the executable graph in place
    cudaGraphExecUpdateResultInfo info;
    if (cudaGraphExecUpdate(b->exec, graph, &info) != cudaSuccess) {
      cudaGetLastError();
      cudaGraphExecDestroy(b->exec);
      b->exec = nullptr;
    }
  }
  e = b->exec ? cudaSuccess : cudaGraphInstantiate(&b->exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return MHD_ERR_CUDA;
  b->graph_stale = false;
  return MHD_OK;
}

// copy every member's control block to the pinned host mirror (asynchronous)
int enqueue_gather(mhd_batch* b) {
  int off = 0;
  for (auto& g : b->groups) {
    const int n = (int)g.members.size();
    if (!n) continue;
    ctl_gather_batched<<<(n + 255) / 256, 256, 0, b->stream>>>(g.insts(), g.ninst(), b->d_status + off);
    off += n;
  }
  CK(cudaGetLastError());
  if (off) CK(cudaMemcpyAsync(b->h_status, b->d_status, sizeof(Ctrl) * off, cudaMemcpyDeviceToHost, b->stream));
  return MHD_OK;
}

// after the stream is idle: hand each member its control block
void unpack_gather(mhd_batch* b) {
  int off = 0;
  for (auto& g : b->groups)
    for (mhd_gpu* h : g.members) *h->ctrl_host = b->h_status[off++];
}

int batch_launch(mhd_batch* b, int tries) {
  if (b->in_flight) return MHD_ERR_STATE;
  CK(cudaSetDevice(b->device));
  if (b->dirty) {
    int rc = refresh_batch(b);
    if (rc) return rc;
  }
  if (!b->members.empty()) {
    if (b->graph_stale) {
      int rc = capture_batch_graph(b);
      if (rc) return rc;
      ++b->captures;
    }
    for (int t = 0; t < tries; ++t) CK(cudaGraphLaunch(b->exec, b->stream));
    for (auto& g : b->groups)
      if (g.members.empty() && ++g.idle_rounds > kIdleRounds) b->dirty = true;  // dropped at the next refresh
  }
  int rc = enqueue_gather(b);
  if (rc) return rc;
  b->in_flight = true;
  return MHD_OK;
}

int batch_wait(mhd_batch* b, int* n_active) {
  if (!b->in_flight) return MHD_ERR_STATE;
  CK(cudaSetDevice(b->device));
  b->in_flight = false;
  CK(cudaStreamSynchronize(b->stream));
  unpack_gather(b);
  if (n_active) {
    int a = 0;
    for (mhd_gpu* h : b->members)
      if (!h->ctrl_host->done && !(h->ctrl_host->flags & FLAGS_FATAL)) ++a;
    *n_active = a;
  }
  return MHD_OK;
}

}  // namespace

extern "C" {

int mhd_batch_create(mhd_batch_t** out) {
  if (!out) return MHD_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MHD_ERR_NO_DEVICE;
  mhd_batch* b = new (std::nothrow) mhd_batch;
  if (!b) return MHD_ERR_INVALID;
  if (cudaGetDevice(&b->device) != cudaSuccess || init_device_tables(b->device) ||
      cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->join_ev, cudaEventDisableTiming) != cudaSuccess) {
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return MHD_ERR_CUDA;
  }
  b->nsm = sm_count(b->device);
  *out = b;
  return MHD_OK;
}

int mhd_batch_destroy(mhd_batch_t* b) {
  if (!b) return MHD_ERR_INVALID;
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->stream);
  b->in_flight = false;
  for (mhd_gpu* h : b->members) h->stream = h->own_stream;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  for (auto& g : b->groups)
    if (g.d_table) cudaFree(g.d_table);
  if (b->d_status) cudaFree(b->d_status);
  if (b->h_stage) cudaFreeHost(b->h_stage);
  if (b->h_status) cudaFreeHost(b->h_status);
  for (auto s : b->branch) cudaStreamDestroy(s);
  for (auto e : b->ev) cudaEventDestroy(e);
  if (b->join_ev) cudaEventDestroy(b->join_ev);
  cudaStreamDestroy(b->stream);
  delete b;
  return MHD_OK;
}

int mhd_batch_add(mhd_batch_t* b, mhd_gpu_t* h) {
  if (!b || !h) return MHD_ERR_INVALID;
  if (h->device != b->device) return MHD_ERR_INVALID;
  if (!h->solve_ready || b->in_flight) return MHD_ERR_STATE;
  if (std::find(b->members.begin(), b->members.end(), h) != b->members.end()) return MHD_ERR_STATE;
  CK(cudaSetDevice(b->device));
  // the batch stream waits (on the device) for the member's queued work
  CK(cudaEventRecord(b->join_ev, h->stream));
  CK(cudaStreamWaitEvent(b->stream, b->join_ev, 0));
  h->stream = b->stream;  // the batch drives the member from now on
  b->members.push_back(h);
  BatchGroup* grp = nullptr;
  for (auto& g : b->groups)
    if (g.p == h->p && g.R == h->R) grp = &g;
  if (!grp) {
    b->groups.emplace_back();
    grp = &b->groups.back();
    grp->p = h->p;
    grp->R = h->R;
    b->graph_stale = true;
  }
  grp->members.push_back(h);
  b->dirty = true;  // tables are uploaded once, at the next advance
  return MHD_OK;
}

int mhd_batch_remove(mhd_batch_t* b, mhd_gpu_t* h) {
  if (!b || !h) return MHD_ERR_INVALID;
  if (b->in_flight) return MHD_ERR_STATE;
  auto it = std::find(b->members.begin(), b->members.end(), h);
  if (it == b->members.end()) return MHD_ERR_STATE;
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  b->members.erase(it);
  for (auto& g : b->groups) g.members.erase(std::remove(g.members.begin(), g.members.end(), h), g.members.end());
  h->stream = h->own_stream;
  b->dirty = true;
  return MHD_OK;
}

int mhd_batch_size(const mhd_batch_t* b, int* n) {
  if (!b || !n) return MHD_ERR_INVALID;
  *n = (int)b->members.size();
  return MHD_OK;
}

int mhd_batch_advance(mhd_batch_t* b, int tries, int* n_active) {
  if (!b || tries < 0) return MHD_ERR_INVALID;
  int rc = batch_launch(b, tries);
  if (rc) return rc;
  return batch_wait(b, n_active);
}

int mhd_batch_launch(mhd_batch_t* b, int tries) {
  if (!b || tries < 0) return MHD_ERR_INVALID;
  return batch_launch(b, tries);
}

int mhd_batch_wait(mhd_batch_t* b, int* n_active) {
  if (!b) return MHD_ERR_INVALID;
  return batch_wait(b, n_active);
}

int mhd_batch_member_status(mhd_batch_t* b, mhd_gpu_t* h, mhd_gpu_status* st) {
  if (!b || !h || !st) return MHD_ERR_INVALID;
  if (std::find(b->members.begin(), b->members.end(), h) == b->members.end()) return MHD_ERR_STATE;
  fill_status(h, st);  // as of the last completed round
  return h->ctrl_host->flags;
}

}  // extern "C"
