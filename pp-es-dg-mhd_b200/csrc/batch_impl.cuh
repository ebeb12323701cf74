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
struct BatchGroup {
  int p = 0, R = 0;
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
  int device;
  int nsm;
  cudaStream_t stream;
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
  using RL = ResLayout<P>;
  constexpr int EB = 8 * (P + 1) * (P + 1), TE = PPCfg<P>::TE;
  const long long nx = h->nx, ny = h->ny;
  cnt[WK_RES] = ((nx + RL::TX - 1) / RL::TX) * ((ny + RL::TY - 1) / RL::TY);
  const long long nelg = (nx + 2) * (ny + 2);
  d.nblk_avg = (int)((nelg + TE - 1) / TE);
  cnt[WK_AVG] = d.nblk_avg;
  cnt[WK_SIG] = (((nx + 1) * ny + nx * (ny + 1)) * 8 + 255) / 256;
  d.nseg_limit = (int)(((nx + TE - 1) / TE) * ny);
  cnt[WK_LIM] = d.nseg_limit;
  cnt[WK_CMB] = (nx * ny * EB + 255) / 256;
  cnt[WK_BC] = (2 * (nx + ny) * EB + 255) / 256;
}

// upload every group's table (one copy per group from pinned staging); grows buffers as needed
int refresh_batch(mhd_batch* b) {
  for (auto& g : b->groups)
    if (g.members.empty()) {
      if (g.d_table) cudaFree(g.d_table);
      g.d_table = nullptr;
      b->graph_stale = true;
    }
  b->groups.erase(std::remove_if(b->groups.begin(), b->groups.end(),
                                 [](const BatchGroup& g) { return g.members.empty(); }),
                  b->groups.end());
  size_t stage_need = 0;
  for (auto& g : b->groups) {
    const int n = (int)g.members.size();
    if (n > g.cap || !g.d_table) {
      if (g.d_table) cudaFree(g.d_table);
      g.cap = std::max(n, 2 * g.cap);
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

template <int P>
void enqueue_group_try(mhd_batch* b, BatchGroup& g, cudaStream_t st) {
  constexpr int EB = 8 * (P + 1) * (P + 1);
  const int R = g.R;
  const int* tot = g.total();
  const int* ninst = g.ninst();
  InstDesc* in = g.insts();
  const int grid_res = b->nsm * ResCfg<P>::MINB;
  const int grid_pp = b->nsm * 4;
  const size_t smem = ResLayout<P>::BYTES;
  ctl_batched<<<1, 256, 0, st>>>(in, ninst, CTL_STEP_BEGIN, R, 0);
  residual_batched<P><<<grid_res, ResCfg<P>::NT, smem, st>>>(in, g.pref(WK_RES), tot + WK_RES, ninst, 0, 1, ST_RECOMPUTE);
  ctl_batched<<<1, 256, 0, st>>>(in, ninst, CTL_DT, R, 0);
  for (int s = 1; s <= R; ++s) {
    const int fin = (s == R);
    ctl_batched<<<1, 256, 0, st>>>(in, ninst, CTL_STAGE_TIME, R, s);
    combine_batched<EB><<<grid_pp, 256, 0, st>>>(in, g.pref(WK_CMB), tot + WK_CMB, ninst, s, ST_RUN);
    bc_batched<P><<<grid_pp, 256, 0, st>>>(in, g.pref(WK_BC), tot + WK_BC, ninst, s, ST_RUN);
    pp_avg_ldf_batched<P><<<grid_pp, PP_NT, 0, st>>>(in, g.pref(WK_AVG), tot + WK_AVG, ninst, s, fin, ST_RUN);
    if (fin) {
      pp_reduce_batched<<<b->nsm, 256, 0, st>>>(in, ninst, fin, ST_RUN);
      pp_sigsum_batched<P><<<grid_pp, 256, 0, st>>>(in, g.pref(WK_SIG), tot + WK_SIG, ninst, s, fin, ST_RUN);
    }
    pp_limit_batched<P><<<grid_pp, PP_NT, 0, st>>>(in, g.pref(WK_LIM), tot + WK_LIM, ninst, s, fin, ST_RUN);
    if (fin) pp_entsum_batched<<<b->nsm, 256, 0, st>>>(in, ninst, ST_RUN);
    ctl_batched<<<1, 256, 0, st>>>(in, ninst, CTL_STAGE_END, R, s);
    bc_batched<P><<<grid_pp, 256, 0, st>>>(in, g.pref(WK_BC), tot + WK_BC, ninst, s, ST_RUN);
    residual_batched<P><<<grid_res, ResCfg<P>::NT, smem, st>>>(in, g.pref(WK_RES), tot + WK_RES, ninst, s, (s % R) + 1, ST_RUN);
  }
  ctl_batched<<<1, 256, 0, st>>>(in, ninst, CTL_STEP_END, R, 0);
}

int capture_batch_graph(mhd_batch* b) {
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
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
  cudaGraph_t graph;
  CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  CK(cudaEventRecord(b->ev[0], b->stream));
  for (size_t gi = 0; gi < b->groups.size(); ++gi) {
    cudaStream_t st = b->branch[gi];
    CK(cudaStreamWaitEvent(st, b->ev[0], 0));
    BatchGroup& g = b->groups[gi];
    switch (g.p) {
      case 1: enqueue_group_try<1>(b, g, st); break;
      case 2: enqueue_group_try<2>(b, g, st); break;
      default: enqueue_group_try<3>(b, g, st); break;
    }
    CK(cudaEventRecord(b->ev[gi + 1], st));
    CK(cudaStreamWaitEvent(b->stream, b->ev[gi + 1], 0));
  }
  cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
  if (e != cudaSuccess) return MHD_ERR_CUDA;
  e = cudaGraphInstantiate(&b->exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return MHD_ERR_CUDA;
  b->graph_stale = false;
  return MHD_OK;
}

// copy every member's control block into the members' host mirrors
int gather_status(mhd_batch* b) {
  int off = 0;
  for (auto& g : b->groups) {
    const int n = (int)g.members.size();
    if (!n) continue;
    ctl_gather_batched<<<(n + 255) / 256, 256, 0, b->stream>>>(g.insts(), g.ninst(), b->d_status + off);
    off += n;
  }
  CK(cudaGetLastError());
  if (off) CK(cudaMemcpyAsync(b->h_status, b->d_status, sizeof(Ctrl) * off, cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  off = 0;
  for (auto& g : b->groups)
    for (mhd_gpu* h : g.members) *h->ctrl_host = b->h_status[off++];
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
      cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
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
  for (mhd_gpu* h : b->members) h->stream = h->own_stream;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  for (auto& g : b->groups)
    if (g.d_table) cudaFree(g.d_table);
  if (b->d_status) cudaFree(b->d_status);
  if (b->h_stage) cudaFreeHost(b->h_stage);
  if (b->h_status) cudaFreeHost(b->h_status);
  for (auto s : b->branch) cudaStreamDestroy(s);
  for (auto e : b->ev) cudaEventDestroy(e);
  cudaStreamDestroy(b->stream);
  delete b;
  return MHD_OK;
}

int mhd_batch_add(mhd_batch_t* b, mhd_gpu_t* h) {
  if (!b || !h) return MHD_ERR_INVALID;
  if (h->device != b->device) return MHD_ERR_INVALID;
  if (!h->solve_ready) return MHD_ERR_STATE;
  if (std::find(b->members.begin(), b->members.end(), h) != b->members.end()) return MHD_ERR_STATE;
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(h->stream));
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
  CK(cudaSetDevice(b->device));
  if (b->dirty) {
    int rc = refresh_batch(b);
    if (rc) return rc;
  }
  if (!b->members.empty()) {
    if (b->graph_stale) {
      int rc = capture_batch_graph(b);
      if (rc) return rc;
    }
    for (int t = 0; t < tries; ++t) CK(cudaGraphLaunch(b->exec, b->stream));
  }
  int rc = gather_status(b);
  if (rc) return rc;
  if (n_active) {
    int a = 0;
    for (mhd_gpu* h : b->members)
      if (!h->ctrl_host->done && !(h->ctrl_host->flags & 0x6)) ++a;
    *n_active = a;
  }
  return MHD_OK;
}

int mhd_batch_member_status(mhd_batch_t* b, mhd_gpu_t* h, mhd_gpu_status* st) {
  if (!b || !h || !st) return MHD_ERR_INVALID;
  if (std::find(b->members.begin(), b->members.end(), h) == b->members.end()) return MHD_ERR_STATE;
  fill_status(h, st);  // as of the last mhd_batch_advance
  return h->ctrl_host->flags;
}

}  // extern "C"
