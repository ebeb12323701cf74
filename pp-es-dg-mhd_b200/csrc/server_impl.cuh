// server_impl.cuh -- continuous-batching request loop (included by mhd_gpu.cu).
//
// Runs (one solve_execute each) are submitted with an arrival time on the server clock.  One
// round of the loop:
//   1. queue a batched round (tries_per_round tries of every active run) and return at once;
//   2. while it runs, admit every run whose arrival time has passed while the HBM budget and the
//      active-run cap allow (create the instance, upload its initial state, solve_begin);
//   3. wait for the round, retire finished runs (download u_avg if asked, free their memory);
//   4. join the runs admitted in step 2 to the batch for the next round.
// With batched = 0 it serves the same queue one plain run at a time (mhd_gpu_advance to the end),
// the comparison point for the batched form.
#pragma once
#include <chrono>
#include <deque>
#include <map>
#include <thread>

// The server's device memory: one allocation of the whole HBM budget, made when the server is
// created and carved into instance blocks by a best-fit allocator over free ranges (coalesced when
// a block comes back).  Admissions then make no CUDA allocation call: allocating from a memory pool
// while a batched round is in flight can make the host wait for the round.
struct Arena {
  static constexpr size_t kAlign = 64 << 10;
  char* base = nullptr;
  size_t size = 0;
  std::map<size_t, size_t> free_ranges;  // offset -> length

  static size_t round_up(size_t b) { return (b + kAlign - 1) / kAlign * kAlign; }
  void reset(char* b, size_t n) {
    base = b;
    size = n / kAlign * kAlign;
    free_ranges.clear();
    if (size) free_ranges[0] = size;
  }
  bool take(size_t bytes, size_t* off) {
    const size_t need = round_up(bytes);
    auto best = free_ranges.end();
    for (auto it = free_ranges.begin(); it != free_ranges.end(); ++it)
      if (it->second >= need && (best == free_ranges.end() || it->second < best->second)) best = it;
    if (best == free_ranges.end()) return false;
    *off = best->first;
    const size_t left = best->second - need;
    const size_t at = best->first + need;
    free_ranges.erase(best);
    if (left) free_ranges[at] = left;
    return true;
  }
  void give(size_t off, size_t bytes) {
    size_t len = round_up(bytes);
    auto next = free_ranges.lower_bound(off);
    if (next != free_ranges.end() && off + len == next->first) {  // merge with the range after
      len += next->second;
      next = free_ranges.erase(next);
    }
    if (next != free_ranges.begin()) {  // and with the range before
      auto prev = std::prev(next);
      if (prev->first + prev->second == off) {
        prev->second += len;
        return;
      }
    }
    free_ranges[off] = len;
  }
};

struct mhd_server {
  int device;
  size_t budget;
  int max_active;
  int tries_per_round;
  int batched;
  size_t used = 0;
  mhd_batch* batch = nullptr;
  Arena arena;
  std::vector<mhd_request> pending;  // sorted by arrival when run starts
  size_t next_pending = 0;
  struct Active {
    mhd_request req;
    mhd_gpu* h;
    size_t bytes;   // footprint
    size_t off;     // its block's offset in the arena
    double admitted;
    bool in_batch;
  };
  std::vector<Active> active;
  std::vector<mhd_request_result> results;
  mhd_server_stats stats{};
  std::chrono::steady_clock::time_point origin;
  bool started = false;
};

namespace {

double server_now(const mhd_server* s) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - s->origin).count();
}

// device bytes mhd_gpu_create allocates for one instance (its one block)
size_t instance_bytes(int nx, int ny, int p, int R) { return inst_layout(nx, ny, p, R).total; }

// mhd_gpu_solve_begin with no host round trip: the same launches, queued on the instance's own
// stream, and the starting control block assembled on the device (ctl_solve_begin).  The host
// mirror holds a provisional status until the first batched round refreshes it; an inadmissible
// initial value shows up there as MHD_FLAG_INIT_NEG_AVG.
int solve_begin_async(mhd_gpu* h, double final_T, double cfl, int use_oedg, int use_ldf, int ent_offset) {
  DISPATCH_P(h, launch_bc, h, h->u[0], GATE_ALWAYS);  // drive.f90:67-73
  ctl_pp_reset<<<1, 1, 0, h->stream>>>(h->ctrl, GATE_ALWAYS);
  DISPATCH_P(h, launch_post, h, 0, false, use_ldf != 0, nullptr, 0.0, false, true, nullptr, GATE_ALWAYS);
  DISPATCH_P(h, launch_bc, h, h->u[0], GATE_ALWAYS);
  CK(cudaMemsetAsync(&h->ctrl->dt_lim_bits, 0xFF, sizeof(unsigned long long), h->stream));
  DISPATCH_P(h, launch_residual, h, h->u[0], h->ut[1], GATE_ALWAYS);
  const double cfl_total = ((h->R <= 3) ? 1.0 : 1.508) * cfl;  // CFL_RK * CFL (drive.f90:57-63,109)
  ctl_solve_begin<<<1, 1, 0, h->stream>>>(h->ctrl, final_T, cfl_total);
  CK(cudaGetLastError());
  h->final_T = final_T;
  h->cfl = cfl;
  h->use_oedg = use_oedg != 0;
  h->use_ldf = use_ldf != 0;
  h->ent_offset = ent_offset != 0;
  std::memset(h->ctrl_host, 0, sizeof(Ctrl));
  h->ctrl_host->final_T = final_T;
  h->ctrl_host->cfl_total = cfl_total;
  h->ctrl_host->step_limit = 0x7fffffffffffffffLL;
  if (h->step_exec) {
    cudaGraphExecDestroy(h->step_exec);
    h->step_exec = nullptr;
  }
  h->solve_ready = 1;
  return MHD_OK;
}

// destroy an instance and give its block back to the arena
void release_instance(mhd_server* s, mhd_gpu* h, size_t off, size_t bytes) {
  mhd_gpu_destroy(h);  // waits for the instance's stream: nothing is left in flight on the block
  s->arena.give(off, bytes);
}

// 1 = admitted (or finished at once), 0 = no room in the arena yet, < 0 = error
int admit(mhd_server* s, const mhd_request& r, double now) {
  mhd_gpu* h = nullptr;
  const size_t need = instance_bytes(r.nx, r.ny, r.p, r.rknstg);
  size_t off = 0;
  if (!s->arena.take(need, &off)) return 0;
  // batched: nothing here waits for the device, so the round in flight keeps running
  int rc = create_instance(r.nx, r.ny, r.p, r.p, r.rknstg, r.left, r.right, r.bottom, r.top, r.gamma, r.bc_kind,
                           r.bc_state8, r.u0, !s->batched, s->arena.base + off, &h);
  if (rc) {
    s->arena.give(off, need);
    return rc;
  }
  if (s->batched)
    rc = solve_begin_async(h, r.final_T, r.cfl, r.use_oedg, r.use_ldf, r.ent_offset);
  else
    rc = mhd_gpu_solve_begin(h, r.final_T, r.cfl, r.use_oedg, r.use_ldf, r.ent_offset, nullptr, nullptr);
  if (rc < 0 || (rc & MHD_FLAG_INIT_NEG_AVG)) {
    mhd_request_result res;
    std::memset(&res, 0, sizeof(res));
    res.id = r.id;
    res.arrival = r.arrival;
    res.admitted = res.finished = now;
    res.flags = rc > 0 ? rc : 0;
    res.error = rc < 0 ? rc : 0;
    s->results.push_back(res);
    release_instance(s, h, off, need);
    return 1;
  }
  s->used += need;
  s->active.push_back({r, h, need, off, now, false});  // joins the batch after the round in flight
  ++s->stats.admitted;
  return 1;
}

int retire(mhd_server* s, size_t k) {
  mhd_server::Active a = s->active[k];
  s->active.erase(s->active.begin() + k);
  if (s->batched && a.in_batch) mhd_batch_remove(s->batch, a.h);
  if (a.req.u_avg_out) mhd_gpu_download_avg(a.h, a.req.u_avg_out);
  const Ctrl* c = a.h->ctrl_host;
  mhd_request_result res;
  std::memset(&res, 0, sizeof(res));
  res.id = a.req.id;
  res.arrival = a.req.arrival;
  res.admitted = a.admitted;
  res.finished = server_now(s);
  res.steps = c->steps;
  res.retries = c->retries;
  res.t = c->t;
  res.done = c->done;
  res.flags = c->flags;
  s->results.push_back(res);
  s->used -= a.bytes;
  release_instance(s, a.h, a.off, a.bytes);
  ++s->stats.retired;
  return MHD_OK;
}

double since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// admit every arrived run that fits (step 2 of a round)
int admit_arrived(mhd_server* s) {
  const auto t0 = std::chrono::steady_clock::now();
  const double now = server_now(s);
  while (s->next_pending < s->pending.size() && (int)s->active.size() < s->max_active) {
    const mhd_request& r = s->pending[s->next_pending];
    if (r.arrival > now) break;
    int rc = admit(s, r, now);
    if (rc < 0) return rc;
    if (rc == 0) break;  // wait for memory
    ++s->next_pending;
  }
  s->stats.admit_s += since(t0);
  return MHD_OK;
}

int retire_finished(mhd_server* s) {
  const auto t0 = std::chrono::steady_clock::now();
  for (size_t k = 0; k < s->active.size();) {
    const Ctrl* c = s->active[k].h->ctrl_host;
    if (c->done || (c->flags & FLAGS_FATAL)) {
      int rc = retire(s, k);
      if (rc) return rc;
    } else {
      ++k;
    }
  }
  if (s->batched)
    for (auto& a : s->active)
      if (!a.in_batch) {
        int rc = mhd_batch_add(s->batch, a.h);
        if (rc) return rc;
        a.in_batch = true;
      }
  s->stats.retire_s += since(t0);
  return MHD_OK;
}

}  // namespace

extern "C" {

int mhd_gpu_footprint(int nx, int ny, int p, int rknstg, size_t* bytes) {
  if (!bytes || nx < 2 || ny < 2 || p < 1 || p > MAXP || rknstg < 1 || rknstg > 5) return MHD_ERR_INVALID;
  *bytes = instance_bytes(nx, ny, p, rknstg);
  return MHD_OK;
}

int mhd_server_create(size_t hbm_budget_bytes, int max_active, int tries_per_round, int batched,
                      mhd_server_t** out) {
  if (!out || max_active < 1 || tries_per_round < 1) return MHD_ERR_INVALID;
  *out = nullptr;
  mhd_server* s = new (std::nothrow) mhd_server;
  if (!s) return MHD_ERR_INVALID;
  if (cudaGetDevice(&s->device) != cudaSuccess) {
    delete s;
    return MHD_ERR_NO_DEVICE;
  }
  void* base = nullptr;
  if (hbm_budget_bytes < Arena::kAlign || cudaMalloc(&base, hbm_budget_bytes) != cudaSuccess) {
    cudaGetLastError();
    delete s;
    return MHD_ERR_UNSUPPORTED;  // the budget cannot be reserved on this device
  }
  s->arena.reset(static_cast<char*>(base), hbm_budget_bytes);
  s->budget = s->arena.size;
  s->max_active = batched ? max_active : 1;
  s->tries_per_round = tries_per_round;
  s->batched = batched != 0;
  if (s->batched) {
    int rc = mhd_batch_create(&s->batch);
    if (rc) {
      cudaFree(s->arena.base);
      delete s;
      return rc;
    }
  }
  *out = s;
  return MHD_OK;
}

int mhd_server_submit(mhd_server_t* s, const mhd_request* r) {
  if (!s || !r || !r->u0) return MHD_ERR_INVALID;
  if (Arena::round_up(instance_bytes(r->nx, r->ny, r->p, r->rknstg)) > s->budget) return MHD_ERR_UNSUPPORTED;
  s->pending.push_back(*r);
  return MHD_OK;
}

int mhd_server_run(mhd_server_t* s, double max_seconds) {
  if (!s) return MHD_ERR_INVALID;
  CK(cudaSetDevice(s->device));
  if (!s->started) {
    std::stable_sort(s->pending.begin(), s->pending.end(),
                     [](const mhd_request& a, const mhd_request& b) { return a.arrival < b.arrival; });
    s->origin = std::chrono::steady_clock::now();
    s->started = true;
  }
  const double t_end = server_now(s) + (max_seconds > 0 ? max_seconds : 1e300);
  for (;;) {
    // 1. queue the round for the runs already in the batch
    bool launched = false;
    if (s->batched && std::any_of(s->active.begin(), s->active.end(), [](const mhd_server::Active& a) { return a.in_batch; })) {
      const auto t0 = std::chrono::steady_clock::now();
      int rc = mhd_batch_launch(s->batch, s->tries_per_round);
      if (rc) return rc;
      s->stats.launch_s += since(t0);
      ++s->stats.rounds;
      launched = true;
    }
    // 2. admissions overlap the round
    if (s->batched || s->active.empty()) {
      int rc = admit_arrived(s);
      if (rc) {
        if (launched) mhd_batch_wait(s->batch, nullptr);
        return rc;
      }
    }
    // 3. wait (batched) or run the one active run to its end (plain)
    if (launched) {
      const auto t0 = std::chrono::steady_clock::now();
      int rc = mhd_batch_wait(s->batch, nullptr);
      if (rc) return rc;
      s->stats.wait_s += since(t0);
    } else if (!s->batched && !s->active.empty()) {
      const auto t0 = std::chrono::steady_clock::now();
      mhd_gpu_status st;
      int rc = mhd_gpu_advance(s->active[0].h, 0, 64, &st);
      if (rc < 0) return rc;
      s->stats.wait_s += since(t0);
      ++s->stats.rounds;
    }
    // 4. retire finished runs, join new ones
    int rc = retire_finished(s);
    if (rc) return rc;
    if (s->active.empty()) {
      if (s->next_pending >= s->pending.size()) break;
      const auto t0 = std::chrono::steady_clock::now();
      const double wait = s->pending[s->next_pending].arrival - server_now(s);
      if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.001)));
      s->stats.idle_s += since(t0);
    }
    if (server_now(s) > t_end) break;  // checked after a full round: every call makes progress
  }
  return MHD_OK;
}

int mhd_server_pending(const mhd_server_t* s, int* queued, int* active, size_t* used_bytes) {
  if (!s) return MHD_ERR_INVALID;
  if (queued) *queued = (int)(s->pending.size() - s->next_pending);
  if (active) *active = (int)s->active.size();
  if (used_bytes) *used_bytes = s->used;
  return MHD_OK;
}

int mhd_server_results(const mhd_server_t* s, mhd_request_result* out, int cap, int* n) {
  if (!s || !n) return MHD_ERR_INVALID;
  *n = (int)s->results.size();
  if (out)
    for (int i = 0; i < *n && i < cap; ++i) out[i] = s->results[i];
  return MHD_OK;
}

int mhd_server_get_stats(const mhd_server_t* s, mhd_server_stats* out) {
  if (!s || !out) return MHD_ERR_INVALID;
  *out = s->stats;
  if (s->batch) out->graph_captures = s->batch->captures;
  return MHD_OK;
}

int mhd_server_destroy(mhd_server_t* s) {
  if (!s) return MHD_ERR_INVALID;
  cudaSetDevice(s->device);
  if (s->batch && s->batch->in_flight) mhd_batch_wait(s->batch, nullptr);
  for (auto& a : s->active) {
    if (s->batched && a.in_batch) mhd_batch_remove(s->batch, a.h);
    release_instance(s, a.h, a.off, a.bytes);
  }
  if (s->batch) mhd_batch_destroy(s->batch);
  cudaFree(s->arena.base);
  delete s;
  return MHD_OK;
}

}  // extern "C"
