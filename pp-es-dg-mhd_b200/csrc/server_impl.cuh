// server_impl.cuh -- continuous-batching request loop (included by mhd_gpu.cu).
//
// Runs (one solve_execute each) are submitted with an arrival time on the server clock.  The loop
// admits every run whose arrival time has passed while the HBM budget and the active-run cap allow
// (create the instance, upload its initial state, solve_begin), packs all active runs into one
// batch so that every round advances all of them with shared launches, and retires finished runs
// (download u_avg if asked, free their memory) so that waiting runs can be admitted.  With
// batched = 0 it serves the same queue one plain run at a time (mhd_gpu_advance to the end), the
// comparison point for the batched form.
#pragma once
#include <chrono>
#include <deque>
#include <thread>

struct mhd_server {
  int device;
  size_t budget;
  int max_active;
  int tries_per_round;
  int batched;
  size_t used = 0;
  mhd_batch* batch = nullptr;
  std::vector<mhd_request> pending;  // sorted by arrival when run starts
  size_t next_pending = 0;
  struct Active {
    mhd_request req;
    mhd_gpu* h;
    size_t bytes;
    double admitted;
  };
  std::vector<Active> active;
  std::vector<mhd_request_result> results;
  std::chrono::steady_clock::time_point origin;
  bool started = false;
};

namespace {

double server_now(const mhd_server* s) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - s->origin).count();
}

// device bytes mhd_gpu_create allocates for one instance (the same sizes, in the same order)
size_t instance_bytes(int nx, int ny, int p, int R) {
  const size_t eb = 8 * (size_t)(p + 1) * (p + 1);
  const size_t sb = sizeof(double) * (size_t)(nx + 2) * (ny + 2) * eb, tb = sizeof(double) * (size_t)nx * ny * eb;
  const size_t nelg = (size_t)(nx + 2) * (ny + 2);
  const size_t n2 = 2 * (size_t)(p + 1) * (p + 1);
  size_t b = (R + 1) * sb + R * tb + sizeof(double) * 8 * nelg + sb + sizeof(double) * n2 * n2;
  b += sizeof(double) * 8 * (size_t)(nx + 1) * ny + sizeof(double) * 8 * (size_t)nx * (ny + 1);
  b += sizeof(double) * 8 * ((nelg + 15) / 16 + 1) + sizeof(double) * ((nx + 15) / 16 + 1) * (size_t)ny;
  b += 2 * sizeof(double) * nelg + nelg + sizeof(Ctrl);
  return b;
}

int admit(mhd_server* s, const mhd_request& r, double now) {
  mhd_gpu* h = nullptr;
  int rc = mhd_gpu_create(r.nx, r.ny, r.p, r.p, r.rknstg, r.left, r.right, r.bottom, r.top, r.gamma,
                          r.bc_kind, r.bc_state8, &h);
  if (rc) return rc;
  rc = mhd_gpu_upload_state(h, 0, r.u0);
  if (!rc) rc = mhd_gpu_solve_begin(h, r.final_T, r.cfl, r.use_oedg, r.use_ldf, r.ent_offset, nullptr, nullptr);
  if (rc < 0 || (rc & MHD_FLAG_INIT_NEG_AVG)) {
    mhd_request_result res;
    std::memset(&res, 0, sizeof(res));
    res.id = r.id;
    res.arrival = r.arrival;
    res.admitted = res.finished = now;
    res.flags = rc > 0 ? rc : 0;
    res.error = rc < 0 ? rc : 0;
    s->results.push_back(res);
    mhd_gpu_destroy(h);
    return MHD_OK;
  }
  if (s->batched) {
    rc = mhd_batch_add(s->batch, h);
    if (rc) {
      mhd_gpu_destroy(h);
      return rc;
    }
  }
  const size_t bytes = h->bytes;
  s->used += bytes;
  s->active.push_back({r, h, bytes, now});
  return MHD_OK;
}

int retire(mhd_server* s, size_t k) {
  mhd_server::Active a = s->active[k];
  s->active.erase(s->active.begin() + k);
  if (s->batched) mhd_batch_remove(s->batch, a.h);
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
  mhd_gpu_destroy(a.h);
  s->used -= a.bytes;
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
  s->budget = hbm_budget_bytes;
  s->max_active = batched ? max_active : 1;
  s->tries_per_round = tries_per_round;
  s->batched = batched != 0;
  if (s->batched) {
    int rc = mhd_batch_create(&s->batch);
    if (rc) {
      delete s;
      return rc;
    }
  }
  *out = s;
  return MHD_OK;
}

int mhd_server_submit(mhd_server_t* s, const mhd_request* r) {
  if (!s || !r || !r->u0) return MHD_ERR_INVALID;
  if (instance_bytes(r->nx, r->ny, r->p, r->rknstg) > s->budget) return MHD_ERR_UNSUPPORTED;
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
    const double now = server_now(s);
    // admit every arrived run that fits
    while (s->next_pending < s->pending.size() && (int)s->active.size() < s->max_active) {
      const mhd_request& r = s->pending[s->next_pending];
      if (r.arrival > now) break;
      const size_t need = instance_bytes(r.nx, r.ny, r.p, r.rknstg);
      if (s->used + need > s->budget && !s->active.empty()) break;  // wait for memory
      int rc = admit(s, r, now);
      if (rc) return rc;
      ++s->next_pending;
    }
    if (s->active.empty()) {
      if (s->next_pending >= s->pending.size()) break;
      const double wait = s->pending[s->next_pending].arrival - server_now(s);
      if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.01)));
      if (server_now(s) > t_end) break;
      continue;
    }
    if (s->batched) {
      int n_active = 0;
      int rc = mhd_batch_advance(s->batch, s->tries_per_round, &n_active);
      if (rc) return rc;
    } else {
      mhd_gpu_status st;
      int rc = mhd_gpu_advance(s->active[0].h, 0, 64, &st);  // the whole run, one at a time
      if (rc < 0) return rc;
    }
    for (size_t k = 0; k < s->active.size();) {
      const Ctrl* c = s->active[k].h->ctrl_host;
      if (c->done || (c->flags & 0x6)) {
        int rc = retire(s, k);
        if (rc) return rc;
      } else {
        ++k;
      }
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

int mhd_server_destroy(mhd_server_t* s) {
  if (!s) return MHD_ERR_INVALID;
  cudaSetDevice(s->device);
  for (auto& a : s->active) {
    if (s->batched) mhd_batch_remove(s->batch, a.h);
    mhd_gpu_destroy(a.h);
  }
  if (s->batch) mhd_batch_destroy(s->batch);
  delete s;
  return MHD_OK;
}

}  // extern "C"
