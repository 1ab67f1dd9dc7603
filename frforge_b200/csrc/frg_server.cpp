// Served execution: a request queue in front of a batch.
//
// Requests (one solve each: descriptor, initial state, integrate! arguments)
// are queued by frg_server_submit.  Every frg_server_pump admits queued
// requests in arrival order into free batch slots while their device
// footprint fits the HBM budget, advances the batch by a bounded number of
// rounds, and delivers finished requests: the final state is copied to the
// caller's host buffer, the result is recorded and the slot is freed for the
// next request (continuous batching: the running instances never wait for
// the queue).  The server has no thread of its own; the caller's loop drives
// it, so arrival timing and latency accounting stay with the caller.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <deque>
#include <new>
#include <unordered_map>
#include <vector>

#include "frg_runtime.h"

using frg::rt::set_err;

namespace {

struct Request {
  int64_t id;
  frg_solve_desc desc;
  const double* u0;  // NULL: the state comes from ic on the device
  frg_ic ic;
  double t0, t_final, cfl, fixed_dt;
  int64_t max_steps;
  double* u_out;
  size_t bytes;
  size_t ndof;
  int hook_slot, hook_id;  // post-step hook applied at admission (id 0: none)
  int hook_nparams;
  double hook_params[2];
};

struct Outcome {
  int done = 0;
  frg_result r{};
  int have_diag = 0;
  frg_diagnostics d{};
};

}  // namespace

struct frg_server {
  frg_ctx* ctx = nullptr;
  frg_batch* batch = nullptr;
  int slots = 0;
  size_t budget = 0;
  int64_t steps_per_pump = 0;
  int64_t next_id = 1;
  std::deque<Request> queue;
  std::vector<Request> active;  // by slot; id 0 = free
  std::unordered_map<int64_t, Outcome> outcome;
  std::vector<int64_t> completed;  // delivered since the last take
  std::vector<frg_result> results;
};

namespace {

size_t ndof_of(const frg_solve_desc* d) {
  const size_t np = (size_t)d->p + 1;
  return d->dim == 2 ? (size_t)d->nx * d->ny * np * np * 4 : (size_t)d->nx * np * 3;
}

void finish(frg_server* s, int64_t id, int status, int64_t n_steps, double t) {
  Outcome& o = s->outcome[id];
  o.done = 1;
  o.r.status = status;
  o.r.n_steps = n_steps;
  o.r.t = t;
  s->completed.push_back(id);
}

// Admit queued requests (arrival order) into free slots within the budget.
int admit(frg_server* s) {
  while (!s->queue.empty()) {
    Request& q = s->queue.front();
    int free_slot = -1;
    for (int i = 0; i < s->slots; ++i)
      if (s->active[i].id == 0) {
        free_slot = i;
        break;
      }
    if (free_slot < 0) return FRG_OK;
    int slot = -1;
    int rc = frg_batch_add(s->batch, &q.desc, &slot);
    if (rc == FRG_ERR_OOM) {
      // budget (or device) full: wait for a running request to free room,
      // unless nothing runs that could
      bool any = false;
      for (const Request& a : s->active) any |= a.id != 0;
      if (any) return FRG_OK;
      finish(s, q.id, FRG_ERR_OOM, 0, q.t0);
      s->queue.pop_front();
      continue;
    }
    if (rc) {
      finish(s, q.id, rc, 0, q.t0);
      s->queue.pop_front();
      continue;
    }
    frg_solve* sv = nullptr;
    frg_batch_get_solve(s->batch, slot, &sv);
    rc = q.u0 ? frg_upload_state(sv, q.u0, q.ndof, q.t0) : frg_set_initial_condition(sv, &q.ic);
    if (!rc && q.hook_id)
      rc = frg_solve_set_hook(sv, q.hook_slot, q.hook_id, q.hook_params, q.hook_nparams);
    if (!rc) rc = frg_batch_start(s->batch, slot, q.t_final, q.cfl, q.fixed_dt, q.max_steps);
    if (rc) {
      frg_batch_remove(s->batch, slot);
      finish(s, q.id, rc, 0, q.t0);
      s->queue.pop_front();
      continue;
    }
    s->active[slot] = q;
    s->queue.pop_front();
  }
  return FRG_OK;
}

}  // namespace

extern "C" {

int frg_server_create(frg_ctx* ctx, int slots, size_t hbm_budget, int64_t steps_per_pump, frg_server** out) {
  if (!ctx || !out || slots < 1 || steps_per_pump < 1) return FRG_ERR_INVALID_ARG;
  *out = nullptr;
  frg_server* s = new (std::nothrow) frg_server();
  if (!s) return FRG_ERR_OOM;
  int rc = frg_batch_create(ctx, slots, hbm_budget, &s->batch);
  if (rc) {
    delete s;
    return rc;
  }
  s->ctx = ctx;
  s->slots = slots;
  s->budget = hbm_budget;
  s->steps_per_pump = steps_per_pump;
  Request empty{};
  s->active.assign(slots, empty);
  s->results.resize(slots);
  frg_batch_set_multirate(s->batch, 1);
  *out = s;
  return FRG_OK;
}

int frg_server_destroy(frg_server* s) {
  if (!s) return FRG_OK;
  frg_batch_destroy(s->batch);
  delete s;
  return FRG_OK;
}

int frg_server_submit(frg_server* s, const frg_solve_desc* desc, const double* u0, double t0, double t_final,
                      double cfl, double fixed_dt, int64_t max_steps, double* u_out, int64_t* request_id) {
  if (!s || !desc || !u0 || !request_id) return FRG_ERR_INVALID_ARG;
  if (max_steps < 1 || (!(fixed_dt > 0.0) && !(cfl > 0.0)))
    return set_err(s->ctx, FRG_ERR_INVALID_ARG, "submit: max_steps >= 1 and cfl > 0 or dt > 0");
  Request q{};
  int rc = frg_solve_bytes(desc, &q.bytes);
  if (rc) return set_err(s->ctx, rc, "submit: invalid descriptor");
  if (s->budget && q.bytes > s->budget) return set_err(s->ctx, FRG_ERR_OOM, "request exceeds the HBM budget");
  q.id = s->next_id++;
  q.desc = *desc;
  q.u0 = u0;
  q.t0 = t0;
  q.t_final = t_final;
  q.cfl = cfl;
  q.fixed_dt = fixed_dt;
  q.max_steps = max_steps;
  q.u_out = u_out;
  q.ndof = ndof_of(desc);
  s->outcome[q.id] = Outcome{};
  s->queue.push_back(q);
  *request_id = q.id;
  return FRG_OK;
}

// As frg_server_submit, with the initial state evaluated on the device at
// admission (frg_set_initial_condition) instead of uploaded.
int frg_server_submit_ic(frg_server* s, const frg_solve_desc* desc, const frg_ic* ic, double t_final, double cfl,
                         double fixed_dt, int64_t max_steps, double* u_out, int64_t* request_id) {
  if (!s || !desc || !ic || !request_id) return FRG_ERR_INVALID_ARG;
  static const double dummy = 0.0;
  int rc = frg_server_submit(s, desc, &dummy, 0.0, t_final, cfl, fixed_dt, max_steps, u_out, request_id);
  if (rc) return rc;
  Request& q = s->queue.back();
  q.u0 = nullptr;
  q.ic = *ic;
  return FRG_OK;
}

// Hook of a queued request, validated against the registry now and applied
// to its solve at admission.
int frg_server_set_hook(frg_server* s, int64_t id, int slot, int hook_id, const double* params, int nparams) {
  if (!s) return FRG_ERR_INVALID_ARG;
  if (slot == FRG_HOOK_PREPROCESS_STATE)
    return set_err(s->ctx, FRG_ERR_UNSUPPORTED_HOOK, "served solves do not run preprocess_state hooks");
  Request* q = nullptr;
  for (Request& r : s->queue)
    if (r.id == id) q = &r;
  if (!q) {
    if (s->outcome.count(id)) return set_err(s->ctx, FRG_ERR_STATE, "set_hook: request already admitted");
    return FRG_ERR_INVALID_ARG;
  }
  if (slot != FRG_HOOK_POST_STEP) return set_err(s->ctx, FRG_ERR_UNSUPPORTED_HOOK, "unknown hook slot");
  if (hook_id != 0) {
    int maxp = -1;
    for (int i = 0, n = frg_hook_count(); i < n; ++i) {
      int sl = -1, hid = -1, np = 0;
      frg_hook_info(i, nullptr, &sl, &hid, &np);
      if (sl == slot && hid == hook_id) maxp = np;
    }
    if (maxp < 0) return set_err(s->ctx, FRG_ERR_UNSUPPORTED_HOOK, "unknown hook implementation");
    if (nparams < 0 || nparams > maxp || nparams > 2 || (nparams > 0 && !params))
      return set_err(s->ctx, FRG_ERR_INVALID_ARG, "hook parameters");
    for (int k = 0; k < nparams; ++k)
      if (!(params[k] > 0.0)) return set_err(s->ctx, FRG_ERR_INVALID_ARG, "hook parameters must be > 0");
  }
  q->hook_slot = slot;
  q->hook_id = hook_id;
  q->hook_nparams = hook_id ? nparams : 0;
  for (int k = 0; k < q->hook_nparams; ++k) q->hook_params[k] = params[k];
  return FRG_OK;
}

int frg_server_cancel(frg_server* s, int64_t id) {
  if (!s) return FRG_ERR_INVALID_ARG;
  auto it = s->outcome.find(id);
  if (it == s->outcome.end()) return FRG_ERR_INVALID_ARG;
  if (it->second.done) return FRG_OK;
  for (auto q = s->queue.begin(); q != s->queue.end(); ++q)
    if (q->id == id) {
      const double t0 = q->t0;
      s->queue.erase(q);
      finish(s, id, FRG_CANCELLED, 0, t0);
      return FRG_OK;
    }
  for (int i = 0; i < s->slots; ++i)
    if (s->active[i].id == id) {
      frg_batch_remove(s->batch, i);
      finish(s, id, FRG_CANCELLED, 0, s->active[i].t0);
      s->active[i].id = 0;
      return FRG_OK;
    }
  return FRG_ERR_STATE;
}

int frg_server_pump(frg_server* s, int* n_done, int* n_queued, int* n_active) {
  if (!s) return FRG_ERR_INVALID_ARG;
  const size_t done0 = s->completed.size();
  int rc = admit(s);
  if (rc) return rc;
  int nrun = 0;
  rc = frg_batch_run(s->batch, s->steps_per_pump, s->results.data(), &nrun);
  if (rc) return rc;
  for (int i = 0; i < s->slots; ++i) {
    Request& a = s->active[i];
    if (a.id == 0) continue;
    const frg_result& r = s->results[i];
    if (r.status == FRG_RUNNING) continue;
    frg_solve* sv = nullptr;
    frg_batch_get_solve(s->batch, i, &sv);
    // diagnostics on the device; the state itself only if the caller wants it
    frg_diagnostics dg;
    rc = frg_diagnostics_compute(sv, FRG_EXACT_NONE, nullptr, 0.0, 0, &dg);
    if (!rc && a.u_out) {
      double t = 0.0;
      rc = frg_download_state(sv, a.u_out, a.ndof, &t);
    }
    finish(s, a.id, rc ? rc : r.status, r.n_steps, r.t);
    if (!rc) {
      Outcome& o = s->outcome[a.id];
      o.have_diag = 1;
      o.d = dg;
    }
    frg_batch_remove(s->batch, i);
    a.id = 0;
  }
  // refill the freed slots at once, so they run in the next pump
  if ((rc = admit(s))) return rc;
  int act = 0;
  for (const Request& a : s->active) act += a.id != 0;
  if (n_done) *n_done = (int)(s->completed.size() - done0);
  if (n_queued) *n_queued = (int)s->queue.size();
  if (n_active) *n_active = act;
  return FRG_OK;
}

int frg_server_result(frg_server* s, int64_t id, int* done, frg_result* r) {
  if (!s || !done) return FRG_ERR_INVALID_ARG;
  auto it = s->outcome.find(id);
  if (it == s->outcome.end()) return FRG_ERR_INVALID_ARG;
  *done = it->second.done;
  if (r) *r = it->second.r;
  return FRG_OK;
}

int frg_server_diagnostics(frg_server* s, int64_t id, frg_diagnostics* out) {
  if (!s || !out) return FRG_ERR_INVALID_ARG;
  auto it = s->outcome.find(id);
  if (it == s->outcome.end()) return FRG_ERR_INVALID_ARG;
  if (!it->second.have_diag) return set_err(s->ctx, FRG_ERR_STATE, "request has no diagnostics (not delivered)");
  *out = it->second.d;
  return FRG_OK;
}

int frg_server_take_completed(frg_server* s, int64_t* ids, int cap, int* n) {
  if (!s || !n || (cap > 0 && !ids)) return FRG_ERR_INVALID_ARG;
  const int k = (int)std::min<size_t>((size_t)(cap > 0 ? cap : 0), s->completed.size());
  for (int i = 0; i < k; ++i) ids[i] = s->completed[i];
  s->completed.erase(s->completed.begin(), s->completed.begin() + k);
  *n = k;
  return FRG_OK;
}

}  // extern "C"
