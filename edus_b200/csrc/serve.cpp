// serve.cpp — request loop over one batch (C ABI edus_server_*).
//
// Threads: submitters (any caller), a pool of setup threads (build the host
// problem of each request), one loop thread that owns the batch: it admits
// ready requests by HBM footprint, advances the batch one chunk at a time and
// retires finished solves; and one starter thread for requests with the
// Coulomb mean field, which run as contexts of their own: it creates the
// context and launches its whole loop as one CUDA graph (capturing a
// 20 000-step loop takes ~0.4 s of host time), after which the loop thread
// adopts the running context into a batch slot. Only the loop thread calls
// the batch API.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "ctx_hooks.hpp"
#include "host/problem.hpp"

namespace {

struct Request {
  int64_t id = 0;
  edus_params p{};
  std::string workdir;
  std::unique_ptr<edus_problem> pb;
  int status = EDUS_REQ_QUEUED;
  int error = 0;
  std::string message;
  int nbands = 0;
  int64_t nk = 0, steps = 0, footprint = 0;
  int slot = -1;
  double t_submit = 0, t_ready = 0, t_admit = 0, t_done = 0;
  std::vector<edus_obs> obs;
};

}  // namespace

struct edus_server {
  edus_server_options opt{};
  edus_batch* batch = nullptr;
  std::chrono::steady_clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv_setup, cv_loop, cv_done;
  std::map<int64_t, std::unique_ptr<Request>> reqs;
  std::deque<int64_t> setup_q;
  std::vector<int64_t> ready;            // submission order
  std::map<int, int64_t> running;        // slot -> request
  int64_t next_id = 1;
  int64_t submitted = 0, completed = 0, failed = 0;
  int64_t bytes_in_use = 0, peak_bytes = 0;
  int peak_active = 0;
  bool stop = false;
  int loop_error = 0;
  std::vector<std::thread> setup_threads;
  std::thread loop;
  // Coulomb requests admitted by the loop thread and started by the starter
  // thread; their footprint and slot stay reserved until adopted
  struct Started {
    int64_t id;
    edus_ctx* ctx;
    int rc;
    std::string message;
  };
  std::deque<int64_t> start_q;
  std::vector<Started> started;
  std::condition_variable cv_start;
  std::thread starter;
  int64_t reserved_bytes = 0;
  int reserved_slots = 0;

  double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace {

void finish(edus_server* s, Request& r, int status) {
  r.status = status;
  r.t_done = s->now();
  if (status == EDUS_REQ_DONE)
    s->completed++;
  else
    s->failed++;
  s->cv_done.notify_all();
}

void setup_worker(edus_server* s) {
  for (;;) {
    int64_t id;
    Request* r;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_setup.wait(lk, [&] { return s->stop || !s->setup_q.empty(); });
      if (s->stop) return;
      id = s->setup_q.front();
      s->setup_q.pop_front();
      r = s->reqs[id].get();
      r->status = EDUS_REQ_SETUP;
    }
    std::unique_ptr<edus_problem> pb(new (std::nothrow) edus_problem());
    // Wannier models are tabulated on the device at admission
    int rc = pb ? edus::build_problem(r->p, r->workdir.c_str(), pb->P, true) : EDUS_ENOMEM;
    if (rc == 0 && s->opt.drop_decoupled_core && pb->P.nch > 0) {
      // applies only where it holds; otherwise the problem is left as built
      if (edus::drop_decoupled_core(pb->P) != 0) edus::clear_error();
    }
    int64_t bytes = 0;
    if (rc == 0) rc = edus_batch_footprint(s->batch, pb.get(), &bytes);
    std::lock_guard<std::mutex> lk(s->mu);
    if (rc != 0) {
      r->error = rc;
      r->message = edus_last_error();
      finish(s, *r, EDUS_REQ_FAILED);
      continue;
    }
    r->nbands = pb->P.ncv;
    r->nk = pb->P.nk;
    r->steps = pb->P.itfi + 1;
    r->footprint = bytes;
    r->pb = std::move(pb);
    r->status = EDUS_REQ_READY;
    r->t_ready = s->now();
    s->ready.insert(std::upper_bound(s->ready.begin(), s->ready.end(), id), id);
    s->cv_loop.notify_all();
  }
}

void starter_main(edus_server* s) {
  cudaSetDevice(s->opt.batch.device);
  for (;;) {
    int64_t id;
    Request* r;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_start.wait(lk, [&] { return s->stop || !s->start_q.empty(); });
      if (s->stop) return;
      id = s->start_q.front();
      s->start_q.pop_front();
      r = s->reqs[id].get();
    }
    edus_options o;
    edus_options_default(&o);
    o.device = s->opt.batch.device;
    o.use_graphs = 1;
    edus_ctx* ctx = nullptr;
    int rc = edus_create(r->pb.get(), &o, &ctx);
    if (!rc) rc = edus::ctx_start_async(ctx);
    std::string msg = rc ? edus_last_error() : "";
    if (rc && ctx) {
      edus_destroy(ctx);
      ctx = nullptr;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->started.push_back({id, ctx, rc, msg});
    s->cv_loop.notify_all();
  }
}

// Started Coulomb contexts join the batch (loop thread).
void adopt(edus_server* s) {
  std::vector<edus_server::Started> done;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    done.swap(s->started);
  }
  for (auto& st : done) {
    std::lock_guard<std::mutex> lk(s->mu);
    Request* r = s->reqs[st.id].get();
    s->reserved_bytes -= r->footprint;
    s->reserved_slots--;
    int32_t slot = -1;
    int rc = st.rc;
    if (!rc) {
      rc = edus::batch_adopt_context(s->batch, st.ctx, r->pb->P, st.id, &slot);
      if (rc) {
        st.message = edus_last_error();
        edus_destroy(st.ctx);
      }
    }
    if (rc) {
      r->error = rc;
      r->message = st.message;
      r->pb.reset();
      s->bytes_in_use -= r->footprint;
      finish(s, *r, EDUS_REQ_FAILED);
      continue;
    }
    r->slot = slot;
    r->pb.reset();
    s->running[slot] = st.id;
    s->peak_active = std::max(s->peak_active, (int)s->running.size());
  }
}

// Admit ready requests in submission order while they fit. A request that
// does not fit may be passed by younger ones until it has waited max_bypass_s.
void admit(edus_server* s, edus_batch_stats& st) {
  std::vector<int64_t> order;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    order = s->ready;
  }
  const double t = s->now();
  {
    // Coulomb requests being started hold their memory and slot already
    std::lock_guard<std::mutex> lk(s->mu);
    st.bytes_used += s->reserved_bytes;
    st.free_slots -= s->reserved_slots;
  }
  for (int64_t id : order) {
    Request* r;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      r = s->reqs[id].get();
    }
    if (r->footprint > st.bytes_budget) {
      std::lock_guard<std::mutex> lk(s->mu);
      s->ready.erase(std::find(s->ready.begin(), s->ready.end(), id));
      r->error = EDUS_ENOMEM;
      r->message = "footprint exceeds the HBM budget of the server";
      r->pb.reset();
      finish(s, *r, EDUS_REQ_FAILED);
      continue;
    }
    const bool fits = st.free_slots > 0 && st.bytes_used + r->footprint <= st.bytes_budget;
    if (!fits) {
      if (t - r->t_ready > s->opt.max_bypass_s) break;  // hold the line for the oldest
      continue;
    }
    if (r->pb->P.p.coulomb) {
      // started on the starter thread, adopted by the loop when it runs
      std::lock_guard<std::mutex> lk(s->mu);
      s->ready.erase(std::find(s->ready.begin(), s->ready.end(), id));
      r->status = EDUS_REQ_RUNNING;
      r->t_admit = s->now();
      s->reserved_bytes += r->footprint;
      s->reserved_slots++;
      s->start_q.push_back(id);
      st.free_slots--;
      st.bytes_used += r->footprint;
      s->bytes_in_use += r->footprint;
      s->peak_bytes = std::max(s->peak_bytes, s->bytes_in_use);
      s->cv_start.notify_one();
      continue;
    }
    int32_t slot = -1;
    const int rc = edus_batch_add(s->batch, r->pb.get(), id, &slot);
    std::lock_guard<std::mutex> lk(s->mu);
    if (rc == EDUS_ENOMEM) {
      if (s->running.empty()) {
        // nothing will free memory for it
        s->ready.erase(std::find(s->ready.begin(), s->ready.end(), id));
        r->error = rc;
        r->message = edus_last_error();
        r->pb.reset();
        finish(s, *r, EDUS_REQ_FAILED);
      }
      break;
    }
    s->ready.erase(std::find(s->ready.begin(), s->ready.end(), id));
    if (rc != 0) {
      r->error = rc;
      r->message = edus_last_error();
      r->pb.reset();
      finish(s, *r, EDUS_REQ_FAILED);
      continue;
    }
    r->slot = slot;
    r->status = EDUS_REQ_RUNNING;
    r->t_admit = s->now();
    r->pb.reset();  // the device holds everything from here on
    s->running[slot] = id;
    st.free_slots--;
    st.bytes_used += r->footprint;
    s->bytes_in_use += r->footprint;
    s->peak_bytes = std::max(s->peak_bytes, s->bytes_in_use);
    s->peak_active = std::max(s->peak_active, (int)s->running.size());
  }
}

// Health check of a finished request's observable log: 0, EDUS_ENONFINITE
// for a record with a non-finite value, or EDUS_ETRACE for a trace that
// drifted past trace_tol (the reference prints the trace check only,
// headers/Observables_MPI.h:396-410; a served request fails instead).
int log_health(const std::vector<edus_obs>& obs, double trace_tol, std::string& why) {
  for (size_t q = 0; q < obs.size(); q++) {
    const edus_obs& o = obs[q];
    bool finite = std::isfinite(o.trace_dev) && std::isfinite(o.p_cond_max) && std::isfinite(o.p_min);
    for (int x = 0; x < 6; x++) finite = finite && std::isfinite(o.J1[x]);
    for (int x = 0; x < 3; x++) finite = finite && std::isfinite(o.J2[x]);
    for (int c = 0; c < EDUS_MAX_BANDS; c++) finite = finite && std::isfinite(o.pop[c]);
    if (!finite) {
      why = "non-finite observables at output instant " + std::to_string(q);
      return EDUS_ENONFINITE;
    }
    if (trace_tol > 0 && std::fabs(o.trace_dev) > trace_tol) {
      why = "trace drift " + std::to_string(o.trace_dev) + " at output instant " + std::to_string(q);
      return EDUS_ETRACE;
    }
  }
  return 0;
}

int retire(edus_server* s) {
  std::vector<std::pair<int, int64_t>> run;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    run.assign(s->running.begin(), s->running.end());
  }
  for (auto& sr : run) {
    int32_t status = 0, it = 0;
    int64_t tag = 0;
    int rc = edus_batch_poll(s->batch, sr.first, &status, &it, &tag);
    if (rc) return rc;
    if (status != EDUS_INST_DONE) continue;
    int32_t n = 0;
    if ((rc = edus_batch_obs_count(s->batch, sr.first, &n))) return rc;
    std::vector<edus_obs> obs(n);
    if (n && (rc = edus_batch_obs_get(s->batch, sr.first, 0, n, obs.data()))) return rc;
    if ((rc = edus_batch_release(s->batch, sr.first))) return rc;
    std::string why;
    const int health = log_health(obs, s->opt.trace_tol, why);
    std::lock_guard<std::mutex> lk(s->mu);
    Request* r = s->reqs[sr.second].get();
    s->running.erase(sr.first);
    s->bytes_in_use -= r->footprint;
    if (health) {
      r->error = health;
      r->message = "request " + std::to_string(sr.second) + ": " + why;
      finish(s, *r, EDUS_REQ_FAILED);
      continue;
    }
    r->obs.swap(obs);
    finish(s, *r, EDUS_REQ_DONE);
  }
  return 0;
}

void loop_main(edus_server* s) {
  cudaSetDevice(s->opt.batch.device);
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_loop.wait_for(lk, std::chrono::milliseconds(2), [&] {
        return s->stop || !s->ready.empty() || !s->running.empty() || !s->started.empty();
      });
      if (s->stop) return;
      if (s->ready.empty() && s->running.empty() && s->started.empty()) continue;
    }
    adopt(s);
    edus_batch_stats st;
    int rc = edus_batch_stats_get(s->batch, &st);
    if (!rc) admit(s, st);
    bool any;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      any = !s->running.empty();
    }
    // with tiles, one chunk; with Coulomb contexts only, a poll (no wait)
    if (!rc && any)
      rc = edus::batch_has_tiles(s->batch) ? edus_batch_advance(s->batch, s->opt.batch.chunk_steps)
                                           : edus::batch_poll_contexts(s->batch);
    if (!rc && any) rc = retire(s);
    if (rc) {
      // a failed chunk leaves no trustworthy state: fail what is running and stop
      std::lock_guard<std::mutex> lk(s->mu);
      s->loop_error = rc;
      for (auto& sr : s->running) {
        Request* r = s->reqs[sr.second].get();
        r->error = rc;
        r->message = edus_last_error();
        finish(s, *r, EDUS_REQ_FAILED);
      }
      s->running.clear();
      s->stop = true;
      s->cv_setup.notify_all();
      s->cv_start.notify_all();
      return;
    }
  }
}

}  // namespace

extern "C" {

int edus_server_options_default(edus_server_options* o) {
  if (!o) return edus::fail(EDUS_EINVAL, "null argument");
  memset(o, 0, sizeof(*o));
  edus_batch_options_default(&o->batch);
  o->setup_threads = 4;
  o->drop_decoupled_core = 1;
  o->max_bypass_s = 2.0;
  o->trace_tol = 1e-3;
  return 0;
}

int edus_server_create(const edus_server_options* o, edus_server** out) {
  if (!o || !out) return edus::fail(EDUS_EINVAL, "null argument");
  if (o->setup_threads < 1) return edus::fail(EDUS_EINVAL, "setup_threads must be >= 1");
  edus_server* s = new edus_server();
  s->opt = *o;
  s->t0 = std::chrono::steady_clock::now();
  int rc = edus_batch_create(&o->batch, &s->batch);
  if (rc) {
    delete s;
    return rc;
  }
  for (int i = 0; i < o->setup_threads; i++) s->setup_threads.emplace_back(setup_worker, s);
  s->starter = std::thread(starter_main, s);
  s->loop = std::thread(loop_main, s);
  *out = s;
  return 0;
}

int edus_server_submit(edus_server* s, const edus_params* p, const char* workdir, int64_t* id) {
  if (!s || !p || !id) return edus::fail(EDUS_EINVAL, "null argument");
  std::unique_ptr<Request> r(new Request());
  r->p = *p;
  r->workdir = workdir ? workdir : ".";
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) return edus::fail(EDUS_ECANCELLED, "server stopped (loop error %d)", s->loop_error);
  r->id = s->next_id++;
  r->t_submit = s->now();
  *id = r->id;
  s->setup_q.push_back(r->id);
  s->reqs[r->id] = std::move(r);
  s->submitted++;
  s->cv_setup.notify_one();
  return 0;
}

int edus_server_info(edus_server* s, int64_t id, edus_request_info* o) {
  if (!s || !o) return edus::fail(EDUS_EINVAL, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return edus::fail(EDUS_EINVAL, "unknown request %lld", (long long)id);
  const Request& r = *it->second;
  memset(o, 0, sizeof(*o));
  o->status = r.status;
  o->error = r.error;
  o->nbands = r.nbands;
  o->nobs = (int32_t)r.obs.size();
  o->nk = r.nk;
  o->steps = r.steps;
  o->footprint_bytes = r.footprint;
  o->t_submit = r.t_submit;
  o->t_ready = r.t_ready;
  o->t_admit = r.t_admit;
  o->t_done = r.t_done;
  if (r.status == EDUS_REQ_FAILED) edus::fail(r.error, "%s", r.message.c_str());
  return 0;
}

int edus_server_obs(edus_server* s, int64_t id, int32_t first, int32_t count, edus_obs* out) {
  if (!s || !out) return edus::fail(EDUS_EINVAL, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return edus::fail(EDUS_EINVAL, "unknown request %lld", (long long)id);
  const Request& r = *it->second;
  if (r.status != EDUS_REQ_DONE) return edus::fail(EDUS_ENOTREADY, "request %lld is not done", (long long)id);
  if (first < 0 || count < 0 || (size_t)first + count > r.obs.size()) return edus::fail(EDUS_EINVAL, "range outside the log");
  memcpy(out, r.obs.data() + first, sizeof(edus_obs) * count);
  return 0;
}

int edus_server_forget(edus_server* s, int64_t id) {
  if (!s) return edus::fail(EDUS_EINVAL, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return 0;
  if (it->second->status != EDUS_REQ_DONE && it->second->status != EDUS_REQ_FAILED)
    return edus::fail(EDUS_ENOTREADY, "request %lld is still in flight", (long long)id);
  it->second->obs.clear();
  it->second->obs.shrink_to_fit();
  return 0;
}

int edus_server_drain(edus_server* s, double timeout_s) {
  if (!s) return edus::fail(EDUS_EINVAL, "null argument");
  std::unique_lock<std::mutex> lk(s->mu);
  const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                      [&] { return s->completed + s->failed == s->submitted || s->stop; });
  if (s->loop_error) return edus::fail(s->loop_error, "server loop stopped");
  if (!ok) return edus::fail(EDUS_ETIMEOUT, "%lld requests still in flight", (long long)(s->submitted - s->completed - s->failed));
  return 0;
}

int edus_server_stats_get(edus_server* s, edus_server_stats* o) {
  if (!s || !o) return edus::fail(EDUS_EINVAL, "null argument");
  memset(o, 0, sizeof(*o));
  std::vector<double> lat;
  double first = 1e300, last = 0, kps = 0;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    o->submitted = s->submitted;
    o->completed = s->completed;
    o->failed = s->failed;
    o->running = (int64_t)s->running.size();
    o->waiting = s->submitted - s->completed - s->failed - o->running;
    o->peak_bytes = s->peak_bytes;
    o->peak_active = s->peak_active;
    for (const auto& kv : s->reqs) {
      const Request& r = *kv.second;
      first = std::min(first, r.t_submit);
      if (r.status != EDUS_REQ_DONE) continue;
      lat.push_back(r.t_done - r.t_submit);
      last = std::max(last, r.t_done);
      kps += (double)r.nk * r.steps;
    }
  }
  if (!lat.empty()) {
    std::sort(lat.begin(), lat.end());
    auto pct = [&](double q) {
      const double x = q * (lat.size() - 1);
      const size_t i = (size_t)x;
      const double f = x - i;
      return i + 1 < lat.size() ? lat[i] * (1 - f) + lat[i + 1] * f : lat.back();
    };
    o->p50_latency_s = pct(0.50);
    o->p99_latency_s = pct(0.99);
    o->max_latency_s = lat.back();
    o->span_s = last - first;
    if (o->span_s > 0) {
      o->solves_per_s = lat.size() / o->span_s;
      o->kpoint_steps_per_s = kps / o->span_s;
    }
  }
  edus_batch_stats bs;
  if (edus_batch_stats_get(s->batch, &bs) == 0) o->device_ms = bs.device_ms;
  return 0;
}

double edus_server_clock(edus_server* s) { return s ? s->now() : 0.0; }

void edus_server_destroy(edus_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_setup.notify_all();
  s->cv_loop.notify_all();
  s->cv_start.notify_all();
  if (s->loop.joinable()) s->loop.join();
  if (s->starter.joinable()) s->starter.join();
  for (auto& t : s->setup_threads)
    if (t.joinable()) t.join();
  for (auto& st : s->started)
    if (st.ctx) edus_destroy(st.ctx);
  edus_batch_destroy(s->batch);
  delete s;
}

}  // extern "C"
