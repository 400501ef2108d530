// Serving loop: continuous batching of MD segments and FIRE quenches.
//
// The reference has no server: each simulation is a separate MPI job
// (scripts/submit_batches_*.sh). Here one worker thread per server owns the
// GPU work. Requests wait in a queue; whenever fewer than max_active_batches
// batches are in flight and the HBM budget allows, the worker admits the
// first request in the admission order together with the following queued
// requests of the same kind in that order (up to max_batch_particles /
// max_batch_systems) as a new batch on its own CUDA stream. The default order
// is least work first (particles x steps), with requests that waited longer
// than max_wait_ms ahead of all others; MDB_ORDER_FIFO admits oldest first. Batches in flight advance in chunks
// issued asynchronously, so the work of requests admitted at different times
// overlaps on the device. After each chunk the worker records the systems
// that finished (their frames and observables become results at once), and
// frees a batch's memory when all of its systems have finished, which lets
// queued requests in.
//
// Every system of a batch evolves exactly as it would alone (per-system cell
// grids, rebuild decisions and fixed-order reductions), so a request's result
// does not depend on what it was batched with.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "mdb200.h"
#include "mdb_util.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
  int64_t id = 0;
  mdb_config_t cfg;
  std::vector<mdb_particle_t> frame;  // the input, then the result frame
  mdb_request_t req;
  mdb_request_result_t res;
  std::string message;
};
using JobPtr = std::shared_ptr<Job>;

struct ActiveBatch {
  mdb_batch_t* b = nullptr;
  int32_t kind = 0;
  std::vector<JobPtr> jobs;  // index = system id
  std::vector<char> harvested;
  int64_t bytes = 0;
  bool in_flight = false;
};

// Device bytes a batch of `particles` particles in `systems` systems is
// expected to hold (state, double buffers, lists, cells); used for admission
// before the batch exists, replaced by the measured figure once it does.
int64_t estimate_bytes(int64_t particles, int64_t systems, int32_t max_nbr) {
  return particles * (400 + 2 * (int64_t)max_nbr) + systems * (64 << 10) + (8 << 20);
}

bool valid_config(const mdb_config_t& c, std::string& why) {
  if (!(c.box_w_global > 0.0) || !(c.box_h_global > 0.0) || !isfinite(c.box_w_global) ||
      !isfinite(c.box_h_global)) {
    why = "box_w_global and box_h_global must be positive";
    return false;
  }
  if (!(c.cutoff > 0.0) || !(c.dt > 0.0) || !isfinite(c.dt)) {
    why = "cutoff and dt must be positive";
    return false;
  }
  if (!(c.MASS_A > 0.0) || !(c.MASS_B > 0.0)) {
    why = "MASS_A and MASS_B must be positive";
    return false;
  }
  if (!(c.SIGMA_AA > 0.0) || !(c.SIGMA_BB > 0.0) || !(c.SIGMA_AB > 0.0)) {
    why = "SIGMA_* must be positive";
    return false;
  }
  return true;
}

// Work of a request for the shortest-first order: particles x steps (FIRE:
// the iteration cap).
double job_work(const Job& j) {
  const double steps = (j.req.kind == MDB_JOB_FIRE) ? (double)j.req.max_steps : (double)j.req.nsteps;
  return (double)j.frame.size() * steps;
}

std::string last_error_text() {
  char buf[512];
  mdb_last_error(buf, sizeof buf);
  return std::string(buf);
}

}  // namespace

struct mdb_server {
  mdb_server_options_t opt;
  int64_t budget = 0;
  Clock::time_point t0;
  std::mutex mu;
  std::condition_variable wake;      // submissions, shutdown
  std::condition_variable finished;  // a request reached DONE or FAILED
  std::deque<JobPtr> queue;
  std::unordered_map<int64_t, JobPtr> jobs;
  int64_t next_id = 1;
  bool stop = false;
  // statistics (under mu)
  int64_t submitted = 0, running = 0, n_finished = 0, n_failed = 0;
  int64_t batches_admitted = 0, active_batches = 0, bytes_in_use = 0;
  double particle_steps = 0.0;
  std::thread worker;
  std::vector<ActiveBatch> active;  // worker thread only

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
  void run();
  bool admit();
  bool advance(ActiveBatch& ab);
  void finish(const JobPtr& j, int32_t status, int32_t error, const std::string& msg);
  void fail_rest(ActiveBatch& ab, int32_t error, const std::string& msg);
};

void mdb_server::finish(const JobPtr& j, int32_t status, int32_t error, const std::string& msg) {
  std::lock_guard<std::mutex> lk(mu);
  j->res.status = status;
  j->res.error = error;
  j->res.t_done = now();
  j->message = msg;
  running -= 1;
  if (status == MDB_REQ_DONE) {
    n_finished += 1;
    particle_steps += (double)j->res.n * (double)j->res.steps;
  } else {
    n_failed += 1;
  }
  finished.notify_all();
}

void mdb_server::fail_rest(ActiveBatch& ab, int32_t error, const std::string& msg) {
  for (size_t s = 0; s < ab.harvested.size(); ++s)
    if (!ab.harvested[s]) {
      ab.harvested[s] = 1;
      finish(ab.jobs[s], MDB_REQ_FAILED, error, msg);
    }
}

// Forms and starts one batch from the queue; false when nothing was admitted.
bool mdb_server::admit() {
  std::vector<JobPtr> group;
  int64_t est = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (queue.empty() || (int)active.size() >= opt.max_active_batches) return false;
    // candidates in admission order (queue order for FIFO)
    std::vector<JobPtr> order(queue.begin(), queue.end());
    if (opt.order == MDB_ORDER_SHORTEST) {
      const double t = now(), wait = 1e-3 * (double)opt.max_wait_ms;
      auto overdue = [&](const JobPtr& j) {
        return opt.max_wait_ms > 0 && t - j->res.t_submit > wait;
      };
      std::stable_sort(order.begin(), order.end(), [&](const JobPtr& a, const JobPtr& b) {
        const bool oa = overdue(a), ob = overdue(b);
        if (oa != ob) return oa;                                 // overdue first,
        if (oa) return a->res.t_submit < b->res.t_submit;        // oldest first;
        return job_work(*a) < job_work(*b);                      // then least work
      });
    }
    const int32_t kind = order.front()->req.kind;
    int64_t particles = 0;
    for (auto it = order.begin(); it != order.end(); ++it) {
      const JobPtr j = *it;
      const int64_t n = (int64_t)j->frame.size();
      if (j->req.kind != kind) continue;
      const bool first = group.empty();
      if (!first && ((int)group.size() >= opt.max_batch_systems ||
                     particles + n > opt.max_batch_particles))
        break;
      const int64_t e = estimate_bytes(particles + n, (int64_t)group.size() + 1, opt.max_neighbors);
      if (bytes_in_use + e > budget) {
        if (first && active.empty()) {
          // does not fit even alone on an idle device: fail it
          queue.erase(std::find(queue.begin(), queue.end(), j));
          j->res.status = MDB_REQ_FAILED;
          j->res.error = MDB_ERR_CAPACITY;
          j->res.t_done = now();
          j->message = "request does not fit the server's HBM budget";
          n_failed += 1;
          finished.notify_all();
          return true;
        }
        break;
      }
      group.push_back(j);
      particles += n;
      est = e;
    }
    if (group.empty()) return false;
    for (const JobPtr& j : group) queue.erase(std::find(queue.begin(), queue.end(), j));
    const double t = now();
    for (auto& j : group) {
      j->res.status = MDB_REQ_RUNNING;
      j->res.t_start = t;
    }
    running += (int64_t)group.size();
    bytes_in_use += est;
    batches_admitted += 1;
    active_batches += 1;
  }
  ActiveBatch ab;
  ab.kind = group.front()->req.kind;
  ab.jobs = group;
  ab.harvested.assign(group.size(), 0);
  mdb_options_t o;
  mdb_options_default(&o);
  o.device = opt.device;
  o.skin = opt.skin;
  o.use_graphs = opt.use_graphs;
  o.max_neighbors = opt.max_neighbors;
  if (opt.priorities) {
    // One stream priority level per decade of batch work (particles x steps):
    // below 1e9 the highest, 1e12 and above the lowest above normal.
    double w = 0.0;
    for (const JobPtr& j : group) w += job_work(*j);
    o.stream_priority = std::min(5, std::max(1, 13 - (int)floor(log10(std::max(w, 1.0)))));
  }
  int rc = mdb_batch_create(&o, &ab.b);
  for (size_t k = 0; rc == MDB_OK && k < group.size(); ++k) {
    const Job& j = *group[k];
    const int64_t n = (int64_t)j.frame.size();
    if (ab.kind == MDB_JOB_FIRE)
      rc = mdb_batch_add_fire(ab.b, &j.cfg, j.frame.data(), n, j.req.force_tol, j.req.max_steps,
                              &j.req.fire, nullptr);
    else
      rc = mdb_batch_add_md(ab.b, &j.cfg, j.frame.data(), n, j.req.kind, j.req.nsteps, nullptr);
  }
  int64_t issued = 0;
  if (rc == MDB_OK) rc = mdb_batch_issue(ab.b, opt.chunk, &issued);  // builds, then issues
  if (rc != MDB_OK) {
    const std::string msg = last_error_text();
    fail_rest(ab, rc, msg);
    if (ab.b) mdb_batch_destroy(ab.b);
    std::lock_guard<std::mutex> lk(mu);
    bytes_in_use -= est;
    active_batches -= 1;
    return true;
  }
  mdb_batch_device_bytes(ab.b, &ab.bytes);
  {
    std::lock_guard<std::mutex> lk(mu);
    bytes_in_use += ab.bytes - est;  // the measured figure replaces the estimate
  }
  ab.in_flight = issued > 0;
  active.push_back(std::move(ab));
  return true;
}

// Collects a finished chunk, turns finished systems into results and issues
// the next chunk. Returns true when the batch is complete (all harvested).
bool mdb_server::advance(ActiveBatch& ab) {
  int rc = MDB_OK;
  if (ab.in_flight) {
    int32_t idle = 0;
    rc = mdb_batch_query(ab.b, &idle);
    if (rc == MDB_OK && !idle) return false;
    if (rc == MDB_OK) rc = mdb_batch_collect(ab.b);
    ab.in_flight = false;
  }
  const int32_t ns = (int32_t)ab.jobs.size();
  std::vector<int32_t> newly, flags((size_t)ns, 0);
  if (rc == MDB_OK) rc = mdb_batch_done_flags(ab.b, flags.data(), ns);
  for (int32_t s = 0; rc == MDB_OK && s < ns; ++s)
    if (!ab.harvested[s] && flags[s]) newly.push_back(s);
  if (rc == MDB_OK && !newly.empty()) {
    std::vector<double> K(ns), U(ns), xi(ns);
    if (ab.kind != MDB_JOB_FIRE) rc = mdb_batch_energies_all(ab.b, K.data(), U.data(), xi.data(), ns);
    for (int32_t s : newly) {
      if (rc != MDB_OK) break;
      Job& j = *ab.jobs[s];
      const int64_t n = (int64_t)j.frame.size();
      std::vector<mdb_particle_t> out((size_t)n);
      rc = mdb_batch_get_frame(ab.b, s, out.data(), n);
      if (rc != MDB_OK) break;
      j.res.n = n;
      if (ab.kind == MDB_JOB_FIRE) {
        mdb_minimize_result_t r;
        rc = mdb_batch_get_fire_result(ab.b, s, &r, nullptr, nullptr, 0);
        if (rc != MDB_OK) break;
        j.res.steps = r.steps;
        j.res.converged = r.converged;
        j.res.max_force = r.max_force;
        j.res.U = r.potential_energy;
        j.res.nonfinite = r.nonfinite;
      } else {
        int32_t done = 0;
        int64_t steps = 0, nn = 0;
        rc = mdb_batch_system_info(ab.b, s, &nn, &done, &steps);
        if (rc != MDB_OK) break;
        j.res.steps = steps;
        j.res.K = K[s];
        j.res.U = U[s];
        j.res.xi = xi[s];
        j.res.nonfinite = (isfinite(K[s]) && isfinite(U[s])) ? 0 : 1;
      }
      {
        std::lock_guard<std::mutex> lk(mu);
        j.frame.swap(out);  // the result frame replaces the input
      }
      ab.harvested[s] = 1;
      finish(ab.jobs[s], MDB_REQ_DONE, MDB_OK, std::string());
    }
  }
  if (rc != MDB_OK) {
    fail_rest(ab, rc, last_error_text());
    return true;
  }
  bool all = true;
  for (char h : ab.harvested) all = all && h;
  if (all) return true;
  int64_t issued = 0;
  rc = mdb_batch_issue(ab.b, opt.chunk, &issued);
  if (rc != MDB_OK || issued == 0) {
    fail_rest(ab, rc != MDB_OK ? rc : MDB_ERR_STATE,
              rc != MDB_OK ? last_error_text() : "batch stopped before every system finished");
    return true;
  }
  ab.in_flight = true;
  return false;
}

void mdb_server::run() {
  cudaSetDevice(opt.device);
  for (;;) {
    bool progress = false;
    bool stopping;
    {
      std::lock_guard<std::mutex> lk(mu);
      stopping = stop;
      if (stopping && !queue.empty()) {
        for (auto& j : queue) {
          j->res.status = MDB_REQ_FAILED;
          j->res.error = MDB_ERR_STATE;
          j->res.t_done = now();
          j->message = "server shut down before the request ran";
          n_failed += 1;
        }
        queue.clear();
        finished.notify_all();
      }
    }
    if (!stopping)
      while (admit()) progress = true;
    for (size_t k = 0; k < active.size();) {
      ActiveBatch& ab = active[k];
      bool complete;
      if (stopping) {
        // let the chunk in flight end, then drop the batch
        int32_t idle = 1;
        if (ab.in_flight && mdb_batch_query(ab.b, &idle) == MDB_OK && !idle) {
          ++k;
          continue;
        }
        fail_rest(ab, MDB_ERR_STATE, "server shut down");
        complete = true;
      } else {
        complete = advance(ab);
      }
      if (complete) {
        mdb_batch_destroy(ab.b);
        {
          std::lock_guard<std::mutex> lk(mu);
          bytes_in_use -= ab.bytes;
          active_batches -= 1;
        }
        active.erase(active.begin() + (long)k);
        progress = true;
      } else {
        ++k;
      }
    }
    if (stopping && active.empty()) return;
    if (!progress) {
      std::unique_lock<std::mutex> lk(mu);
      wake.wait_for(lk, std::chrono::microseconds(200));
    }
  }
}

extern "C" {

void mdb_server_options_default(mdb_server_options_t* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->device = 0;
  o->max_active_batches = 8;
  o->hbm_budget_bytes = 0;
  // 1Mi: small batches let short requests through (served stream p50: 8Mi 85 s,
  // 2Mi 55 s, 1Mi 38 s at the same throughput); a larger request runs alone
  o->max_batch_particles = 1 << 20;
  o->max_batch_systems = 1024;
  o->chunk = 500;
  o->skin = 0.0;
  o->use_graphs = 1;
  o->max_neighbors = 48;
  o->order = MDB_ORDER_SHORTEST;
  o->max_wait_ms = 60000;
  o->priorities = 1;
}

int mdb_server_create(const mdb_server_options_t* opt, mdb_server_t** out) {
  if (!out) return mdb::set_error(MDB_ERR_ARG, "null argument");
  *out = nullptr;
  std::unique_ptr<mdb_server> s(new (std::nothrow) mdb_server());
  if (!s) return mdb::set_error(MDB_ERR_CAPACITY, "out of host memory");
  if (opt)
    s->opt = *opt;
  else
    mdb_server_options_default(&s->opt);
  mdb_server_options_t& o = s->opt;
  if (o.max_active_batches <= 0 || o.max_batch_systems <= 0 || o.max_batch_particles <= 0 ||
      o.chunk <= 0)
    return mdb::set_error(MDB_ERR_ARG, "server limits must be positive");
  if ((o.order != MDB_ORDER_FIFO && o.order != MDB_ORDER_SHORTEST) || o.max_wait_ms < 0)
    return mdb::set_error(MDB_ERR_ARG, "bad admission order or max_wait_ms");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return mdb::set_error(MDB_ERR_NODEVICE, "no CUDA device available");
  if (o.device < 0 || o.device >= ndev) return mdb::set_error(MDB_ERR_ARG, "bad device ordinal");
  MDB_CUDA(cudaSetDevice(o.device));
  if (o.hbm_budget_bytes > 0) {
    s->budget = o.hbm_budget_bytes;
  } else {
    size_t fr = 0, tot = 0;
    MDB_CUDA(cudaMemGetInfo(&fr, &tot));
    s->budget = (int64_t)((double)fr * 0.8);
  }
  s->t0 = Clock::now();
  mdb_server* raw = s.get();
  s->worker = std::thread([raw] { raw->run(); });
  *out = s.release();
  return MDB_OK;
}

int mdb_server_destroy(mdb_server_t* s) {
  if (!s) return MDB_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->wake.notify_all();
  if (s->worker.joinable()) s->worker.join();
  delete s;
  return MDB_OK;
}

int mdb_server_submit(mdb_server_t* s, const mdb_config_t* cfg, const mdb_particle_t* frame,
                      int64_t n, const mdb_request_t* req, int64_t* id) {
  if (!s || !cfg || !frame || !req || n <= 0) return mdb::set_error(MDB_ERR_ARG, "bad arguments");
  if (n > INT32_MAX / 2) return mdb::set_error(MDB_ERR_CAPACITY, "too many particles");
  if (req->kind == MDB_JOB_FIRE) {
    if (req->max_steps <= 0) return mdb::set_error(MDB_ERR_ARG, "max_steps must be positive");
  } else if (req->kind == MDB_JOB_NVE || req->kind == MDB_JOB_NVT) {
    if (req->nsteps <= 0 || req->nsteps > INT32_MAX)
      return mdb::set_error(MDB_ERR_ARG, "nsteps out of range");
  } else {
    return mdb::set_error(MDB_ERR_ARG, "unknown request kind");
  }
  std::string why;
  if (!valid_config(*cfg, why)) return mdb::set_error(MDB_ERR_CONFIG, why);
  JobPtr j = std::make_shared<Job>();
  j->cfg = *cfg;
  j->frame.assign(frame, frame + n);
  j->req = *req;
  memset(&j->res, 0, sizeof(j->res));
  j->res.status = MDB_REQ_QUEUED;
  j->res.n = n;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return mdb::set_error(MDB_ERR_STATE, "server is shutting down");
    j->id = s->next_id++;
    j->res.t_submit = s->now();
    s->queue.push_back(j);
    s->jobs[j->id] = j;
    s->submitted += 1;
  }
  s->wake.notify_all();
  if (id) *id = j->id;
  return MDB_OK;
}

int mdb_server_wait(mdb_server_t* s, int64_t id, double timeout_s, mdb_request_result_t* info) {
  if (!s) return mdb::set_error(MDB_ERR_ARG, "null argument");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return mdb::set_error(MDB_ERR_ARG, "unknown request id");
  JobPtr j = it->second;
  auto ready = [&] {
    return j->res.status == MDB_REQ_DONE || j->res.status == MDB_REQ_FAILED;
  };
  if (timeout_s < 0)
    s->finished.wait(lk, ready);
  else
    s->finished.wait_for(lk, std::chrono::duration<double>(timeout_s), ready);
  if (info) *info = j->res;
  return MDB_OK;
}

int mdb_server_result(mdb_server_t* s, int64_t id, mdb_particle_t* frame_out, int64_t n,
                      mdb_request_result_t* info) {
  if (!s) return mdb::set_error(MDB_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return mdb::set_error(MDB_ERR_ARG, "unknown request id");
  JobPtr j = it->second;
  if (info) *info = j->res;
  if (j->res.status == MDB_REQ_QUEUED || j->res.status == MDB_REQ_RUNNING)
    return mdb::set_error(MDB_ERR_STATE, "request has not finished");
  if (j->res.status == MDB_REQ_FAILED) {
    s->jobs.erase(it);
    return mdb::set_error(j->res.error ? j->res.error : MDB_ERR_STATE, j->message);
  }
  if (frame_out) {
    if (n != (int64_t)j->frame.size())
      return mdb::set_error(MDB_ERR_CAPACITY, "n must equal the request's particle count");
    memcpy(frame_out, j->frame.data(), sizeof(mdb_particle_t) * (size_t)n);
  }
  s->jobs.erase(it);
  return MDB_OK;
}

int mdb_server_stats(mdb_server_t* s, mdb_server_stats_t* out) {
  if (!s || !out) return mdb::set_error(MDB_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  memset(out, 0, sizeof(*out));
  out->submitted = s->submitted;
  out->queued = (int64_t)s->queue.size();
  out->running = s->running;
  out->finished = s->n_finished;
  out->failed = s->n_failed;
  out->batches_admitted = s->batches_admitted;
  out->active_batches = s->active_batches;
  out->device_bytes = s->bytes_in_use;
  out->hbm_budget_bytes = s->budget;
  out->particle_steps = s->particle_steps;
  out->elapsed_s = s->now();
  return MDB_OK;
}

}  // extern "C"
