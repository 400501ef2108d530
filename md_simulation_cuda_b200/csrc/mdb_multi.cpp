// Independent systems spread over several GPUs (no counterpart in the
// reference, which runs one system per job: scripts/submit_batches_*.sh).
//
// mdb_place_lpt places systems on devices by the greedy longest-processing-
// time rule (largest cost first, each to the least-loaded device, ties to the
// lower device). A multi-device batch buffers the systems it is given, places
// them at its first run by that rule on cost = particles x steps (FIRE: the
// iteration cap), and drives one mdb_batch per device from the calling thread:
// a chunk is issued on every device, then each device is collected as it goes
// idle, so the devices run concurrently. No data crosses between devices; a
// system's results do not depend on where it runs (a batch evolves each system
// bit for bit as it would run alone).
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <new>
#include <thread>
#include <vector>

#include "mdb200.h"
#include "mdb_util.h"

namespace {

struct PendingSystem {
  mdb_config_t cfg;
  std::vector<mdb_particle_t> frame;
  int32_t job;  // MDB_JOB_*
  double tol = 0.0;
  int32_t max_steps = 0;
  int64_t nsteps = 0;
  mdb_fire_params_t fire{};
};

}  // namespace

struct mdb_multibatch {
  mdb_options_t opt{};
  std::vector<int32_t> devices;
  std::vector<PendingSystem> pending;
  std::vector<mdb_batch_t*> subs;      // one per device (null when it got no system)
  std::vector<int32_t> where;          // system -> index into devices
  std::vector<int32_t> local;          // system -> id inside its sub-batch
  bool placed = false;
  ~mdb_multibatch() {
    for (mdb_batch_t* b : subs)
      if (b) mdb_batch_destroy(b);
  }
};

namespace {

int place(mdb_multibatch_t* m) {
  if (m->placed) return MDB_OK;
  if (m->pending.empty()) return mdb::set_error(MDB_ERR_STATE, "no systems");
  const int32_t ns = (int32_t)m->pending.size(), nd = (int32_t)m->devices.size();
  std::vector<double> cost(ns);
  for (int32_t s = 0; s < ns; ++s) {
    const PendingSystem& p = m->pending[s];
    const double steps = p.job == MDB_JOB_FIRE ? (double)p.max_steps : (double)p.nsteps;
    cost[s] = (double)p.frame.size() * steps;
  }
  m->where.assign(ns, 0);
  if (int rc = mdb_place_lpt(cost.data(), ns, nd, m->where.data(), nullptr)) return rc;
  m->subs.assign(nd, nullptr);
  m->local.assign(ns, -1);
  for (int32_t d = 0; d < nd; ++d) {
    mdb_options_t o = m->opt;
    o.device = m->devices[d];
    for (int32_t s = 0; s < ns; ++s) {
      if (m->where[s] != d) continue;
      if (!m->subs[d])
        if (int rc = mdb_batch_create(&o, &m->subs[d])) return rc;
      const PendingSystem& p = m->pending[s];
      int rc;
      if (p.job == MDB_JOB_FIRE)
        rc = mdb_batch_add_fire(m->subs[d], &p.cfg, p.frame.data(), (int64_t)p.frame.size(),
                                p.tol, p.max_steps, &p.fire, &m->local[s]);
      else
        rc = mdb_batch_add_md(m->subs[d], &p.cfg, p.frame.data(), (int64_t)p.frame.size(),
                              p.job, p.nsteps, &m->local[s]);
      if (rc) return rc;
    }
  }
  m->pending.clear();  // the sub-batches hold copies now
  m->pending.shrink_to_fit();
  m->placed = true;
  return MDB_OK;
}

int sub_of(mdb_multibatch_t* m, int32_t sys_id, mdb_batch_t** b, int32_t* id) {
  if (int rc = place(m)) return rc;
  if (sys_id < 0 || sys_id >= (int32_t)m->where.size())
    return mdb::set_error(MDB_ERR_ARG, "bad system id");
  *b = m->subs[m->where[sys_id]];
  *id = m->local[sys_id];
  return MDB_OK;
}

int check_kind(mdb_multibatch_t* m, int32_t job) {
  if (m->placed) return mdb::set_error(MDB_ERR_STATE, "systems cannot be added after the first run");
  if (!m->pending.empty() && (m->pending.front().job == MDB_JOB_FIRE) != (job == MDB_JOB_FIRE))
    return mdb::set_error(MDB_ERR_STATE, "every system of a batch has the same kind");
  if (!m->pending.empty() && job != MDB_JOB_FIRE && m->pending.front().job != job)
    return mdb::set_error(MDB_ERR_STATE, "every system of a batch has the same kind");
  return MDB_OK;
}

}  // namespace

extern "C" {

int mdb_place_lpt(const double* costs, int32_t n, int32_t nbins, int32_t* bin_out,
                  double* load_out) {
  if (n < 0 || nbins <= 0 || (n > 0 && (!costs || !bin_out)))
    return mdb::set_error(MDB_ERR_ARG, "bad arguments");
  std::vector<int32_t> order(n);
  for (int32_t k = 0; k < n; ++k) order[k] = k;
  std::stable_sort(order.begin(), order.end(),
                   [&](int32_t a, int32_t b) { return costs[a] > costs[b]; });
  std::vector<double> load(nbins, 0.0);
  for (int32_t k : order) {
    int32_t best = 0;
    for (int32_t d = 1; d < nbins; ++d)
      if (load[d] < load[best]) best = d;
    bin_out[k] = best;
    load[best] += costs[k];
  }
  if (load_out) std::copy(load.begin(), load.end(), load_out);
  return MDB_OK;
}

int mdb_multibatch_create(const mdb_options_t* opt, const int32_t* devices, int32_t ndev,
                          mdb_multibatch_t** out) {
  if (!out || !devices || ndev <= 0) return mdb::set_error(MDB_ERR_ARG, "bad arguments");
  mdb_multibatch_t* m = new (std::nothrow) mdb_multibatch();
  if (!m) return mdb::set_error(MDB_ERR_CAPACITY, "out of host memory");
  if (opt)
    m->opt = *opt;
  else
    mdb_options_default(&m->opt);
  m->devices.assign(devices, devices + ndev);
  *out = m;
  return MDB_OK;
}

int mdb_multibatch_destroy(mdb_multibatch_t* m) {
  delete m;
  return MDB_OK;
}

int mdb_multibatch_add_fire(mdb_multibatch_t* m, const mdb_config_t* cfg,
                            const mdb_particle_t* frame, int64_t n, double force_tol,
                            int32_t max_steps, const mdb_fire_params_t* params, int32_t* sys_id) {
  if (!m || !cfg || !frame || !params || n <= 0 || max_steps <= 0)
    return mdb::set_error(MDB_ERR_ARG, "bad arguments");
  if (int rc = check_kind(m, MDB_JOB_FIRE)) return rc;
  PendingSystem p;
  p.cfg = *cfg;
  p.frame.assign(frame, frame + n);
  p.job = MDB_JOB_FIRE;
  p.tol = force_tol;
  p.max_steps = max_steps;
  p.fire = *params;
  m->pending.push_back(std::move(p));
  if (sys_id) *sys_id = (int32_t)m->pending.size() - 1;
  return MDB_OK;
}

int mdb_multibatch_add_md(mdb_multibatch_t* m, const mdb_config_t* cfg,
                          const mdb_particle_t* frame, int64_t n, int32_t kind, int64_t nsteps,
                          int32_t* sys_id) {
  if (!m || !cfg || !frame || n <= 0 || nsteps <= 0)
    return mdb::set_error(MDB_ERR_ARG, "bad arguments");
  if (kind != MDB_JOB_NVE && kind != MDB_JOB_NVT)
    return mdb::set_error(MDB_ERR_ARG, "kind must be MDB_JOB_NVE or MDB_JOB_NVT");
  if (int rc = check_kind(m, kind)) return rc;
  PendingSystem p;
  p.cfg = *cfg;
  p.frame.assign(frame, frame + n);
  p.job = kind;
  p.nsteps = nsteps;
  m->pending.push_back(std::move(p));
  if (sys_id) *sys_id = (int32_t)m->pending.size() - 1;
  return MDB_OK;
}

int mdb_multibatch_run(mdb_multibatch_t* m, int64_t iterations) {
  if (!m) return mdb::set_error(MDB_ERR_ARG, "null argument");
  if (int rc = place(m)) return rc;
  const size_t nd = m->subs.size();
  std::vector<int64_t> left(nd, iterations);
  std::vector<char> busy(nd, 0), finished(nd, 0);
  for (size_t d = 0; d < nd; ++d) finished[d] = m->subs[d] ? 0 : 1;
  for (;;) {
    bool any = false, progressed = false;
    for (size_t d = 0; d < nd; ++d) {
      if (finished[d]) continue;
      any = true;
      if (busy[d]) {
        int32_t idle = 0;
        if (int rc = mdb_batch_query(m->subs[d], &idle)) return rc;
        if (!idle) continue;
        if (int rc = mdb_batch_collect(m->subs[d])) return rc;
        busy[d] = 0;
        progressed = true;
      }
      if (iterations >= 0 && left[d] <= 0) {
        finished[d] = 1;
        continue;
      }
      int64_t issued = 0;
      if (int rc = mdb_batch_issue(m->subs[d], iterations >= 0 ? left[d] : -1, &issued))
        return rc;
      if (issued == 0) {
        finished[d] = 1;
        continue;
      }
      if (iterations >= 0) left[d] -= issued;
      busy[d] = 1;
      progressed = true;
    }
    if (!any) break;
    if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
  return MDB_OK;
}

int mdb_multibatch_placement(mdb_multibatch_t* m, int32_t* device_of, int32_t n) {
  if (!m || !device_of) return mdb::set_error(MDB_ERR_ARG, "null argument");
  if (int rc = place(m)) return rc;
  if (n != (int32_t)m->where.size())
    return mdb::set_error(MDB_ERR_CAPACITY, "n must equal the number of systems");
  for (int32_t s = 0; s < n; ++s) device_of[s] = m->devices[m->where[s]];
  return MDB_OK;
}

int mdb_multibatch_progress(mdb_multibatch_t* m, int32_t* n_systems, int32_t* n_done) {
  if (!m) return mdb::set_error(MDB_ERR_ARG, "null argument");
  if (!m->placed) {
    if (n_systems) *n_systems = (int32_t)m->pending.size();
    if (n_done) *n_done = 0;
    return MDB_OK;
  }
  int32_t ns = 0, nd = 0;
  for (mdb_batch_t* b : m->subs) {
    if (!b) continue;
    int32_t a = 0, c = 0;
    if (int rc = mdb_batch_progress(b, &a, &c)) return rc;
    ns += a;
    nd += c;
  }
  if (n_systems) *n_systems = ns;
  if (n_done) *n_done = nd;
  return MDB_OK;
}

int mdb_multibatch_system_info(mdb_multibatch_t* m, int32_t sys_id, int64_t* n, int32_t* done,
                               int64_t* steps) {
  if (!m) return mdb::set_error(MDB_ERR_ARG, "null argument");
  mdb_batch_t* b = nullptr;
  int32_t id = 0;
  if (int rc = sub_of(m, sys_id, &b, &id)) return rc;
  return mdb_batch_system_info(b, id, n, done, steps);
}

int mdb_multibatch_get_frame(mdb_multibatch_t* m, int32_t sys_id, mdb_particle_t* out,
                             int64_t n) {
  if (!m) return mdb::set_error(MDB_ERR_ARG, "null argument");
  mdb_batch_t* b = nullptr;
  int32_t id = 0;
  if (int rc = sub_of(m, sys_id, &b, &id)) return rc;
  return mdb_batch_get_frame(b, id, out, n);
}

int mdb_multibatch_get_fire_result(mdb_multibatch_t* m, int32_t sys_id,
                                   mdb_minimize_result_t* result, int32_t* energy_steps,
                                   double* energy_trace, int64_t trace_cap) {
  if (!m) return mdb::set_error(MDB_ERR_ARG, "null argument");
  mdb_batch_t* b = nullptr;
  int32_t id = 0;
  if (int rc = sub_of(m, sys_id, &b, &id)) return rc;
  return mdb_batch_get_fire_result(b, id, result, energy_steps, energy_trace, trace_cap);
}

int mdb_multibatch_energies(mdb_multibatch_t* m, int32_t sys_id, double* K, double* U,
                            double* xi) {
  if (!m) return mdb::set_error(MDB_ERR_ARG, "null argument");
  mdb_batch_t* b = nullptr;
  int32_t id = 0;
  if (int rc = sub_of(m, sys_id, &b, &id)) return rc;
  return mdb_batch_energies(b, id, K, U, xi);
}

}  // extern "C"
