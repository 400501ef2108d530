// The NPH driver protocol of the reference's NPH test driver
// (tests/run_NPH_test/run_test_NPH.cpp:137-290; docs/20260303_NPH.md, steps
// of the protocol): AUTO_TARGET (Nose-Hoover steps whose sampled pressure sets
// the target) -> NPH_WARMUP (NPH at the target until a rolling window of
// pressure samples is within tolerance for enough consecutive steps, or a
// step limit) -> NPH_PRODUCTION (a fixed number of NPH steps).
//
// The reference runs one step per loop iteration with a host round trip each
// time. By default the whole protocol runs as one graph launch with the
// decisions on the device (mdb_nph_graph.cu). The host-driven form here
// issues the steps between two points where the protocol can observe or
// decide anything (a pressure sample, the end of a phase, the step at which
// the warmup criterion can first be met) as one chunk of captured steps, so
// the host waits once per sample instead of once per step; it also serves the
// dry run. The decisions are taken exactly where the per-step loop takes
// them.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <deque>
#include <numeric>
#include <vector>

#include "mdb200.h"
#include "mdb_engine.h"
#include "mdb_util.h"

namespace {

#define MDB_TRY(expr)              \
  do {                             \
    const int rc_ = (expr);        \
    if (rc_ != MDB_OK) return rc_; \
  } while (0)

enum { PH_AUTO = 0, PH_WARMUP = 1, PH_PRODUCTION = 2 };

// What the protocol needs from a simulation.
struct Driver {
  virtual ~Driver() = default;
  // advance k steps of the phase (Nose-Hoover for AUTO_TARGET, NPH at p else)
  virtual int steps(int phase, double p, int64_t k) = 0;
  // P_inst after the last step: cal_instant_pressure in AUTO_TARGET,
  // get_last_instant_pressure in the NPH phases
  virtual int pressure(int phase, int64_t step, double* out) = 0;
  virtual int observe(double* t, double* Lx, double* Ly, double* rate) = 0;
};

struct SimDriver : Driver {
  mdb_sim_t* sim;
  explicit SimDriver(mdb_sim_t* s) : sim(s) {}
  int steps(int phase, double p, int64_t k) override {
    return phase == PH_AUTO ? mdb_sim_step_nose_hoover(sim, k, 0) : mdb_sim_step_nph(sim, p, k);
  }
  int pressure(int phase, int64_t, double* out) override {
    if (phase == PH_AUTO) return mdb_sim_instant_pressure(sim, out);
    mdb_observables_t o;
    const int rc = mdb_sim_observables(sim, &o);
    *out = o.last_instant_pressure;
    return rc;
  }
  int observe(double* t, double* Lx, double* Ly, double* rate) override {
    mdb_observables_t o;
    const int rc = mdb_sim_observables(sim, &o);
    *t = o.t;
    *Lx = o.Lx;
    *Ly = o.Ly;
    *rate = o.nph_area_rate;
    return rc;
  }
};

// Pressures given per step (the dry run: protocol logic without a GPU).
struct ScriptDriver : Driver {
  const double* p;
  int64_t n;
  int64_t done = 0;
  int64_t chunks = 0;
  ScriptDriver(const double* pp, int64_t nn) : p(pp), n(nn) {}
  int steps(int, double, int64_t k) override {
    done += k;
    chunks += 1;
    return MDB_OK;
  }
  int pressure(int, int64_t step, double* out) override {
    if (step < 0 || step >= n) return mdb::set_error(MDB_ERR_CAPACITY, "script too short");
    *out = p[step];
    return MDB_OK;
  }
  int observe(double* t, double* Lx, double* Ly, double* rate) override {
    *t = (double)done;
    *Lx = *Ly = 0.0;
    *rate = 0.0;
    return MDB_OK;
  }
};

struct Stats {
  double mean = 0.0, stddev = 0.0;
};

// compute_stats (run_test_NPH.cpp:36-56): mean and sample standard deviation.
Stats window_stats(const std::deque<double>& v) {
  Stats s;
  if (v.empty()) return s;
  s.mean = std::accumulate(v.begin(), v.end(), 0.0) / (double)v.size();
  if (v.size() <= 1) return s;
  double var = 0.0;
  for (double x : v) {
    const double d = x - s.mean;
    var += d * d;
  }
  s.stddev = sqrt(var / (double)(v.size() - 1));
  return s;
}

int run_protocol(Driver& d, const mdb_nph_protocol_t& q, mdb_nph_record_t* rec, int64_t cap,
                 mdb_nph_result_t* res) {
  const int64_t eval = std::max(1, q.eval_interval);
  const int64_t auto_steps = std::max(1, q.auto_steps);
  const size_t window = (size_t)std::max(2, q.window_samples);
  const int64_t stable_req = std::max(1, q.stable_required);
  const int64_t warm_min = std::max(0, q.warmup_min_steps);
  const int64_t warm_max = std::max<int64_t>(warm_min + 1, q.warmup_max_steps);
  const int64_t prod = std::max(1, q.production_steps);
  const int64_t hard = auto_steps + warm_max + prod + 50000;
  int phase = q.auto_target ? PH_AUTO : PH_WARMUP;
  double P_target = q.auto_target ? 0.0 : q.P_target;
  int64_t auto_done = 0, warm_done = 0, prod_done = 0, stable = 0, nrec = 0;
  std::deque<double> auto_samples, win;
  memset(res, 0, sizeof(*res));
  res->auto_end_step = -1;
  res->warmup_end_step = -1;
  int64_t step = 0;
  bool finished = false;
  while (step < hard && !finished) {
    const int used = phase;
    // Steps [step, step + k) change nothing the protocol looks at except its
    // counters: stop before the next sample step, the end of the phase, and
    // (warmup) the first step at which the stability test runs or switches.
    const int64_t next_sample = (step % eval == 0) ? step : step + (eval - step % eval);
    int64_t k = next_sample - step;  // steps before the sample step
    bool window_ok = false;          // warmup test result with the current window
    if (used == PH_AUTO) {
      k = std::min(k, auto_steps - auto_done - 1);
    } else if (used == PH_WARMUP) {
      k = std::min(k, warm_max - warm_done - 1);
      if (warm_done + 1 < warm_min) {
        k = std::min(k, warm_min - warm_done - 1);
      } else if (win.size() >= window) {
        const Stats st = window_stats(win);
        const double den = std::max(1e-12, fabs(P_target));
        window_ok = fabs(st.mean - P_target) / den <= q.tolerance_rel &&
                    st.stddev / den <= q.tolerance_rel;
        if (window_ok) k = std::min(k, stable_req - stable - 1);
      }
    } else {
      k = std::min(k, prod - prod_done - 1);
    }
    k = std::max<int64_t>(0, std::min(k, hard - step - 1));
    if (k > 0) {
      // k quiet steps: counters only (the stability test gives the same
      // answer on each of them, the window does not change)
      MDB_TRY(d.steps(used, P_target, k));
      step += k;
      if (used == PH_AUTO) auto_done += k;
      if (used == PH_WARMUP) {
        if (warm_done + k >= warm_min && win.size() >= window) stable = window_ok ? stable + k : 0;
        warm_done += k;
      }
      if (used == PH_PRODUCTION) prod_done += k;
      continue;
    }
    // one step with the per-step logic of the driver
    MDB_TRY(d.steps(used, P_target, 1));
    const bool sample = (step % eval == 0);
    double P_inst = 0.0;
    if (sample) MDB_TRY(d.pressure(used, step, &P_inst));
    if (used == PH_AUTO)
      ++auto_done;
    else if (used == PH_WARMUP)
      ++warm_done;
    else
      ++prod_done;
    if (sample) {
      if (used == PH_AUTO) {
        auto_samples.push_back(P_inst);
      } else {
        win.push_back(P_inst);
        while (win.size() > window) win.pop_front();
      }
    }
    if (used == PH_AUTO && auto_done >= auto_steps && !auto_samples.empty()) {
      P_target = std::accumulate(auto_samples.begin(), auto_samples.end(), 0.0) /
                 (double)auto_samples.size();
      phase = PH_WARMUP;
      win.clear();
      stable = 0;
      res->auto_end_step = step;
    }
    if (used == PH_WARMUP) {
      if (warm_done >= warm_min && win.size() >= window) {
        const Stats st = window_stats(win);
        const double den = std::max(1e-12, fabs(P_target));
        const bool ok = fabs(st.mean - P_target) / den <= q.tolerance_rel &&
                        st.stddev / den <= q.tolerance_rel;
        stable = ok ? stable + 1 : 0;
        if (stable >= stable_req) {
          phase = PH_PRODUCTION;
          res->warmup_end_step = step;
        }
      }
      if (phase == PH_WARMUP && warm_done >= warm_max) {
        phase = PH_PRODUCTION;
        res->warmup_end_step = step;
        res->forced_switch = 1;
      }
    }
    if (used == PH_PRODUCTION && prod_done >= prod) finished = true;
    if (sample && rec && nrec < cap) {
      mdb_nph_record_t& r = rec[nrec];
      memset(&r, 0, sizeof(r));
      r.step = step;
      r.phase = used;
      r.P_inst = P_inst;
      r.P_target = P_target;
      const Stats st = window_stats(win);
      r.mean = st.mean;
      r.stddev = st.stddev;
      r.rel_err = fabs(st.mean - P_target) / std::max(1e-12, fabs(P_target));
      double rate = 0.0;
      MDB_TRY(d.observe(&r.t, &r.Lx, &r.Ly, &rate));
      r.dA_dt = (used == PH_AUTO) ? 0.0 : rate;
    }
    if (sample) ++nrec;
    ++step;
  }
  res->P_target = P_target;
  res->total_steps = step;
  res->finished = finished ? 1 : 0;
  res->n_records = nrec;
  return MDB_OK;
}

}  // namespace

extern "C" {

int mdb_nph_protocol_from_config(const mdb_config_t* cfg, mdb_nph_protocol_t* out) {
  if (!cfg || !out) return mdb::set_error(MDB_ERR_ARG, "null argument");
  memset(out, 0, sizeof(*out));
  out->auto_target = strcmp(cfg->pressure_target_mode, "auto_initial") == 0 ? 1 : 0;
  out->P_target = cfg->P_target;
  out->auto_steps = cfg->pressure_target_auto_steps;
  out->eval_interval = cfg->pressure_eval_interval_steps;
  out->window_samples = cfg->pressure_window_samples;
  out->stable_required = cfg->pressure_stable_required_windows;
  out->warmup_min_steps = cfg->nph_warmup_min_steps;
  out->warmup_max_steps = cfg->nph_warmup_max_steps;
  out->production_steps = cfg->nph_steps;
  out->tolerance_rel = cfg->pressure_tolerance_rel;
  return MDB_OK;
}

int mdb_sim_run_nph_protocol(mdb_sim_t* sim, const mdb_nph_protocol_t* protocol,
                             mdb_nph_record_t* records, int64_t cap, mdb_nph_result_t* result) {
  if (!sim || !protocol || !result || cap < 0 || (cap > 0 && !records))
    return mdb::set_error(MDB_ERR_ARG, "bad arguments");
  if (!protocol->host_driven && mdb::sim_uses_graphs(sim))
    return mdb::sim_run_nph_protocol_graph(sim, *protocol, records, cap, result);
  const long long waits0 = mdb::sim_host_waits(sim);
  SimDriver d(sim);
  const int rc = run_protocol(d, *protocol, records, cap, result);
  result->host_waits = mdb::sim_host_waits(sim) - waits0;
  return rc;
}

int mdb_nph_protocol_dry_run(const mdb_nph_protocol_t* protocol, const double* pressures,
                             int64_t n, mdb_nph_record_t* records, int64_t cap,
                             mdb_nph_result_t* result, int64_t* chunks) {
  if (!protocol || !pressures || !result || n < 0 || cap < 0)
    return mdb::set_error(MDB_ERR_ARG, "bad arguments");
  ScriptDriver d(pressures, n);
  const int rc = run_protocol(d, *protocol, records, cap, result);
  if (chunks) *chunks = d.chunks;
  return rc;
}

}  // extern "C"
