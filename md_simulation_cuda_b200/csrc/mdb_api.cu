// extern "C" entry points of libmdb200 (declared in include/mdb200.h).
// The reference-facing semantics (MDSimulation, EnergyMinimizer) live here on
// top of the engine; each function cites the reference code it replaces.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "mdb200.h"
#include "mdb_engine.h"
#include "mdb_util.h"

using mdb::Engine;
using mdb::SysState;
using mdb::SystemSpec;

struct mdb_sim {
  std::unique_ptr<Engine> eng;
  mdb_config_t cfg;
  double t = 0.0;
  bool piston_active = false;  // piston_mode_active (md_env.hpp:218)
  bool k_valid = false;        // S.K holds K of the current velocities
  bool p_valid = false;        // S.P_cur holds the current scalar pressure
  bool nph_init = false;       // nph_state_initialized
  bool vp_init = false;        // nph_piston_velocity_initialized
  int periodic_y = 1;          // y convention of the cell binning
};

namespace {

#define MDB_TRY(expr)            \
  do {                           \
    int rc_ = (expr);            \
    if (rc_ != MDB_OK) return rc_; \
  } while (0)

mdb_options_t opts_or_default(const mdb_options_t* opt) {
  mdb_options_t o;
  mdb_options_default(&o);
  if (opt) o = *opt;
  return o;
}

int check_status(mdb_sim_t* sim) {
  SysState S;
  MDB_TRY(sim->eng->get_state(0, &S));
  if (S.err == MDB_ERR_BOX) return mdb::set_error(MDB_ERR_BOX, "invalid box (area <= 0 or non-finite) in a barostat step");
  if (S.err) return mdb::set_error(S.err, "device error flag set");
  return MDB_OK;
}

int sim_make(const mdb_config_t* cfg, std::vector<mdb_particle_t>&& frame,
             const mdb_options_t* opt, mdb_sim_t** out) {
  std::unique_ptr<mdb_sim> sim(new (std::nothrow) mdb_sim());
  if (!sim) return mdb::set_error(MDB_ERR_CAPACITY, "out of host memory");
  sim->cfg = *cfg;
  mdb_options_t o = opts_or_default(opt);
  // a lone small system splits its pair candidates over four lanes
  if (o.lanes == MDB_LANES_AUTO) o.lanes = MDB_LANES_SPLIT;
  sim->eng.reset(new Engine(o));
  SystemSpec spec;
  spec.cfg = *cfg;
  spec.frame = std::move(frame);
  spec.kind = mdb::K_NVE;
  MDB_TRY(sim->eng->add_system(std::move(spec)));
  MDB_TRY(sim->eng->build());
  // the constructors end with cal_forces() (src/md_env.cu:61-79, 147-158)
  MDB_TRY(sim->eng->force(mdb::FM_INIT, true));
  MDB_TRY(sim->eng->sync());
  *out = sim.release();
  return MDB_OK;
}

// Leaves the piston's walled y convention (every non-piston step sets
// piston_mode_active = false, src/md_env.cu:1577, 1640, 1796).
int leave_piston(mdb_sim_t* sim) {
  sim->piston_active = false;
  if (sim->periodic_y != 1) {
    MDB_TRY(sim->eng->rebuild_now(1));
    sim->periodic_y = 1;
  }
  return MDB_OK;
}

void advance_time(mdb_sim_t* sim, int64_t n) {
  for (int64_t k = 0; k < n; ++k) sim->t += sim->cfg.dt;
}

}  // namespace

namespace mdb {

int sim_export_async(mdb_sim_t* sim, mdb_particle_t* host, cudaEvent_t ev) {
  MDB_TRY(sim->eng->export_async(0, host));
  MDB_CUDA(cudaEventRecord(ev, sim->eng->stream()));
  return MDB_OK;
}

int64_t sim_particles(mdb_sim_t* sim) { return sim->eng->n(0); }

int sim_device(mdb_sim_t* sim) { return sim->eng->device(); }

long long sim_host_waits(mdb_sim_t* sim) { return sim->eng->host_waits(); }

bool sim_uses_graphs(mdb_sim_t* sim) { return sim->eng->graphs(); }

int sim_run_nph_protocol_graph(mdb_sim_t* sim, const mdb_nph_protocol_t& p,
                               mdb_nph_record_t* rec, int64_t cap, mdb_nph_result_t* res) {
  const long long waits0 = sim->eng->host_waits();
  MDB_TRY(leave_piston(sim));
  // parameters clamped as the host protocol clamps them
  NphProto q;
  memset(&q, 0, sizeof(q));
  q.eval = std::max(1, p.eval_interval);
  q.auto_steps = std::max(1, p.auto_steps);
  q.window = std::max(2, p.window_samples);
  q.stable_req = std::max(1, p.stable_required);
  q.warm_min = std::max(0, p.warmup_min_steps);
  q.warm_max = std::max<int64_t>(q.warm_min + 1, p.warmup_max_steps);
  q.prod = std::max(1, p.production_steps);
  q.hard = q.auto_steps + q.warm_max + q.prod + 50000;
  q.tol = p.tolerance_rel;
  q.W = sim->cfg.barostat_mass > 1e-12 ? sim->cfg.barostat_mass : 1e-12;
  q.rate_init = sim->cfg.barostat_area_rate_init;
  q.dt = sim->cfg.dt;
  q.t = sim->t;
  q.phase = p.auto_target ? 0 : 1;
  q.P_target = p.auto_target ? 0.0 : p.P_target;
  q.auto_end = -1;
  q.warm_end = -1;
  q.p_valid = sim->p_valid ? 1 : 0;
  q.nph_init = sim->nph_init ? 1 : 0;
  if (q.phase == 0) {
    // the first Nose-Hoover step needs K of the current velocities
    if (!sim->k_valid) MDB_TRY(sim->eng->reduce_K());
  } else {
    MDB_TRY(sim->eng->set_pext(q.P_target));
  }
  const int rc = sim->eng->run_nph_protocol(&q, rec, cap);
  if (rc != MDB_OK) return rc;
  sim->t = q.t;
  sim->nph_init = q.nph_init != 0;
  if (q.step > 0) {
    if (q.last_phase == 0) {
      sim->k_valid = true;
      sim->p_valid = q.last_sample != 0;
    } else {
      sim->k_valid = false;
      sim->p_valid = true;
    }
  }
  memset(res, 0, sizeof(*res));
  res->P_target = q.P_target;
  res->auto_end_step = q.auto_end;
  res->warmup_end_step = q.warm_end;
  res->total_steps = q.step;
  res->n_records = q.nrec;
  res->forced_switch = q.forced;
  res->finished = q.finished;
  res->host_waits = sim->eng->host_waits() - waits0;
  if (q.err == MDB_ERR_BOX && !q.nph_init)
    return set_error(MDB_ERR_BOX, "invalid initial box for NPH");
  if (q.err != 0) return check_status(sim);
  return MDB_OK;
}

}  // namespace mdb

extern "C" {

int mdb_sim_create(const mdb_config_t* cfg, const mdb_particle_t* frame, int64_t n,
                   const mdb_options_t* opt, mdb_sim_t** out) {
  if (!cfg || !out) return mdb::set_error(MDB_ERR_ARG, "null argument");
  *out = nullptr;
  std::vector<mdb_particle_t> f;
  if (frame) {
    if (n <= 0) return mdb::set_error(MDB_ERR_ARG, "frame size must be positive");
    f.assign(frame, frame + n);
  } else {
    MDB_TRY(mdb::reference_initial_frame(*cfg, f));
    if (n > 0 && n != (int64_t)f.size())
      return mdb::set_error(MDB_ERR_ARG, "n must equal n_particles_global");
  }
  return sim_make(cfg, std::move(f), opt, out);
}

int mdb_sim_create_from_pframe(const mdb_config_t* cfg, const char* path, uint64_t step,
                               const mdb_options_t* opt, mdb_sim_t** out) {
  if (!cfg || !path || !out) return mdb::set_error(MDB_ERR_ARG, "null argument");
  *out = nullptr;
  int64_t n = 0;
  int rc = mdb_pframe_read(path, step, nullptr, 0, &n);
  if (rc != MDB_OK && rc != MDB_ERR_CAPACITY) return rc;
  if (n <= 0) return mdb::set_error(MDB_ERR_IO, "frame is empty");
  std::vector<mdb_particle_t> f((size_t)n);
  MDB_TRY(mdb_pframe_read(path, step, f.data(), n, &n));
  return sim_make(cfg, std::move(f), opt, out);
}

int mdb_sim_destroy(mdb_sim_t* sim) {
  delete sim;
  return MDB_OK;
}

int mdb_sim_step_nve(mdb_sim_t* sim, int64_t nsteps) {
  if (!sim || nsteps < 0) return mdb::set_error(MDB_ERR_ARG, "bad arguments");
  if (nsteps == 0) return MDB_OK;
  MDB_TRY(leave_piston(sim));
  MDB_TRY(sim->eng->run_md(mdb::DM_NVE, mdb::FM_NVE, true, nsteps));
  sim->k_valid = false;
  sim->p_valid = false;
  advance_time(sim, nsteps);
  return MDB_OK;
}

int mdb_sim_step_nose_hoover(mdb_sim_t* sim, int64_t nsteps, int32_t do_middle_wrap) {
  if (!sim || nsteps < 0) return mdb::set_error(MDB_ERR_ARG, "bad arguments");
  if (do_middle_wrap)
    return mdb::set_error(MDB_ERR_ARG, "do_middle_wrap (LG slab reflection) is not provided");
  if (nsteps == 0) return MDB_OK;
  MDB_TRY(leave_piston(sim));
  if (!sim->k_valid) MDB_TRY(sim->eng->reduce_K());
  MDB_TRY(sim->eng->run_md(mdb::DM_NH, mdb::FM_NH, true, nsteps));
  sim->k_valid = true;
  sim->p_valid = false;
  advance_time(sim, nsteps);
  return MDB_OK;
}

int mdb_sim_step_nph(mdb_sim_t* sim, double p_ext, int64_t nsteps) {
  if (!sim || nsteps < 0) return mdb::set_error(MDB_ERR_ARG, "bad arguments");
  if (nsteps == 0) return MDB_OK;
  MDB_TRY(leave_piston(sim));
  SysState S;
  if (!sim->nph_init || !sim->p_valid) {
    if (!sim->p_valid) MDB_TRY(sim->eng->force(mdb::FM_OBS, true));
    MDB_TRY(sim->eng->get_state(0, &S));
    if (S.err) return check_status(sim);
    if (!sim->nph_init) {
      // init_nph_state_if_needed (src/md_env.cu:1757-1778)
      if (!(S.Lx > 0.0) || !(S.Ly > 0.0))
        return mdb::set_error(MDB_ERR_BOX, "invalid initial box for NPH");
      S.aspect = S.Lx / S.Ly;
      const double W = sim->cfg.barostat_mass > 1e-12 ? sim->cfg.barostat_mass : 1e-12;
      S.pA = W * sim->cfg.barostat_area_rate_init;
      sim->nph_init = true;
    }
    if (!sim->p_valid) {
      const double A = S.Lx * S.Ly;
      S.P_cur = (A > 0.0) ? (S.kin + S.Wv) / (2.0 * A) : 0.0;
    }
    MDB_TRY(sim->eng->put_state(0, S));
  }
  MDB_TRY(sim->eng->set_pext(p_ext));
  MDB_TRY(sim->eng->run_md(mdb::DM_NPH, mdb::FM_NPH, true, nsteps));
  sim->p_valid = true;
  sim->k_valid = false;
  advance_time(sim, nsteps);
  return MDB_OK;
}

int mdb_sim_step_nph_piston(mdb_sim_t* sim, double p_ext, int64_t nsteps) {
  if (!sim || nsteps < 0) return mdb::set_error(MDB_ERR_ARG, "bad arguments");
  if (nsteps == 0) return MDB_OK;
  if (!sim->vp_init || !sim->piston_active) {
    // init_nph_piston_state_if_needed (src/md_env.cu:1780-1793)
    if (!sim->piston_active) {
      if (sim->periodic_y != 0) {
        MDB_TRY(sim->eng->rebuild_now(0));
        sim->periodic_y = 0;
      }
      MDB_TRY(sim->eng->force(mdb::FM_INIT, false));
    }
    SysState S;
    MDB_TRY(sim->eng->get_state(0, &S));
    if (!sim->vp_init) {
      S.vp = 0.0;
      sim->vp_init = true;
    }
    if (!sim->piston_active) {
      S.last_P = (S.Lx > 0.0) ? (S.Fp / S.Lx) : 0.0;
      sim->piston_active = true;
    }
    MDB_TRY(sim->eng->put_state(0, S));
  }
  MDB_TRY(sim->eng->set_pext(p_ext));
  MDB_TRY(sim->eng->run_md(mdb::DM_PISTON, mdb::FM_PISTON, false, nsteps));
  sim->k_valid = false;
  sim->p_valid = false;
  advance_time(sim, nsteps);
  return MDB_OK;
}

int mdb_sim_total_K(mdb_sim_t* sim, double* out) {
  if (!sim || !out) return mdb::set_error(MDB_ERR_ARG, "null argument");
  MDB_TRY(sim->eng->reduce_K());
  SysState S;
  MDB_TRY(sim->eng->get_state(0, &S));
  sim->k_valid = true;
  *out = S.K;
  return check_status(sim);
}

int mdb_sim_total_U(mdb_sim_t* sim, double* out) {
  if (!sim || !out) return mdb::set_error(MDB_ERR_ARG, "null argument");
  MDB_TRY(sim->eng->force(mdb::FM_OBS, !sim->piston_active));
  SysState S;
  MDB_TRY(sim->eng->get_state(0, &S));
  *out = sim->piston_active ? S.U + S.wallU : S.U;
  return check_status(sim);
}

int mdb_sim_partial_U_lambda(mdb_sim_t* sim, double epsilon_lambda, double* out) {
  if (!sim || !out) return mdb::set_error(MDB_ERR_ARG, "null argument");
  // periodic_y = piston_mode_active ? 0 : 1 (src/md_env.cu:2369)
  MDB_TRY(sim->eng->force(mdb::FM_OBS, !sim->piston_active));
  SysState S;
  MDB_TRY(sim->eng->get_state(0, &S));
  *out = -epsilon_lambda * S.Wani;
  return check_status(sim);
}

int mdb_sim_n_profile(mdb_sim_t* sim, int32_t nb, int32_t* out) {
  if (!sim || !out || nb <= 0) return mdb::set_error(MDB_ERR_ARG, "bad arguments");
  return sim->eng->profiles(0, nb, sim->periodic_y != 0, nullptr, out);
}

int mdb_sim_density_profile(mdb_sim_t* sim, int32_t nb, double* out) {
  if (!sim || !out || nb <= 0) return mdb::set_error(MDB_ERR_ARG, "bad arguments");
  std::vector<int32_t> c((size_t)2 * nb);
  MDB_TRY(sim->eng->profiles(0, nb, sim->periodic_y != 0, nullptr, c.data()));
  // get_density_profile (src/md_env.cu:4086-4104)
  for (int32_t k = 0; k < nb; ++k) {
    const double a = (double)c[k], b = (double)c[nb + k];
    const double sum = a + b;
    out[k] = (sum == 0.0) ? 0.0 : (a - b) / sum;
  }
  return MDB_OK;
}

int mdb_sim_pressure_profile(mdb_sim_t* sim, int32_t nb, double* out) {
  if (!sim || !out || nb <= 0) return mdb::set_error(MDB_ERR_ARG, "bad arguments");
  std::vector<double> acc((size_t)3 * nb);
  MDB_TRY(sim->eng->profiles(0, nb, sim->periodic_y != 0, acc.data(), nullptr));
  SysState S;
  MDB_TRY(sim->eng->get_state(0, &S));
  // per bin area Lx * (Ly / nb) (src/md_env.cu:3899-3916)
  const double vol = S.Lx * (S.Ly / (double)nb);
  for (size_t k = 0; k < acc.size(); ++k) out[k] = (vol > 0.0) ? acc[k] / vol : acc[k];
  return check_status(sim);
}

int mdb_sim_instant_pressure(mdb_sim_t* sim, double* out) {
  if (!sim || !out) return mdb::set_error(MDB_ERR_ARG, "null argument");
  MDB_TRY(sim->eng->force(mdb::FM_OBS, !sim->piston_active));
  SysState S;
  MDB_TRY(sim->eng->get_state(0, &S));
  if (sim->piston_active) {
    S.Fp = S.kin2;
    S.last_P = (S.Lx > 0.0) ? (S.Fp / S.Lx) : 0.0;
  } else {
    const double A = S.Lx * S.Ly;
    S.last_P = (A > 0.0) ? (S.kin + S.Wv) / (2.0 * A) : 0.0;
    S.P_cur = S.last_P;
    sim->p_valid = true;
  }
  MDB_TRY(sim->eng->put_state(0, S));
  *out = S.last_P;
  return check_status(sim);
}

int mdb_sim_observables(mdb_sim_t* sim, mdb_observables_t* out) {
  if (!sim || !out) return mdb::set_error(MDB_ERR_ARG, "null argument");
  SysState S;
  MDB_TRY(sim->eng->get_state(0, &S));
  memset(out, 0, sizeof(*out));
  out->t = sim->t;
  out->Lx = S.Lx;
  out->Ly = S.Ly;
  out->xi = S.xi;
  out->last_instant_pressure = S.last_P;
  out->nph_area_momentum = S.pA;
  const double W = sim->cfg.barostat_mass > 1e-12 ? sim->cfg.barostat_mass : 1e-12;
  out->nph_area_rate = S.pA / W;
  out->nph_piston_velocity = S.vp;
  out->nph_piston_force = S.Fp;
  out->n = sim->eng->n(0);
  out->steps = S.steps;
  out->rebuilds = S.rebuilds;
  out->piston_mode_active = sim->piston_active ? 1 : 0;
  out->nonfinite = S.nonfinite;
  return check_status(sim);
}

int mdb_sim_observables_async(mdb_sim_t* sim, mdb_observables_t* out) {
  if (!sim || !out) return mdb::set_error(MDB_ERR_ARG, "null argument");
  return sim->eng->observables_async(0, sim->t, sim->piston_active ? 1 : 0, out);
}

int mdb_sim_get_frame(mdb_sim_t* sim, mdb_particle_t* out, int64_t n) {
  if (!sim || !out) return mdb::set_error(MDB_ERR_ARG, "null argument");
  if (n != sim->eng->n(0)) return mdb::set_error(MDB_ERR_CAPACITY, "n must equal the particle count");
  return sim->eng->get_frame(0, out);
}

int mdb_sim_set_frame(mdb_sim_t* sim, const mdb_particle_t* frame, int64_t n) {
  if (!sim || !frame) return mdb::set_error(MDB_ERR_ARG, "null argument");
  if (n != sim->eng->n(0)) return mdb::set_error(MDB_ERR_CAPACITY, "n must equal the particle count");
  MDB_TRY(sim->eng->set_frame(0, frame));
  MDB_TRY(sim->eng->rebuild_now(sim->periodic_y));
  MDB_TRY(sim->eng->force(mdb::FM_INIT, sim->periodic_y != 0));
  sim->k_valid = false;
  sim->p_valid = false;
  return sim->eng->sync();
}

int mdb_sim_save_pframe(mdb_sim_t* sim, const char* path, uint64_t frame_index) {
  if (!sim || !path) return mdb::set_error(MDB_ERR_ARG, "null argument");
  std::vector<mdb_particle_t> f((size_t)sim->eng->n(0));
  MDB_TRY(sim->eng->get_frame(0, f.data()));
  // save_env: open for append, create the file when that fails
  int rc = mdb_pframe_write(path, 1, f.data(), (int64_t)f.size(), frame_index);
  if (rc != MDB_OK) rc = mdb_pframe_write(path, 0, f.data(), (int64_t)f.size(), frame_index);
  return rc;
}

namespace {

// Integrator state beside a PFRAME frame: one "key": value per line.
struct Checkpoint {
  uint64_t frame_index = 0;
  int64_t n = 0, steps = 0;
  double t = 0, Lx = 0, Ly = 0, xi = 0, K = 0, pA = 0, aspect = 0, P_cur = 0, last_P = 0;
  double fl = 0, ce = 0, vp = 0, Fp = 0, wallU = 0, p_ext = 0;
  int clamped = 0, piston_active = 0, nph_init = 0, vp_init = 0, k_valid = 0, p_valid = 0;
  int periodic_y = 1;
};

const char* kCheckpointFormat = "mdb200-checkpoint-1";

bool ck_find(const std::string& text, const char* key, double* out) {
  const std::string pat = std::string("\"") + key + "\":";
  const size_t at = text.find(pat);
  if (at == std::string::npos) return false;
  const char* p = text.c_str() + at + pat.size();
  char* end = nullptr;
  const double v = strtod(p, &end);
  if (end == p) return false;
  *out = v;
  return true;
}

}  // namespace

int mdb_sim_save_checkpoint(mdb_sim_t* sim, const char* frame_path, uint64_t frame_index,
                            const char* state_path) {
  if (!sim || !frame_path || !state_path) return mdb::set_error(MDB_ERR_ARG, "null argument");
  MDB_TRY(mdb_sim_save_pframe(sim, frame_path, frame_index));
  SysState S;
  MDB_TRY(sim->eng->get_state(0, &S));
  FILE* f = fopen(state_path, "wb");
  if (!f) return mdb::set_error(MDB_ERR_IO, std::string("cannot open ") + state_path);
  fprintf(f, "{\n  \"format\": \"%s\",\n", kCheckpointFormat);
  fprintf(f, "  \"frame_index\": %llu,\n  \"n\": %lld,\n  \"steps\": %lld,\n",
          (unsigned long long)frame_index, (long long)sim->eng->n(0), (long long)S.steps);
  const struct {
    const char* k;
    double v;
  } dv[] = {{"t", sim->t},     {"Lx", S.Lx},         {"Ly", S.Ly},         {"xi", S.xi},
            {"K", S.K},        {"pA", S.pA},         {"aspect", S.aspect}, {"P_cur", S.P_cur},
            {"last_P", S.last_P}, {"fl", S.fl},      {"ce", S.ce},         {"vp", S.vp},
            {"Fp", S.Fp},      {"wallU", S.wallU},   {"p_ext", S.p_ext}};
  for (const auto& e : dv) fprintf(f, "  \"%s\": %.17g,\n", e.k, e.v);
  fprintf(f,
          "  \"clamped\": %d,\n  \"piston_active\": %d,\n  \"nph_init\": %d,\n"
          "  \"vp_init\": %d,\n  \"k_valid\": %d,\n  \"p_valid\": %d,\n  \"periodic_y\": %d\n}\n",
          S.clamped, sim->piston_active ? 1 : 0, sim->nph_init ? 1 : 0, sim->vp_init ? 1 : 0,
          sim->k_valid ? 1 : 0, sim->p_valid ? 1 : 0, sim->periodic_y);
  if (fclose(f) != 0) return mdb::set_error(MDB_ERR_IO, "failed to write the checkpoint state");
  return MDB_OK;
}

int mdb_sim_create_from_checkpoint(const mdb_config_t* cfg, const char* frame_path,
                                   uint64_t frame_index, const char* state_path,
                                   const mdb_options_t* opt, mdb_sim_t** out) {
  if (!cfg || !frame_path || !state_path || !out)
    return mdb::set_error(MDB_ERR_ARG, "null argument");
  *out = nullptr;
  FILE* f = fopen(state_path, "rb");
  if (!f) return mdb::set_error(MDB_ERR_IO, std::string("cannot open ") + state_path);
  std::string text;
  char buf[4096];
  size_t k;
  while ((k = fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, k);
  fclose(f);
  if (text.find(kCheckpointFormat) == std::string::npos)
    return mdb::set_error(MDB_ERR_IO, "not a checkpoint state file");
  Checkpoint c;
  double v;
  const struct {
    const char* k;
    double* p;
  } dk[] = {{"t", &c.t},           {"Lx", &c.Lx},         {"Ly", &c.Ly},     {"xi", &c.xi},
            {"K", &c.K},           {"pA", &c.pA},         {"aspect", &c.aspect},
            {"P_cur", &c.P_cur},   {"last_P", &c.last_P}, {"fl", &c.fl},     {"ce", &c.ce},
            {"vp", &c.vp},         {"Fp", &c.Fp},         {"wallU", &c.wallU},
            {"p_ext", &c.p_ext}};
  for (const auto& e : dk)
    if (!ck_find(text, e.k, e.p))
      return mdb::set_error(MDB_ERR_IO, std::string("checkpoint state lacks ") + e.k);
  const struct {
    const char* k;
    int* p;
  } ik[] = {{"clamped", &c.clamped},   {"piston_active", &c.piston_active},
            {"nph_init", &c.nph_init}, {"vp_init", &c.vp_init},
            {"k_valid", &c.k_valid},   {"p_valid", &c.p_valid},
            {"periodic_y", &c.periodic_y}};
  for (const auto& e : ik) {
    if (!ck_find(text, e.k, &v))
      return mdb::set_error(MDB_ERR_IO, std::string("checkpoint state lacks ") + e.k);
    *e.p = (int)v;
  }
  if (!ck_find(text, "steps", &v)) return mdb::set_error(MDB_ERR_IO, "checkpoint state lacks steps");
  c.steps = (int64_t)v;
  // the box of the checkpoint, not the configuration's initial box
  mdb_config_t cfg2 = *cfg;
  cfg2.box_w_global = c.Lx;
  cfg2.box_h_global = c.Ly;
  mdb_sim_t* sim = nullptr;
  MDB_TRY(mdb_sim_create_from_pframe(&cfg2, frame_path, frame_index, opt, &sim));
  std::unique_ptr<mdb_sim> guard(sim);
  if (c.periodic_y == 0) {
    MDB_TRY(sim->eng->rebuild_now(0));
    sim->periodic_y = 0;
    MDB_TRY(sim->eng->force(mdb::FM_INIT, false));  // pair forces and walls
  }
  SysState S;
  MDB_TRY(sim->eng->get_state(0, &S));
  S.xi = c.xi;
  S.K = c.K;
  S.pA = c.pA;
  S.aspect = c.aspect;
  S.P_cur = c.P_cur;
  S.last_P = c.last_P;
  S.fl = c.fl;
  S.ce = c.ce;
  S.vp = c.vp;
  S.Fp = c.Fp;
  S.wallU = c.wallU;
  S.p_ext = c.p_ext;
  S.clamped = c.clamped;
  S.steps = c.steps;
  MDB_TRY(sim->eng->put_state(0, S));
  sim->t = c.t;
  sim->piston_active = c.piston_active != 0;
  sim->nph_init = c.nph_init != 0;
  sim->vp_init = c.vp_init != 0;
  sim->k_valid = c.k_valid != 0;
  sim->p_valid = c.p_valid != 0;
  *out = guard.release();
  return MDB_OK;
}

int mdb_sim_get_config(mdb_sim_t* sim, mdb_config_t* out) {
  if (!sim || !out) return mdb::set_error(MDB_ERR_ARG, "null argument");
  SysState S;
  MDB_TRY(sim->eng->get_state(0, &S));
  *out = sim->cfg;
  out->box_w_global = S.Lx;
  out->box_h_global = S.Ly;
  return MDB_OK;
}

int mdb_sim_cuda_stream(mdb_sim_t* sim, void** stream) {
  if (!sim || !stream) return mdb::set_error(MDB_ERR_ARG, "null argument");
  *stream = (void*)sim->eng->stream();
  return MDB_OK;
}

int mdb_sim_schedule(mdb_sim_t* sim, mdb_schedule_t* out) {
  if (!sim || !out) return mdb::set_error(MDB_ERR_ARG, "null argument");
  *out = sim->eng->schedule();
  return MDB_OK;
}

int mdb_sim_phase_times(mdb_sim_t* sim, int32_t kind, int64_t nsteps, double* ms_out) {
  if (!sim || !ms_out || nsteps < 0) return mdb::set_error(MDB_ERR_ARG, "bad arguments");
  if (kind != MDB_JOB_NVE && kind != MDB_JOB_NVT && kind != 3)
    return mdb::set_error(MDB_ERR_ARG, "kind must be 1 (NVE), 2 (Nose-Hoover) or 3 (NPH)");
  MDB_TRY(leave_piston(sim));
  if (kind == 3) {
    if (!sim->nph_init || !sim->p_valid)
      return mdb::set_error(MDB_ERR_STATE,
                            "NPH phase times need a preceding mdb_sim_step_nph call");
    MDB_TRY(sim->eng->run_md_timed(mdb::DM_NPH, mdb::FM_NPH, true, nsteps, ms_out));
    sim->k_valid = false;
    advance_time(sim, nsteps);
    return MDB_OK;
  }
  if (kind == MDB_JOB_NVT) {
    if (!sim->k_valid) MDB_TRY(sim->eng->reduce_K());
    MDB_TRY(sim->eng->run_md_timed(mdb::DM_NH, mdb::FM_NH, true, nsteps, ms_out));
    sim->k_valid = true;
  } else {
    MDB_TRY(sim->eng->run_md_timed(mdb::DM_NVE, mdb::FM_NVE, true, nsteps, ms_out));
    sim->k_valid = false;
  }
  sim->p_valid = false;
  advance_time(sim, nsteps);
  return MDB_OK;
}

int mdb_sim_synchronize(mdb_sim_t* sim) {
  if (!sim) return mdb::set_error(MDB_ERR_ARG, "null argument");
  MDB_TRY(sim->eng->sync());
  return check_status(sim);
}

// ------------------------------------------------------------------ FIRE --

int mdb_fire_params_from_config(const mdb_config_t* cfg, mdb_fire_params_t* out) {
  if (!cfg || !out) return mdb::set_error(MDB_ERR_ARG, "null argument");
  memset(out, 0, sizeof(*out));
  out->dt_init = cfg->dt;
  out->dt_max = 5.0 * cfg->dt;
  out->alpha0 = 0.1;
  out->f_inc = 1.1;
  out->f_dec = 0.5;
  out->N_min = 5;
  return MDB_OK;
}

namespace {

// Energy samples of one FIRE run (MinimizeResult::energy_steps/_trace).
struct Trace {
  std::vector<int32_t> steps;
  std::vector<double> u;
  void add(int32_t s, double v) {
    steps.push_back(s);
    u.push_back(v);
  }
};

int obs_energies(Engine& eng, std::vector<SysState>& S) {
  MDB_TRY(eng.force(mdb::FM_OBS, true));
  return eng.get_states(S);
}

void copy_trace(const Trace& tr, int32_t* es, double* et, int64_t cap) {
  for (size_t k = 0; k < tr.steps.size() && (int64_t)k < cap; ++k) {
    if (es) es[k] = tr.steps[k];
    if (et) et[k] = tr.u[k];
  }
}

}  // namespace

int mdb_fire_minimize(const mdb_config_t* cfg, const mdb_particle_t* frame, int64_t n,
                      double force_tol, int32_t max_steps, const mdb_fire_params_t* params,
                      const mdb_options_t* opt, mdb_particle_t* frame_out,
                      mdb_minimize_result_t* result, int32_t* energy_steps,
                      double* energy_trace, int64_t trace_cap) {
  if (!cfg || !frame || !params || !result || n <= 0)
    return mdb::set_error(MDB_ERR_ARG, "bad arguments");
  if (max_steps <= 0) return mdb::set_error(MDB_ERR_ARG, "EnergyMinimizer: max_steps must be positive.");
  mdb_options_t o = opts_or_default(opt);
  Engine eng(o);
  SystemSpec spec;
  spec.cfg = *cfg;
  spec.frame.assign(frame, frame + n);
  spec.kind = mdb::K_FIRE;
  spec.fire = *params;
  spec.tol = force_tol;
  spec.max_steps = max_steps;
  spec.fire_prepare = true;
  MDB_TRY(eng.add_system(std::move(spec)));
  MDB_TRY(eng.build());
  Trace tr;
  std::vector<SysState> S;
  MDB_TRY(obs_energies(eng, S));
  tr.add(0, S[0].U);
  int64_t done = 0;
  bool converged = false;
  int32_t steps = max_steps;
  while (done < max_steps) {
    const int64_t to_sample = 1000 - (done % 1000);
    const int64_t chunk = std::min<int64_t>(to_sample, (int64_t)max_steps - done);
    MDB_TRY(eng.run_fire(chunk));
    done += chunk;
    MDB_TRY(eng.get_states(S));
    if (S[0].f_conv) {
      converged = true;
      steps = S[0].f_conv_step;
      MDB_TRY(obs_energies(eng, S));
      tr.add(steps + 1, S[0].U);
      break;
    }
    if (done % 1000 == 0) {
      MDB_TRY(obs_energies(eng, S));
      tr.add((int32_t)done, S[0].U);
    }
  }
  if (!converged && (tr.steps.empty() || tr.steps.back() != max_steps)) {
    MDB_TRY(obs_energies(eng, S));
    tr.add(max_steps, S[0].U);
  }
  MDB_TRY(obs_energies(eng, S));
  memset(result, 0, sizeof(*result));
  result->steps = steps;
  result->converged = converged ? 1 : 0;
  result->max_force = S[0].f_maxf;
  result->potential_energy = S[0].U;
  result->n_energy_samples = (int64_t)tr.steps.size();
  result->nonfinite = S[0].nonfinite;
  copy_trace(tr, energy_steps, energy_trace, trace_cap);
  if (frame_out) MDB_TRY(eng.get_frame(0, frame_out));
  return MDB_OK;
}

// ------------------------------------------------------------- batches --

}  // extern "C"

struct mdb_batch {
  mdb_options_t opt;
  std::unique_ptr<Engine> eng;
  std::vector<SystemSpec> pending;
  std::vector<Trace> traces;
  std::vector<int32_t> recorded_done;  // FIRE: final sample recorded; MD: segment finished
  std::vector<int32_t> max_steps;      // FIRE: iteration cap; MD: segment length
  int32_t kind = -1;                   // K_FIRE, K_NVE or K_NVT, shared by every system
  int64_t iter = 0;                    // iterations / steps issued so far
  bool built = false;
};

namespace {

int batch_build(mdb_batch_t* b) {
  if (b->built) return MDB_OK;
  if (b->pending.empty()) return mdb::set_error(MDB_ERR_STATE, "batch has no systems");
  b->eng.reset(new Engine(b->opt));
  const size_t ns = b->pending.size();
  for (auto& s : b->pending) MDB_TRY(b->eng->add_system(std::move(s)));
  b->pending.clear();
  MDB_TRY(b->eng->build());
  b->traces.assign(ns, Trace());
  b->recorded_done.assign(ns, 0);
  if (b->kind == mdb::K_FIRE) {
    std::vector<SysState> S;
    MDB_TRY(obs_energies(*b->eng, S));
    for (size_t s = 0; s < ns; ++s) b->traces[s].add(0, S[s].U);
  } else {
    // what the MDSimulation constructor leaves: forces, and K for the first
    // Nose-Hoover half step
    MDB_TRY(b->eng->force(mdb::FM_INIT, true));
    if (b->kind == mdb::K_NVT) MDB_TRY(b->eng->reduce_K());
  }
  b->built = true;
  return MDB_OK;
}

bool fire_finished(const SysState& S, int32_t max_steps) {
  return S.f_conv != 0 || S.f_step >= max_steps || S.err != 0;
}

int32_t batch_cap(const mdb_batch_t* b) {
  int32_t cap = 0;
  for (int32_t m : b->max_steps) cap = m > cap ? m : cap;
  return cap;
}

// Length of the next chunk: chunks end on multiples of 1000 iterations (the
// energy samples of minimize_frame for FIRE; for MD, finished segments are
// noticed at least that often).
int64_t batch_next_chunk(const mdb_batch_t* b, int64_t left) {
  const int64_t cap = batch_cap(b);
  int64_t chunk = std::min<int64_t>(left, cap - b->iter);
  chunk = std::min<int64_t>(chunk, 1000 - (b->iter % 1000));
  return chunk;
}

// Issues one chunk on the batch's stream without waiting for it.
int batch_issue(mdb_batch_t* b, int64_t chunk) {
  if (chunk <= 0) return MDB_OK;
  if (b->kind == mdb::K_FIRE) {
    MDB_TRY(b->eng->run_fire(chunk));
  } else if (b->kind == mdb::K_NVT) {
    MDB_TRY(b->eng->run_md(mdb::DM_NH, mdb::FM_NH, true, chunk));
  } else {
    MDB_TRY(b->eng->run_md(mdb::DM_NVE, mdb::FM_NVE, true, chunk));
  }
  b->iter += chunk;
  return MDB_OK;
}

// Records finished systems (and FIRE energy samples) after a chunk that ended
// at iteration b->iter; waits for the batch's stream.
int batch_harvest(mdb_batch_t* b) {
  std::vector<SysState> S;
  MDB_TRY(b->eng->get_states(S));
  const size_t ns = S.size();
  if (b->kind != mdb::K_FIRE) {
    for (size_t s = 0; s < ns; ++s)
      if (S[s].done || S[s].err) b->recorded_done[s] = 1;
    return MDB_OK;
  }
  bool need_u = false;
  for (size_t s = 0; s < ns; ++s) {
    if (b->recorded_done[s]) continue;
    if (S[s].f_conv || S[s].f_step >= b->max_steps[s] || (b->iter % 1000 == 0)) need_u = true;
  }
  if (!need_u) return MDB_OK;
  std::vector<SysState> U;
  MDB_TRY(obs_energies(*b->eng, U));
  for (size_t s = 0; s < ns; ++s) {
    if (b->recorded_done[s]) continue;
    Trace& tr = b->traces[s];
    if (S[s].f_conv) {
      tr.add(S[s].f_conv_step + 1, U[s].U);
      b->recorded_done[s] = 1;
    } else if (S[s].f_step >= b->max_steps[s]) {
      if (tr.steps.empty() || tr.steps.back() != b->max_steps[s]) tr.add(b->max_steps[s], U[s].U);
      b->recorded_done[s] = 1;
    } else if (b->iter % 1000 == 0) {
      tr.add((int32_t)b->iter, U[s].U);
    }
  }
  return MDB_OK;
}

bool batch_all_done(const mdb_batch_t* b) {
  for (int32_t x : b->recorded_done)
    if (!x) return false;
  return true;
}

int batch_add(mdb_batch_t* b, SystemSpec&& spec, int32_t kind, int32_t cap, int32_t* sys_id) {
  if (b->built) return mdb::set_error(MDB_ERR_STATE, "systems can only be added before the first run");
  if (b->kind >= 0 && b->kind != kind)
    return mdb::set_error(MDB_ERR_STATE, "every system of a batch must be of the same job kind");
  b->kind = kind;
  b->pending.push_back(std::move(spec));
  b->max_steps.push_back(cap);
  if (sys_id) *sys_id = (int32_t)b->pending.size() - 1;
  return MDB_OK;
}

}  // namespace

extern "C" {

int mdb_batch_create(const mdb_options_t* opt, mdb_batch_t** out) {
  if (!out) return mdb::set_error(MDB_ERR_ARG, "null argument");
  mdb_batch_t* b = new (std::nothrow) mdb_batch();
  if (!b) return mdb::set_error(MDB_ERR_CAPACITY, "out of host memory");
  b->opt = opts_or_default(opt);
  *out = b;
  return MDB_OK;
}

int mdb_batch_destroy(mdb_batch_t* b) {
  delete b;
  return MDB_OK;
}

int mdb_batch_add_fire(mdb_batch_t* b, const mdb_config_t* cfg, const mdb_particle_t* frame,
                       int64_t n, double force_tol, int32_t max_steps,
                       const mdb_fire_params_t* params, int32_t* sys_id) {
  if (!b || !cfg || !frame || !params || n <= 0) return mdb::set_error(MDB_ERR_ARG, "bad arguments");
  if (max_steps <= 0) return mdb::set_error(MDB_ERR_ARG, "max_steps must be positive");
  SystemSpec spec;
  spec.cfg = *cfg;
  spec.frame.assign(frame, frame + n);
  spec.kind = mdb::K_FIRE;
  spec.fire = *params;
  spec.tol = force_tol;
  spec.max_steps = max_steps;
  spec.fire_prepare = true;
  return batch_add(b, std::move(spec), mdb::K_FIRE, max_steps, sys_id);
}

int mdb_batch_add_md(mdb_batch_t* b, const mdb_config_t* cfg, const mdb_particle_t* frame,
                     int64_t n, int32_t kind, int64_t nsteps, int32_t* sys_id) {
  if (!b || !cfg || !frame || n <= 0) return mdb::set_error(MDB_ERR_ARG, "bad arguments");
  if (kind != MDB_JOB_NVE && kind != MDB_JOB_NVT)
    return mdb::set_error(MDB_ERR_ARG, "kind must be MDB_JOB_NVE or MDB_JOB_NVT");
  if (nsteps <= 0 || nsteps > INT32_MAX) return mdb::set_error(MDB_ERR_ARG, "nsteps out of range");
  SystemSpec spec;
  spec.cfg = *cfg;
  spec.cfg.n_particles_global = (int32_t)n;  // g = 2N - 2 counts this system
  spec.frame.assign(frame, frame + n);
  const int32_t k = kind == MDB_JOB_NVT ? mdb::K_NVT : mdb::K_NVE;
  spec.kind = k;
  spec.target_steps = nsteps;
  return batch_add(b, std::move(spec), k, (int32_t)nsteps, sys_id);
}

int mdb_batch_run(mdb_batch_t* b, int64_t iterations) {
  if (!b) return mdb::set_error(MDB_ERR_ARG, "null argument");
  MDB_TRY(batch_build(b));
  const int32_t cap = batch_cap(b);
  int64_t left = iterations < 0 ? (int64_t)cap - b->iter : iterations;
  while (left > 0 && b->iter < cap) {
    const int64_t chunk = batch_next_chunk(b, left);
    MDB_TRY(batch_issue(b, chunk));
    left -= chunk;
    MDB_TRY(batch_harvest(b));
    if (batch_all_done(b)) break;
  }
  return MDB_OK;
}

int mdb_batch_issue(mdb_batch_t* b, int64_t iterations, int64_t* issued) {
  if (!b) return mdb::set_error(MDB_ERR_ARG, "null argument");
  if (issued) *issued = 0;
  MDB_TRY(batch_build(b));
  const int64_t left = iterations < 0 ? (int64_t)batch_cap(b) - b->iter : iterations;
  if (left <= 0 || batch_all_done(b)) return MDB_OK;
  const int64_t chunk = batch_next_chunk(b, left);
  MDB_TRY(batch_issue(b, chunk));
  if (issued) *issued = chunk;
  return MDB_OK;
}

int mdb_batch_query(mdb_batch_t* b, int32_t* idle) {
  if (!b || !idle) return mdb::set_error(MDB_ERR_ARG, "null argument");
  if (!b->built) {
    *idle = 1;
    return MDB_OK;
  }
  bool v = false;
  MDB_TRY(b->eng->idle(&v));
  *idle = v ? 1 : 0;
  return MDB_OK;
}

int mdb_batch_collect(mdb_batch_t* b) {
  if (!b) return mdb::set_error(MDB_ERR_ARG, "null argument");
  MDB_TRY(batch_build(b));
  return batch_harvest(b);
}

int mdb_batch_energies_all(mdb_batch_t* b, double* K, double* U, double* xi, int32_t n) {
  if (!b) return mdb::set_error(MDB_ERR_ARG, "null argument");
  MDB_TRY(batch_build(b));
  if (n != b->eng->nsys()) return mdb::set_error(MDB_ERR_CAPACITY, "n must equal the number of systems");
  std::vector<SysState> S;
  MDB_TRY(obs_energies(*b->eng, S));
  for (int32_t s = 0; s < n; ++s) {
    if (K) K[s] = 0.5 * S[s].kin;
    if (U) U[s] = S[s].U;
    if (xi) xi[s] = S[s].xi;
  }
  return MDB_OK;
}

int mdb_batch_energies(mdb_batch_t* b, int32_t sys_id, double* K, double* U, double* xi) {
  if (!b) return mdb::set_error(MDB_ERR_ARG, "null argument");
  MDB_TRY(batch_build(b));
  if (sys_id < 0 || sys_id >= b->eng->nsys()) return mdb::set_error(MDB_ERR_ARG, "bad system id");
  std::vector<SysState> S;
  MDB_TRY(obs_energies(*b->eng, S));
  if (K) *K = 0.5 * S[sys_id].kin;
  if (U) *U = S[sys_id].U;
  if (xi) *xi = S[sys_id].xi;
  if (S[sys_id].nonfinite) return mdb::set_error(MDB_ERR_NONFINITE, "non-finite state");
  return MDB_OK;
}

int mdb_batch_partial_U_lambda_all(mdb_batch_t* b, double epsilon_lambda, double* out,
                                   int32_t n) {
  if (!b || !out) return mdb::set_error(MDB_ERR_ARG, "null argument");
  MDB_TRY(batch_build(b));
  if (n != b->eng->nsys()) return mdb::set_error(MDB_ERR_CAPACITY, "n must equal the number of systems");
  std::vector<SysState> S;
  MDB_TRY(obs_energies(*b->eng, S));
  for (int32_t s = 0; s < n; ++s) out[s] = -epsilon_lambda * S[s].Wani;
  return MDB_OK;
}

int mdb_batch_done_flags(mdb_batch_t* b, int32_t* done, int32_t n) {
  if (!b || !done) return mdb::set_error(MDB_ERR_ARG, "null argument");
  MDB_TRY(batch_build(b));
  if (n != (int32_t)b->recorded_done.size())
    return mdb::set_error(MDB_ERR_CAPACITY, "n must equal the number of systems");
  for (int32_t s = 0; s < n; ++s) done[s] = b->recorded_done[s] ? 1 : 0;
  return MDB_OK;
}

int mdb_batch_schedule(mdb_batch_t* b, mdb_schedule_t* out) {
  if (!b || !out) return mdb::set_error(MDB_ERR_ARG, "null argument");
  memset(out, 0, sizeof(*out));
  if (b->built) *out = b->eng->schedule();
  return MDB_OK;
}

int mdb_batch_device_bytes(mdb_batch_t* b, int64_t* bytes) {
  if (!b || !bytes) return mdb::set_error(MDB_ERR_ARG, "null argument");
  *bytes = b->built ? b->eng->device_bytes() : 0;
  return MDB_OK;
}

int mdb_batch_progress(mdb_batch_t* b, int32_t* n_systems, int32_t* n_done) {
  if (!b) return mdb::set_error(MDB_ERR_ARG, "null argument");
  const int32_t ns = b->built ? (int32_t)b->recorded_done.size() : (int32_t)b->pending.size();
  int32_t d = 0;
  if (b->built)
    for (int32_t x : b->recorded_done) d += x ? 1 : 0;
  if (n_systems) *n_systems = ns;
  if (n_done) *n_done = d;
  return MDB_OK;
}

int mdb_batch_system_info(mdb_batch_t* b, int32_t sys_id, int64_t* n, int32_t* done,
                          int64_t* steps) {
  if (!b) return mdb::set_error(MDB_ERR_ARG, "null argument");
  MDB_TRY(batch_build(b));
  if (sys_id < 0 || sys_id >= b->eng->nsys()) return mdb::set_error(MDB_ERR_ARG, "bad system id");
  SysState S;
  MDB_TRY(b->eng->get_state(sys_id, &S));
  if (n) *n = b->eng->n(sys_id);
  if (b->kind == mdb::K_FIRE) {
    if (done) *done = fire_finished(S, b->max_steps[sys_id]) ? 1 : 0;
    if (steps) *steps = S.f_conv ? S.f_conv_step : S.f_step;
  } else {
    if (done) *done = (S.done || S.err) ? 1 : 0;
    if (steps) *steps = S.steps;
  }
  return MDB_OK;
}

int mdb_batch_system_stats(mdb_batch_t* b, int32_t sys_id, int64_t* rebuilds,
                           int32_t* list_overflow) {
  if (!b) return mdb::set_error(MDB_ERR_ARG, "null argument");
  MDB_TRY(batch_build(b));
  if (sys_id < 0 || sys_id >= b->eng->nsys()) return mdb::set_error(MDB_ERR_ARG, "bad system id");
  SysState S;
  MDB_TRY(b->eng->get_state(sys_id, &S));
  if (rebuilds) *rebuilds = S.rebuilds;
  if (list_overflow) *list_overflow = S.nl_overflow;
  return MDB_OK;
}

int mdb_batch_get_frame(mdb_batch_t* b, int32_t sys_id, mdb_particle_t* out, int64_t n) {
  if (!b || !out) return mdb::set_error(MDB_ERR_ARG, "null argument");
  MDB_TRY(batch_build(b));
  if (sys_id < 0 || sys_id >= b->eng->nsys()) return mdb::set_error(MDB_ERR_ARG, "bad system id");
  if (n != b->eng->n(sys_id)) return mdb::set_error(MDB_ERR_CAPACITY, "n must equal the system size");
  return b->eng->get_frame(sys_id, out);
}

int mdb_batch_get_fire_result(mdb_batch_t* b, int32_t sys_id, mdb_minimize_result_t* result,
                              int32_t* energy_steps, double* energy_trace, int64_t trace_cap) {
  if (!b || !result) return mdb::set_error(MDB_ERR_ARG, "null argument");
  MDB_TRY(batch_build(b));
  if (sys_id < 0 || sys_id >= b->eng->nsys()) return mdb::set_error(MDB_ERR_ARG, "bad system id");
  std::vector<SysState> U;
  MDB_TRY(obs_energies(*b->eng, U));
  const SysState& S = U[sys_id];
  memset(result, 0, sizeof(*result));
  result->converged = S.f_conv ? 1 : 0;
  result->steps = S.f_conv ? S.f_conv_step : b->max_steps[sys_id];
  result->max_force = S.f_maxf;
  result->potential_energy = S.U;
  result->n_energy_samples = (int64_t)b->traces[sys_id].steps.size();
  result->nonfinite = S.nonfinite;
  copy_trace(b->traces[sys_id], energy_steps, energy_trace, trace_cap);
  return MDB_OK;
}

int mdb_batch_cuda_stream(mdb_batch_t* b, void** stream) {
  if (!b || !stream) return mdb::set_error(MDB_ERR_ARG, "null argument");
  MDB_TRY(batch_build(b));
  *stream = (void*)b->eng->stream();
  return MDB_OK;
}

// ----------------------------------------------------- single-call kernels --

int mdb_compute_forces(const mdb_config_t* cfg, const mdb_particle_t* frame, int64_t n,
                       double Lx, double Ly, int32_t periodic_y, const mdb_options_t* opt,
                       double* acc_out, double* U_out, double* W_out) {
  if (!cfg || !frame || n <= 0) return mdb::set_error(MDB_ERR_ARG, "bad arguments");
  mdb_options_t o = opts_or_default(opt);
  Engine eng(o);
  SystemSpec spec;
  spec.cfg = *cfg;
  spec.cfg.box_w_global = Lx;
  spec.cfg.box_h_global = Ly;
  spec.cfg.k_piston = 0.0;  // pair forces only
  spec.frame.assign(frame, frame + n);
  MDB_TRY(eng.add_system(std::move(spec)));
  MDB_TRY(eng.build());
  const bool py = periodic_y != 0;
  if (!py) MDB_TRY(eng.rebuild_now(0));
  MDB_TRY(eng.force(mdb::FM_INIT, py));
  if (acc_out) {
    std::vector<mdb_particle_t> f((size_t)n);
    MDB_TRY(eng.get_frame(0, f.data()));
    for (int64_t i = 0; i < n; ++i) {
      acc_out[2 * i] = f[i].acc.x;
      acc_out[2 * i + 1] = f[i].acc.y;
    }
  }
  if (U_out || W_out) {
    MDB_TRY(eng.force(mdb::FM_OBS, py));
    SysState S;
    MDB_TRY(eng.get_state(0, &S));
    if (U_out) *U_out = S.U;
    if (W_out) *W_out = S.Wv;
  }
  return eng.sync();
}

int mdb_cell_build(const double* pos, int64_t n, double Lx, double Ly, double cell_min,
                   int32_t device, int32_t* cell_out, int32_t* perm_out, int32_t* ncx_out,
                   int32_t* ncy_out) {
  if (!pos || n <= 0 || !(cell_min > 0.0)) return mdb::set_error(MDB_ERR_ARG, "bad arguments");
  mdb_options_t o;
  mdb_options_default(&o);
  o.device = device;
  o.skin = cell_min * 0.5;
  Engine eng(o);
  SystemSpec spec;
  mdb_config_default(&spec.cfg);
  spec.cfg.box_w_global = Lx;
  spec.cfg.box_h_global = Ly;
  spec.cfg.SIGMA_AA = spec.cfg.SIGMA_BB = spec.cfg.SIGMA_AB = 1.0;
  spec.cfg.cutoff = cell_min * 0.5;  // r_cell = cutoff * sigma_max + skin = cell_min
  spec.cfg.barostat_height_max_ratio = 1.0;
  spec.frame.assign((size_t)n, mdb_particle_t{});
  for (int64_t i = 0; i < n; ++i) {
    spec.frame[i].pos.x = pos[2 * i];
    spec.frame[i].pos.y = pos[2 * i + 1];
  }
  MDB_TRY(eng.add_system(std::move(spec)));
  MDB_TRY(eng.build());
  std::vector<int32_t> orig((size_t)n), cell((size_t)n);
  MDB_TRY(eng.debug_cells(0, orig.data(), cell.data()));
  for (int64_t k = 0; k < n; ++k) {
    if (perm_out) perm_out[k] = orig[k];
    if (cell_out) cell_out[orig[k]] = cell[k];
  }
  SysState S;
  MDB_TRY(eng.get_state(0, &S));
  if (ncx_out) *ncx_out = S.ncx;
  if (ncy_out) *ncy_out = S.ncy;
  return MDB_OK;
}

}  // extern "C"
