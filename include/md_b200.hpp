// md_b200.hpp — C++ drop-in for the MD stepping path of MD_Simulation_CUDA.
//
// Header-only classes with the reference's names and signatures, implemented
// over the C ABI of libmdb200.so (mdb200.h). A caller of the reference's
// MDSimulation / EnergyMinimizer / MDConfigManager switches by including this
// header instead of md_env.hpp, md_energy_minimizer.hpp and md_config.hpp and
// linking -lmdb200 (no MPI, no RAFT):
//
//   reference                                    this header
//   struct Particle (md_particle.hpp:31-38)      Particle (same 64-byte layout)
//   struct MDConfig (md_config.hpp:14-75)        MDConfig (same fields/defaults)
//   class MDConfigManager (md_config.hpp:82-111) MDConfigManager
//   class MDSimulation (md_env.hpp:51-263)       MDSimulation (the stepping path)
//   struct FireParams / MinimizeResult /         FireParams / MinimizeResult /
//   class EnergyMinimizer                        EnergyMinimizer
//     (md_energy_minimizer.hpp:11-97)
//
// The MPI_Comm argument of the reference constructors is accepted and ignored
// (every system lives on one GPU). Errors: where the reference exits or calls
// MPI_Abort, these classes throw mdb200::Error (a std::runtime_error) with the
// library's message. Only the stepping path is provided: members of the
// reference classes outside it (plotting, triangulation, interface analysis,
// ABP, profiles) are not declared, so code that calls them fails to compile
// rather than silently doing nothing.
//
// Define MDB200_NO_GLOBAL_NAMES to keep the names inside namespace mdb200.
#pragma once

#include <vector_types.h>

#include <cstddef>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "mdb200.h"

namespace mdb200 {

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& what) : std::runtime_error(what), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

inline void check(int rc, const char* where) {
  if (rc == MDB_OK) return;
  char msg[1024];
  mdb_last_error(msg, sizeof msg);
  throw Error(rc, std::string(where) + ": " + msg);
}

// Particle (include/md_particle.hpp:31-38), layout-identical to mdb_particle_t.
struct Particle {
  double2 pos;
  double2 vel;
  double2 acc;
  int type;
  double theta;
};
static_assert(sizeof(Particle) == sizeof(mdb_particle_t), "Particle must be 64 bytes");
static_assert(offsetof(Particle, type) == offsetof(mdb_particle_t, type), "type offset");
static_assert(offsetof(Particle, theta) == offsetof(mdb_particle_t, theta), "theta offset");

inline const mdb_particle_t* as_c(const Particle* p) {
  return reinterpret_cast<const mdb_particle_t*>(p);
}
inline mdb_particle_t* as_c(Particle* p) { return reinterpret_cast<mdb_particle_t*>(p); }

// Numeric MDConfig fields in declaration order: X(type, name).
#define MDB200_CONFIG_NUMERIC(X)                                                              \
  X(int, n_particles_global) X(int, n_particles_type0) X(double, box_w_global)                \
  X(double, box_h_global) X(double, T_init) X(double, T_target) X(double, SIGMA_AA)           \
  X(double, SIGMA_BB) X(double, SIGMA_AB) X(double, EPSILON_AA) X(double, EPSILON_BB)         \
  X(double, EPSILON_AB) X(double, MASS_A) X(double, MASS_B) X(double, devide_p) X(double, dt) \
  X(double, Q) X(double, save_dt_interval) X(double, cutoff) X(int, THREADS_PER_BLOCK)        \
  X(int, rank_size) X(double, mu) X(double, v0) X(double, D_r) X(double, D_theta)             \
  X(double, barostat_mass) X(double, k_piston) X(double, barostat_area_rate_init)             \
  X(double, barostat_height_min_ratio) X(double, barostat_height_max_ratio)                   \
  X(double, P_target) X(int, pressure_target_auto_steps) X(int, pressure_eval_interval_steps) \
  X(int, pressure_window_samples) X(double, pressure_tolerance_rel)                           \
  X(int, pressure_stable_required_windows) X(int, nph_warmup_min_steps)                       \
  X(int, nph_warmup_max_steps) X(int, nph_steps) X(int, rank_idx) X(int, n_local)             \
  X(int, n_halo_left) X(int, n_halo_right) X(int, n_cap) X(int, halo_left_cap)                \
  X(int, halo_right_cap) X(int, left_rank) X(int, right_rank) X(double, x_min)                \
  X(double, x_max)
#define MDB200_CONFIG_STRINGS(X) X(run_name) X(load_name) X(pressure_target_mode)

// MDConfig (include/md_config.hpp:14-75): same field names; a default-built
// MDConfig holds the reference's defaults.
struct MDConfig {
#define MDB200_DECL_NUM(T, name) T name{};
#define MDB200_DECL_STR(name) std::string name;
  MDB200_CONFIG_NUMERIC(MDB200_DECL_NUM)
  MDB200_CONFIG_STRINGS(MDB200_DECL_STR)
#undef MDB200_DECL_NUM
#undef MDB200_DECL_STR

  MDConfig() {
    mdb_config_t c;
    check(mdb_config_default(&c), "mdb_config_default");
    from_c(c);
  }
  explicit MDConfig(const mdb_config_t& c) { from_c(c); }

  void from_c(const mdb_config_t& c) {
#define MDB200_FROM_NUM(T, name) name = static_cast<T>(c.name);
#define MDB200_FROM_STR(name) name = std::string(c.name);
    MDB200_CONFIG_NUMERIC(MDB200_FROM_NUM)
    MDB200_CONFIG_STRINGS(MDB200_FROM_STR)
#undef MDB200_FROM_NUM
#undef MDB200_FROM_STR
  }

  mdb_config_t to_c() const {
    mdb_config_t c;
    std::memset(&c, 0, sizeof c);
#define MDB200_TO_NUM(T, name) c.name = name;
#define MDB200_TO_STR(name)                                      \
  if (name.size() >= sizeof c.name)                              \
    throw Error(MDB_ERR_CONFIG, "MDConfig." #name " is too long"); \
  std::memcpy(c.name, name.c_str(), name.size() + 1);
    MDB200_CONFIG_NUMERIC(MDB200_TO_NUM)
    MDB200_CONFIG_STRINGS(MDB200_TO_STR)
#undef MDB200_TO_NUM
#undef MDB200_TO_STR
    return c;
  }
};

// MDConfigOverride (include/md_config.hpp:77-80).
struct MDConfigOverride {
  std::string key;
  std::string value;
};

// MDConfigManager (include/md_config.hpp:82-111; src/md_config.cpp).
class MDConfigManager {
 public:
  MDConfigManager() = default;
  MDConfigManager(MDConfig c) : config(std::move(c)) {}

  MDConfig config;

  static MDConfigManager config_from_json(const std::string& filepath) {
    mdb_config_t c;
    check(mdb_config_from_json_file(filepath.c_str(), &c), "config_from_json");
    return MDConfigManager(MDConfig(c));
  }

  void config_to_json(const std::string& filepath) {
    const std::string text = dump(4);
    FILE* f = std::fopen(filepath.c_str(), "wb");
    if (!f) throw Error(MDB_ERR_IO, "config_to_json: cannot open " + filepath);
    const size_t k = std::fwrite(text.data(), 1, text.size(), f);
    std::fclose(f);
    if (k != text.size()) throw Error(MDB_ERR_IO, "config_to_json: short write to " + filepath);
  }

  std::string serialize() const { return dump(-1); }

  void deserialize(const std::string& data) {
    mdb_config_t c;
    check(mdb_config_from_json(data.c_str(), &c), "deserialize");
    config.from_c(c);
  }

  bool apply_override(const std::string& key, const std::string& value) {
    mdb_config_t c = config.to_c();
    const int rc = mdb_config_apply_override(&c, key.c_str(), value.c_str());
    if (rc != MDB_OK) return false;
    config.from_c(c);
    return true;
  }

  void apply_overrides(const std::vector<MDConfigOverride>& overrides) {
    for (const auto& o : overrides)
      if (!apply_override(o.key, o.value))
        throw Error(MDB_ERR_CONFIG, "unknown or invalid override " + o.key + "=" + o.value);
  }

  static bool parse_override_argument(const std::string& argument, std::string& out_key,
                                      std::string& out_value) {
    std::vector<char> k(argument.size() + 1), v(argument.size() + 1);
    if (mdb_parse_override_argument(argument.c_str(), k.data(), k.size(), v.data(), v.size()) !=
        MDB_OK)
      return false;
    out_key = k.data();
    out_value = v.data();
    return true;
  }

 private:
  std::string dump(int indent) const {
    const mdb_config_t c = config.to_c();
    size_t need = 0;
    mdb_config_to_json(&c, indent, nullptr, 0, &need);
    std::vector<char> buf(need + 1);
    check(mdb_config_to_json(&c, indent, buf.data(), buf.size(), &need), "serialize");
    return std::string(buf.data(), need);
  }
};

// Engine knobs with no MDConfig counterpart (device, skin, graphs, lists).
inline mdb_options_t default_options() {
  mdb_options_t o;
  mdb_options_default(&o);
  return o;
}

// MDSimulation (include/md_env.hpp:51-263): the stepping path.
class MDSimulation {
 public:
  explicit MDSimulation(MDConfigManager config_manager,
                        const mdb_options_t& opt = default_options())
      : cfg_manager(std::move(config_manager)) {
    const mdb_config_t c = cfg_manager.config.to_c();
    check(mdb_sim_create(&c, nullptr, c.n_particles_global, &opt, &sim_), "MDSimulation");
  }
  // MDSimulation(MDConfigManager, MPI_Comm) (src/md_env.cu:21-79).
  template <class Comm>
  MDSimulation(MDConfigManager config_manager, Comm /*ignored*/)
      : MDSimulation(std::move(config_manager)) {}
  // MDSimulation(MDConfigManager, MPI_Comm, file, step) (src/md_env.cu:81-164).
  template <class Comm>
  MDSimulation(MDConfigManager config_manager, Comm /*ignored*/, const std::string& filename,
               int step, const mdb_options_t& opt = default_options())
      : cfg_manager(std::move(config_manager)) {
    const mdb_config_t c = cfg_manager.config.to_c();
    check(mdb_sim_create_from_pframe(&c, filename.c_str(), (uint64_t)step, &opt, &sim_),
          "MDSimulation(file)");
  }
  // Restart from a checkpoint (frame `step` of `filename` + its state file).
  template <class Comm>
  MDSimulation(MDConfigManager config_manager, Comm /*ignored*/, const std::string& filename,
               int step, const std::string& state_file,
               const mdb_options_t& opt = default_options())
      : cfg_manager(std::move(config_manager)) {
    const mdb_config_t c = cfg_manager.config.to_c();
    check(mdb_sim_create_from_checkpoint(&c, filename.c_str(), (uint64_t)step,
                                         state_file.c_str(), &opt, &sim_),
          "MDSimulation(checkpoint)");
  }
  // A frame given directly (what the ctor-from-file does after reading it).
  MDSimulation(MDConfigManager config_manager, const std::vector<Particle>& frame,
               const mdb_options_t& opt = default_options())
      : cfg_manager(std::move(config_manager)) {
    const mdb_config_t c = cfg_manager.config.to_c();
    check(mdb_sim_create(&c, as_c(frame.data()), (int64_t)frame.size(), &opt, &sim_),
          "MDSimulation(frame)");
  }
  ~MDSimulation() {
    if (sim_) mdb_sim_destroy(sim_);
  }
  MDSimulation(const MDSimulation&) = delete;
  MDSimulation& operator=(const MDSimulation&) = delete;

  void step_single_NVE() { check(mdb_sim_step_nve(sim_, 1), "step_single_NVE"); }
  void step_single() { step_single_NVE(); }
  void step_single_nose_hoover(bool do_middle_wrap = false) {
    check(mdb_sim_step_nose_hoover(sim_, 1, do_middle_wrap ? 1 : 0), "step_single_nose_hoover");
  }
  void step_single_NPH(double pressure_ext) {
    check(mdb_sim_step_nph(sim_, pressure_ext, 1), "step_single_NPH");
  }
  void step_single_NPH_piston(double pressure_ext) {
    check(mdb_sim_step_nph_piston(sim_, pressure_ext, 1), "step_single_NPH_piston");
  }
  // Several steps in one call (captured step chunks; no host round trip).
  void step_NVE(int64_t n) { check(mdb_sim_step_nve(sim_, n), "step_NVE"); }
  void step_nose_hoover(int64_t n) {
    check(mdb_sim_step_nose_hoover(sim_, n, 0), "step_nose_hoover");
  }
  void step_NPH(double p, int64_t n) { check(mdb_sim_step_nph(sim_, p, n), "step_NPH"); }
  void step_NPH_piston(double p, int64_t n) {
    check(mdb_sim_step_nph_piston(sim_, p, n), "step_NPH_piston");
  }

  double cal_total_K() { return scalar(mdb_sim_total_K, "cal_total_K"); }
  double cal_total_U() { return scalar(mdb_sim_total_U, "cal_total_U"); }
  // get_N_profile / get_density_profile / get_pressure_profile
  // (src/md_env.cu:3821-4104), world size 1
  std::vector<int> get_N_profile(int n_bins) {
    std::vector<int> out((size_t)(n_bins > 0 ? 2 * n_bins : 0));
    check(mdb_sim_n_profile(sim_, n_bins, out.data()), "get_N_profile");
    return out;
  }
  std::vector<double> get_density_profile(int n_bins) {
    std::vector<double> out((size_t)(n_bins > 0 ? n_bins : 0));
    check(mdb_sim_density_profile(sim_, n_bins, out.data()), "get_density_profile");
    return out;
  }
  std::vector<double> get_pressure_profile(int n_bins) {
    std::vector<double> out((size_t)(n_bins > 0 ? 3 * n_bins : 0));
    check(mdb_sim_pressure_profile(sim_, n_bins, out.data()), "get_pressure_profile");
    return out;
  }
  // cal_partial_U_lambda (src/md_env.cu:2362-2406)
  double cal_partial_U_lambda(double epsilon_lambda) {
    double v = 0.0;
    check(mdb_sim_partial_U_lambda(sim_, epsilon_lambda, &v), "cal_partial_U_lambda");
    return v;
  }
  double cal_instant_pressure() {
    return scalar(mdb_sim_instant_pressure, "cal_instant_pressure");
  }

  double get_Lx() const { return obs().Lx; }
  double get_Ly() const { return obs().Ly; }
  double get_last_instant_pressure() const { return obs().last_instant_pressure; }
  double get_nph_area_rate() const { return obs().nph_area_rate; }
  double get_nph_piston_velocity() const { return obs().nph_piston_velocity; }
  double get_nph_piston_force() const { return obs().nph_piston_force; }
  double get_t() const { return obs().t; }
  double get_xi() const { return obs().xi; }

  // sample_collect gathers the frame to the host (src/md_env.cu:2502-2506);
  // get_host_particles returns the last gathered frame (:2508-2514), the
  // current one if nothing was gathered yet.
  void sample_collect() {
    host_.resize((size_t)obs().n);
    check(mdb_sim_get_frame(sim_, as_c(host_.data()), (int64_t)host_.size()), "sample_collect");
    collected_ = true;
  }
  void get_host_particles(std::vector<Particle>& out) {
    if (!collected_) sample_collect();
    out = host_;
  }
  void save_env(const std::string& filename, const int step) {
    check(mdb_sim_save_pframe(sim_, filename.c_str(), (uint64_t)step), "save_env");
  }

  // save_env plus the integrator state (restore with the checkpoint constructor)
  void save_checkpoint(const std::string& filename, int step, const std::string& state_file) {
    check(mdb_sim_save_checkpoint(sim_, filename.c_str(), (uint64_t)step, state_file.c_str()),
          "save_checkpoint");
  }
  // The protocol of tests/run_NPH_test/run_test_NPH.cpp (parameters from the
  // configuration); records receive the per-sample log.
  mdb_nph_result_t run_nph_protocol(std::vector<mdb_nph_record_t>* records = nullptr) {
    mdb_nph_protocol_t q;
    const mdb_config_t c = cfg_manager.config.to_c();
    check(mdb_nph_protocol_from_config(&c, &q), "run_nph_protocol");
    std::vector<mdb_nph_record_t> buf(records ? 1 << 16 : 0);
    mdb_nph_result_t r;
    check(mdb_sim_run_nph_protocol(sim_, &q, buf.data(), (int64_t)buf.size(), &r),
          "run_nph_protocol");
    if (records) {
      buf.resize((size_t)(r.n_records < (int64_t)buf.size() ? r.n_records : (int64_t)buf.size()));
      records->swap(buf);
    }
    return r;
  }

  mdb_observables_t observables() const { return obs(); }
  mdb_sim_t* handle() const { return sim_; }

  MDConfigManager cfg_manager;

 private:
  double scalar(int (*fn)(mdb_sim_t*, double*), const char* what) {
    double v = 0.0;
    check(fn(sim_, &v), what);
    return v;
  }
  mdb_observables_t obs() const {
    mdb_observables_t o;
    check(mdb_sim_observables(sim_, &o), "observables");
    return o;
  }
  mdb_sim_t* sim_ = nullptr;
  std::vector<Particle> host_;
  bool collected_ = false;
};

// FireParams (include/md_energy_minimizer.hpp:11-25).
struct FireParams {
  double dt_init = 0.0;
  double dt_max = 0.0;
  double alpha0 = 0.1;
  double f_inc = 1.1;
  double f_dec = 0.5;
  int N_min = 5;

  static FireParams from_config(const MDConfig& cfg) {
    FireParams p;
    p.dt_init = cfg.dt;
    p.dt_max = 5.0 * cfg.dt;
    return p;
  }
  mdb_fire_params_t to_c() const {
    mdb_fire_params_t p;
    std::memset(&p, 0, sizeof p);
    p.dt_init = dt_init;
    p.dt_max = dt_max;
    p.alpha0 = alpha0;
    p.f_inc = f_inc;
    p.f_dec = f_dec;
    p.N_min = N_min;
    return p;
  }
};

// MinimizeResult (include/md_energy_minimizer.hpp:27-35).
struct MinimizeResult {
  std::vector<Particle> frame;
  std::vector<int> energy_steps;
  std::vector<double> energy_trace;
  int steps = 0;
  bool converged = false;
  double max_force = 0.0;
  double potential_energy = 0.0;
};

// EnergyMinimizer (include/md_energy_minimizer.hpp:37-97).
class EnergyMinimizer {
 public:
  explicit EnergyMinimizer(MDConfigManager config_manager,
                           const mdb_options_t& opt = default_options())
      : cfg_manager(std::move(config_manager)), opt_(opt) {}
  template <class Comm>
  EnergyMinimizer(MDConfigManager config_manager, Comm /*ignored*/)
      : EnergyMinimizer(std::move(config_manager)) {}

  MinimizeResult minimize_frame(const std::vector<Particle>& frame, double force_tol,
                                int max_steps, const FireParams& params) {
    const mdb_config_t c = cfg_manager.config.to_c();
    const mdb_fire_params_t p = params.to_c();
    MinimizeResult r;
    r.frame.resize(frame.size());
    // samples: step 0, every 1000 iterations, the last one
    const int64_t cap = (max_steps > 0 ? max_steps / 1000 : 0) + 2;
    std::vector<int32_t> steps((size_t)cap);
    std::vector<double> trace((size_t)cap);
    mdb_minimize_result_t res;
    check(mdb_fire_minimize(&c, as_c(frame.data()), (int64_t)frame.size(), force_tol, max_steps,
                            &p, &opt_, as_c(r.frame.data()), &res, steps.data(), trace.data(),
                            cap),
          "minimize_frame");
    const size_t ns = (size_t)(res.n_energy_samples < cap ? res.n_energy_samples : cap);
    r.energy_steps.assign(steps.begin(), steps.begin() + (long)ns);
    r.energy_trace.assign(trace.begin(), trace.begin() + (long)ns);
    r.steps = res.steps;
    r.converged = res.converged != 0;
    r.max_force = res.max_force;
    r.potential_energy = res.potential_energy;
    return r;
  }

  MDConfigManager cfg_manager;

 private:
  mdb_options_t opt_;
};

}  // namespace mdb200

#ifndef MDB200_NO_GLOBAL_NAMES
using mdb200::EnergyMinimizer;
using mdb200::FireParams;
using mdb200::MDConfig;
using mdb200::MDConfigManager;
using mdb200::MDConfigOverride;
using mdb200::MDSimulation;
using mdb200::MinimizeResult;
using mdb200::Particle;
#endif
