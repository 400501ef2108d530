/*
 * mdb200.h — C ABI of libmdb200.so, the B200-native (sm_100a) MD stepping
 * library for the 2D binary A/B Lennard-Jones system of MD_Simulation_CUDA.
 *
 * Plain C types only: pointers, sizes, POD structs. Every function returns an
 * int status (MDB_OK == 0) and never exits, aborts or traps; the message of
 * the last failure on the calling thread is available from mdb_last_error().
 *
 * Each entry point names the reference interface it replaces
 * (file:line in the MD_Simulation_CUDA source tree).
 *
 * Ownership: the library owns all device memory of a handle. Frames cross the
 * boundary as caller-owned host buffers in the 64-byte Particle layout of
 * include/md_particle.hpp:31-38 and are copied in and out.
 * Threading: a handle may be used by one host thread at a time.
 */
#ifndef MDB200_H
#define MDB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define MDB_OK 0
#define MDB_ERR_CONFIG 1    /* invalid configuration value / unknown key   */
#define MDB_ERR_ARG 2       /* invalid argument (null, size, range)        */
#define MDB_ERR_CAPACITY 3  /* a buffer or frame exceeds a stated capacity */
#define MDB_ERR_NONFINITE 4 /* NaN/Inf detected in the state               */
#define MDB_ERR_BOX 5       /* invalid box (area <= 0, non-finite)         */
#define MDB_ERR_CUDA 6      /* CUDA runtime error                          */
#define MDB_ERR_IO 7        /* file I/O, format or CRC error               */
#define MDB_ERR_STATE 8     /* call not valid in the current state         */
#define MDB_ERR_NODEVICE 9  /* no CUDA device available                    */

/* ---- frame layout -------------------------------------------------------
 * Particle (include/md_particle.hpp:31-38): sizeof 64, align 16,
 * offsets pos 0 / vel 16 / acc 32 / type 48 / theta 56. acc holds F/m.    */
typedef struct mdb_double2 {
  double x, y;
} mdb_double2_t;

typedef struct mdb_particle {
  mdb_double2_t pos;
  mdb_double2_t vel;
  mdb_double2_t acc;
  int32_t type;
  int32_t _pad; /* implicit padding of the reference struct */
  double theta;
} mdb_particle_t;

/* ---- configuration ------------------------------------------------------
 * Field-for-field MDConfig (include/md_config.hpp:14-75); JSON keys are the
 * field names (src/md_config.cpp:43-130). Strings are NUL-terminated.     */
typedef struct mdb_config {
  int32_t n_particles_global;
  int32_t n_particles_type0;
  double box_w_global;
  double box_h_global;
  double T_init;
  double T_target;
  double SIGMA_AA, SIGMA_BB, SIGMA_AB;
  double EPSILON_AA, EPSILON_BB, EPSILON_AB;
  double MASS_A, MASS_B;
  double devide_p;
  double dt;
  double Q;
  double save_dt_interval;
  double cutoff;
  char run_name[256];
  char load_name[256];
  int32_t THREADS_PER_BLOCK;
  int32_t rank_size;
  double mu, v0, D_r, D_theta;
  double barostat_mass;
  double k_piston;
  double barostat_area_rate_init;
  double barostat_height_min_ratio;
  double barostat_height_max_ratio;
  char pressure_target_mode[64];
  double P_target;
  int32_t pressure_target_auto_steps;
  int32_t pressure_eval_interval_steps;
  int32_t pressure_window_samples;
  double pressure_tolerance_rel;
  int32_t pressure_stable_required_windows;
  int32_t nph_warmup_min_steps;
  int32_t nph_warmup_max_steps;
  int32_t nph_steps;
  int32_t rank_idx;
  int32_t n_local;
  int32_t n_halo_left;
  int32_t n_halo_right;
  int32_t n_cap;
  int32_t halo_left_cap;
  int32_t halo_right_cap;
  int32_t left_rank;
  int32_t right_rank;
  double x_min;
  double x_max;
} mdb_config_t;

/* Engine options with no counterpart in MDConfig (B200 engine knobs). */
typedef struct mdb_options {
  int32_t device;     /* CUDA device ordinal (default 0)                    */
  double skin;        /* Verlet-list skin in sigma units; 0 (default):
                         0.45, or 0.2 when every system is a FIRE run    */
  int32_t use_graphs; /* 1: replay captured CUDA graphs for step chunks     */
  int32_t max_neighbors; /* neighbour-list capacity per particle (default 48;
                            -1: no lists, always scan the cell stencil)     */
  int32_t stream_priority; /* 0 (default): the handle's stream has normal
                              priority; k > 0: k levels above it (clamped to
                              the device's range), so its kernels' blocks
                              are scheduled before those of lower streams   */
  int32_t fire_precision; /* FIRE pair arithmetic: MDB_FIRE_AUTO (default)
                             runs the reference's FP32 pair terms until a
                             system's max |a| falls below 1e-3, then FP64
                             pair terms and sums for that system, so that
                             max |a| < 1e-6 is reachable; MDB_FIRE_FP32 keeps
                             FP32 pair terms throughout (stalls near 1e-6, as
                             the reference does); MDB_FIRE_FP64 uses FP64
                             pair terms from the first iteration           */
  int32_t autotune;       /* 1: at build, time the engine's schedule
                             candidates on the device (list prefetch depth
                             of the force phase, list-build grid, rebuild
                             grid) and keep the fastest, cached per device
                             and workload shape in the file named by
                             MDB_SCHEDULE_CACHE (default
                             ~/.cache/md_simulation_cuda_b200/schedule.txt).
                             None of these changes any result bit.
                             0 (default): the built-in schedule           */
  int32_t step_kernel;    /* MD steps of a single-system handle:
                             MDB_STEPS_AUTO (0, default) or MDB_STEPS_MULTI:
                             the multi-step kernel when every block of the
                             system fits on the device at once (two per SM,
                             so up to ~75k particles on a B200): one
                             cooperative launch runs the drift and force
                             phases of many steps with grid barriers between
                             them and returns only for a cell-list rebuild
                             (calls of fewer than 4 steps use the per-phase
                             kernels, whose launch costs less);
                             MDB_STEPS_PER_PHASE: one kernel per phase.
                             Both give the same result bits.               */
  int32_t lanes;          /* lanes per particle in the force phase of MD
                             systems of at most 16,384 particles:
                             MDB_LANES_SPLIT: 4 lanes split each particle's
                             pair candidates (4x the warps for a small system;
                             the force sums change in their last bits);
                             MDB_LANES_ONE: one lane (the order of batches);
                             MDB_LANES_AUTO (0, default): SPLIT for
                             single-system simulation handles, ONE for batch,
                             multi-device and server handles (where a batch
                             fills the GPU and splitting costs ~30%). A system
                             gives the same bits alone and in a batch when
                             both handles use the same setting. FIRE systems
                             always use one lane.                          */
  int32_t reserved[7];
} mdb_options_t;

#define MDB_LANES_AUTO 0
#define MDB_LANES_ONE 1
#define MDB_LANES_SPLIT 4

#define MDB_STEPS_AUTO 0
#define MDB_STEPS_PER_PHASE 1
#define MDB_STEPS_MULTI 2

#define MDB_FIRE_AUTO 0
#define MDB_FIRE_FP32 1
#define MDB_FIRE_FP64 2

/* The engine schedule a handle runs with (no counterpart in the reference):
 * chosen by the autotuner (mdb_options_t.autotune) or built in. */
typedef struct mdb_schedule {
  int32_t list_prefetch_rows; /* force phase: next chunk's list rows per warp
                                 prefetched into L1                         */
  int32_t nlist_grid;         /* blocks of the list-build kernel             */
  int32_t rebuild_grid;       /* blocks of the other rebuild kernels         */
  int32_t items;              /* particles per thread of the largest system  */
  int32_t tuned;              /* 1: chosen by the autotuner                  */
  int32_t from_cache;         /* 1: read from the schedule cache file        */
  double skin;                /* neighbour-list skin                         */
  double tune_ms;             /* time spent timing candidates                */
  int32_t multi_step;         /* 1: MD steps run in the multi-step kernel    */
  int32_t multi_step_blocks;  /* blocks the device holds at once for it      */
} mdb_schedule_t;

/* MDConfig{} value-initialised defaults (include/md_config.hpp:14-75). */
int mdb_config_default(mdb_config_t* out);
/* MDConfigManager::config_from_json / deserialize (src/md_config.cpp:43-130,
 * 289-325): keys absent from the JSON object keep the struct defaults. */
int mdb_config_from_json(const char* json_text, mdb_config_t* out);
int mdb_config_from_json_file(const char* path, mdb_config_t* out);
/* MDConfigManager::serialize / config_to_json (src/md_config.cpp:132-195,
 * 304-319). indent < 0 gives the compact form of serialize(). `needed`
 * (optional) receives the length excluding the NUL. */
int mdb_config_to_json(const mdb_config_t* cfg, int32_t indent, char* buf, size_t cap,
                       size_t* needed);
/* MDConfigManager::apply_override (src/md_config.cpp:327-452): MDB_OK on
 * success, MDB_ERR_CONFIG for an unknown key or a value that does not parse. */
int mdb_config_apply_override(mdb_config_t* cfg, const char* key, const char* value);
/* MDConfigManager::parse_override_argument (src/md_config.cpp:465-495):
 * strips "--" then "D", splits on '='. MDB_ERR_ARG when it is not an override. */
int mdb_parse_override_argument(const char* arg, char* key, size_t key_cap, char* value,
                                size_t value_cap);
void mdb_options_default(mdb_options_t* out);

/* ---- PFRAME v2 files (include/md_common.hpp:17-31, src/md_common.cpp:110-320)
 * 16-byte FileHeader {"PFRAME", version 2, 0}; per frame a packed 36-byte
 * FrameHeader {frame_index, n, raw bytes, compressed bytes, crc32} and a zlib
 * (level 9) payload of Particle[n].                                          */
/* FileWriter(path, append) + write_frame: append != 0 opens an existing file
 * (validating its header) and appends; otherwise the file is created. */
int mdb_pframe_write(const char* path, int32_t append, const mdb_particle_t* frame, int64_t n,
                     uint64_t frame_index);
/* FileReader + next_frame scan used by MDSimulation(cfg, comm, file, step)
 * (src/md_env.cu:81-164): finds the first frame whose index equals
 * frame_index. n_out receives the frame size; when cap < n only n_out is set
 * and MDB_ERR_CAPACITY is returned. */
int mdb_pframe_read(const char* path, uint64_t frame_index, mdb_particle_t* out, int64_t cap,
                    int64_t* n_out);
/* Number of complete frames and the index of the last one. */
int mdb_pframe_count(const char* path, int64_t* n_frames, uint64_t* last_index);

/* ---- single-system simulation (class MDSimulation, include/md_env.hpp:51-263)
 */
typedef struct mdb_sim mdb_sim_t;

/* MDSimulation(MDConfigManager, MPI_Comm) (src/md_env.cu:21-79) when frame is
 * NULL: the reference-style lattice initialisation (src/md_env.cu:1276-1445).
 * With a frame: the frame is loaded as-is (the path the ctor-from-file takes,
 * src/md_env.cu:81-164). Forces are computed before returning, as the
 * reference constructors do. n must equal cfg->n_particles_global when frame is
 * NULL. */
int mdb_sim_create(const mdb_config_t* cfg, const mdb_particle_t* frame, int64_t n,
                   const mdb_options_t* opt, mdb_sim_t** out);
/* MDSimulation(cfg, comm, filename, step) (src/md_env.cu:81-164). */
int mdb_sim_create_from_pframe(const mdb_config_t* cfg, const char* path, uint64_t step,
                               const mdb_options_t* opt, mdb_sim_t** out);
int mdb_sim_destroy(mdb_sim_t* sim);

/* step_single_NVE (src/md_env.cu:1576-1637), repeated nsteps times. */
int mdb_sim_step_nve(mdb_sim_t* sim, int64_t nsteps);
/* step_single_nose_hoover(do_middle_wrap) (src/md_env.cu:1639-1728).
 * do_middle_wrap (LG slab reflection) is not part of this library: a
 * non-zero value returns MDB_ERR_ARG. */
int mdb_sim_step_nose_hoover(mdb_sim_t* sim, int64_t nsteps, int32_t do_middle_wrap);
/* step_single_NPH(P_ext) (src/md_env.cu:1795-1918). */
int mdb_sim_step_nph(mdb_sim_t* sim, double p_ext, int64_t nsteps);
/* step_single_NPH_piston(P_ext) (src/md_env.cu:1920-2023). */
int mdb_sim_step_nph_piston(mdb_sim_t* sim, double p_ext, int64_t nsteps);

/* cal_total_K (src/md_env.cu:2141-2146). */
int mdb_sim_total_K(mdb_sim_t* sim, double* out);
/* cal_total_U (src/md_env.cu:2347-2360), including wall energy in piston mode. */
int mdb_sim_total_U(mdb_sim_t* sim, double* out);
/* cal_partial_U_lambda (src/md_env.cu:2362-2406, kernel
 * src/md_cuda_common.cu:266-377): -epsilon_lambda * 1/2 sum_i sum_j
 * (Fx dx - Fy dy) over the current frame (FP32 pair force, FP64 products and
 * sums), y periodic unless the piston mode is active. The reference counts
 * x-edge partners twice at MPI world size 1; this is the nearest-image sum. */
int mdb_sim_partial_U_lambda(mdb_sim_t* sim, double epsilon_lambda, double* out);
/* get_N_profile (src/md_env.cu:3920-3985, kernel src/md_cuda_common.cu:827-871)
 * at MPI world size 1: counts of type 0 in out[0..nb) and of the other types
 * in out[nb..2nb), in nb equal x bins over [0, Lx]. */
int mdb_sim_n_profile(mdb_sim_t* sim, int32_t nb, int32_t* out);
/* get_density_profile (src/md_env.cu:4086-4104): (n_A - n_B) / (n_A + n_B)
 * per x bin, 0 for an empty bin; out holds nb doubles. */
int mdb_sim_density_profile(mdb_sim_t* sim, int32_t nb, double* out);
/* get_pressure_profile (src/md_env.cu:3821-3918, kernel
 * src/md_cuda_common.cu:873-1030): Irving-Kirkwood pressure tensor in nb y
 * bins, out[3*nb] = {P_xx | P_yy | P_xy}: kinetic m v_a v_b at the bin of
 * y_i, pair 1/2 r_a F_b at the bin of the minimum-image midpoint, divided by
 * the bin area Lx * Ly / nb. Pairs from the cell stencil; sums in 64-bit
 * fixed point (2^-24), so the result does not depend on thread order. The y
 * axis is periodic unless the piston mode is active (the reference always
 * treats it as periodic). */
int mdb_sim_pressure_profile(mdb_sim_t* sim, int32_t nb, double* out);
/* cal_instant_pressure (src/md_env.cu:2254-2266). */
int mdb_sim_instant_pressure(mdb_sim_t* sim, double* out);

typedef struct mdb_observables {
  double t;                       /* MDSimulation::t                        */
  double Lx, Ly;                  /* get_Lx / get_Ly                        */
  double xi;                      /* Nose-Hoover xi                         */
  double last_instant_pressure;   /* get_last_instant_pressure              */
  double nph_area_momentum;       /* p_A                                    */
  double nph_area_rate;           /* get_nph_area_rate                      */
  double nph_piston_velocity;     /* get_nph_piston_velocity                */
  double nph_piston_force;        /* get_nph_piston_force                   */
  int64_t n;                      /* particles                              */
  int64_t steps;                  /* steps taken since creation             */
  int64_t rebuilds;               /* cell-list rebuilds since creation      */
  int32_t piston_mode_active;
  int32_t nonfinite;              /* 1 when NaN/Inf was seen in the state   */
} mdb_observables_t;
int mdb_sim_observables(mdb_sim_t* sim, mdb_observables_t* out);
/* The same record, queued on the handle's stream after the steps issued so
 * far, without waiting (no counterpart in the reference, whose getters read
 * host copies after a device synchronisation): *out is written when the
 * stream reaches the copy, so it is valid after mdb_sim_synchronize (or any
 * synchronous call). For a copy that overlaps with computation, *out should
 * be pinned host memory; any host memory works. An error state is reported by
 * the next synchronous call. */
int mdb_sim_observables_async(mdb_sim_t* sim, mdb_observables_t* out);

/* sample_collect + get_host_particles (src/md_env.cu:2502-2514): the frame in
 * the caller's original particle order. n must equal the particle count. */
int mdb_sim_get_frame(mdb_sim_t* sim, mdb_particle_t* out, int64_t n);
/* Replace the state with a frame and recompute forces (ctor semantics). */
int mdb_sim_set_frame(mdb_sim_t* sim, const mdb_particle_t* frame, int64_t n);
/* save_env (src/md_env.cu:4106-4124): appends the current frame to a PFRAME
 * file (created when absent). */
int mdb_sim_save_pframe(mdb_sim_t* sim, const char* path, uint64_t frame_index);
/* Checkpoint: save_env's PFRAME frame (appended to frame_path) plus a state
 * file (JSON text) with what the reference's restart from a frame loses
 * (MDSimulation(cfg, comm, file, step), src/md_env.cu:81-164, restarts with
 * the configuration's box, xi = 0 and fresh barostat / piston state): t, the
 * box, xi, K, p_A, the aspect ratio and Ly clamps, the piston velocity and
 * force, the external pressure and the mode flags. Restoring builds the
 * simulation from the frame with the saved box and state, so the following
 * steps continue the saved trajectory. */
int mdb_sim_save_checkpoint(mdb_sim_t* sim, const char* frame_path, uint64_t frame_index,
                            const char* state_path);
int mdb_sim_create_from_checkpoint(const mdb_config_t* cfg, const char* frame_path,
                                   uint64_t frame_index, const char* state_path,
                                   const mdb_options_t* opt, mdb_sim_t** out);
int mdb_sim_get_config(mdb_sim_t* sim, mdb_config_t* out);
/* The cudaStream_t (as void*) all work of this handle is issued on. */
int mdb_sim_cuda_stream(mdb_sim_t* sim, void** stream);
/* Measurement aid: runs nsteps Nose-Hoover (kind 2), NVE (kind 1) or NPH
 * (kind 3, at the external pressure of the last mdb_sim_step_nph call) steps
 * with each phase launched separately and bracketed by CUDA events on the
 * handle's stream; ms_out[0..2] receive the summed drift, cell-rebuild and
 * force-phase times in milliseconds. The steps advance the simulation like
 * mdb_sim_step_*. No counterpart in the reference (which has no timers). */
int mdb_sim_phase_times(mdb_sim_t* sim, int32_t kind, int64_t nsteps, double* ms_out);
/* The schedule the simulation runs with (no counterpart in the reference). */
int mdb_sim_schedule(mdb_sim_t* sim, mdb_schedule_t* out);
/* Block until all issued work of the handle has finished. */
int mdb_sim_synchronize(mdb_sim_t* sim);

/* ---- asynchronous trajectory writer ---------------------------------------
 * save_env (src/md_env.cu:4106-4124) writes a PFRAME frame and returns when it
 * is on disk. mdb_traj_writer_write instead queues the export of the
 * simulation's current frame on the simulation's stream (after the steps
 * issued so far) into one of `depth` pinned staging slots and returns; a
 * writer thread compresses and appends each frame to `path` (created unless
 * append != 0) in the same PFRAME v2 format. A write waits only when all
 * slots are in flight. flush waits until every queued frame is on disk; close
 * flushes, stops the thread and frees the slots. Both return the first I/O or
 * CUDA error of any queued frame. */
typedef struct mdb_traj_writer mdb_traj_writer_t;
int mdb_traj_writer_open(const char* path, int32_t append, int32_t depth,
                         mdb_traj_writer_t** out);
int mdb_traj_writer_write(mdb_traj_writer_t* w, mdb_sim_t* sim, uint64_t frame_index);
int mdb_traj_writer_flush(mdb_traj_writer_t* w);
int mdb_traj_writer_close(mdb_traj_writer_t* w);

/* ---- NPH driver protocol ---------------------------------------------------
 * The protocol of the reference's NPH driver (tests/run_NPH_test/
 * run_test_NPH.cpp:137-290): AUTO_TARGET (Nose-Hoover steps; the pressure
 * sampled every eval_interval steps, averaged over auto_steps steps, becomes
 * the target) -> NPH_WARMUP (NPH steps at the target; once warmup_min_steps
 * have run and the rolling window of window_samples samples is full, each
 * step whose window mean and standard deviation are within tolerance_rel of
 * the target counts, stable_required such steps in a row end the warmup; it
 * ends anyway after warmup_max_steps) -> NPH_PRODUCTION (production_steps NPH
 * steps). The decisions fall on the same steps, with the same arithmetic, as
 * in the driver's per-step loop. records (up to cap) receive one entry per
 * sample step, like the driver's pressure log.
 *
 * By default the whole protocol is one graph launch: a while node runs one
 * step per iteration, a switch node picks the Nose-Hoover or NPH step body,
 * and the pressure samples, window statistics and phase switches are taken
 * on the device; the host waits only after the last step. With host_driven
 * set (or a handle created with use_graphs = 0) the host takes the decisions
 * and issues the steps between two decision points as captured chunks,
 * waiting once per sample. */
typedef struct mdb_nph_protocol {
  int32_t auto_target;   /* 1: start with AUTO_TARGET ("auto_initial" mode)  */
  int32_t _pad0;
  double P_target;       /* the target when auto_target == 0                  */
  int32_t auto_steps, eval_interval, window_samples, stable_required;
  int32_t warmup_min_steps, warmup_max_steps, production_steps, _pad1;
  double tolerance_rel;
  int32_t host_driven;   /* 1: decisions on the host between step chunks      */
  int32_t reserved[7];
} mdb_nph_protocol_t;

#define MDB_PHASE_AUTO_TARGET 0
#define MDB_PHASE_NPH_WARMUP 1
#define MDB_PHASE_NPH_PRODUCTION 2

typedef struct mdb_nph_record {
  int64_t step;
  double t;
  int32_t phase; /* MDB_PHASE_* the step ran in */
  int32_t _pad;
  double P_inst, P_target, mean, stddev, rel_err; /* rolling window stats */
  double Lx, Ly, dA_dt;
} mdb_nph_record_t;

typedef struct mdb_nph_result {
  double P_target;
  int64_t auto_end_step;   /* -1 when there was no AUTO_TARGET phase        */
  int64_t warmup_end_step; /* -1 when the warmup did not end                */
  int64_t total_steps;
  int64_t n_records;       /* sample steps (may exceed cap)                 */
  int32_t forced_switch;   /* the warmup ended at warmup_max_steps          */
  int32_t finished;        /* production completed                          */
  int64_t host_waits;      /* blocking waits of the host during the run     */
} mdb_nph_result_t;

/* The protocol parameters as the driver derives them from MDConfig
 * (pressure_target_mode, P_target, pressure_*, nph_warmup_*, nph_steps). */
int mdb_nph_protocol_from_config(const mdb_config_t* cfg, mdb_nph_protocol_t* out);
int mdb_sim_run_nph_protocol(mdb_sim_t* sim, const mdb_nph_protocol_t* protocol,
                             mdb_nph_record_t* records, int64_t cap, mdb_nph_result_t* result);
/* The protocol's decisions for a given pressure per step (pressures[step],
 * n entries), without a simulation; chunks receives the number of step
 * chunks the real run would issue. */
int mdb_nph_protocol_dry_run(const mdb_nph_protocol_t* protocol, const double* pressures,
                             int64_t n, mdb_nph_record_t* records, int64_t cap,
                             mdb_nph_result_t* result, int64_t* chunks);

/* ---- FIRE minimiser (class EnergyMinimizer, include/md_energy_minimizer.hpp)
 */
typedef struct mdb_fire_params { /* FireParams (md_energy_minimizer.hpp:11-25) */
  double dt_init, dt_max, alpha0, f_inc, f_dec;
  int32_t N_min;
  int32_t _pad;
} mdb_fire_params_t;
/* FireParams::from_config: dt_init = dt, dt_max = 5 dt, alpha0 0.1,
 * f_inc 1.1, f_dec 0.5, N_min 5. */
int mdb_fire_params_from_config(const mdb_config_t* cfg, mdb_fire_params_t* out);

typedef struct mdb_minimize_result { /* MinimizeResult (.hpp:27-35) */
  int32_t steps;
  int32_t converged;
  double max_force;        /* max |a| at the last evaluated iteration */
  double potential_energy; /* U of the final frame                    */
  int64_t n_energy_samples;
  int32_t nonfinite;
  int32_t _pad;
} mdb_minimize_result_t;

/* EnergyMinimizer::minimize_frame (src/md_energy_minimizer.cu:122-272) for one
 * frame. energy_steps / energy_trace receive up to trace_cap samples (step 0,
 * every 1000 iterations, and the final one). */
int mdb_fire_minimize(const mdb_config_t* cfg, const mdb_particle_t* frame, int64_t n,
                      double force_tol, int32_t max_steps, const mdb_fire_params_t* params,
                      const mdb_options_t* opt, mdb_particle_t* frame_out,
                      mdb_minimize_result_t* result, int32_t* energy_steps,
                      double* energy_trace, int64_t trace_cap);

/* ---- batched independent systems -------------------------------------------
 * Many independent systems of uneven N advanced together: one launch per
 * phase covers every system (per-system cell grids, reductions and scalar
 * state), so small systems do not leave the GPU idle. The reference runs each
 * system as a separate job (scripts/submit_batches_*.sh); the per-system
 * semantics are those of EnergyMinimizer::minimize_frame and the MDSimulation
 * step functions above. */
typedef struct mdb_batch mdb_batch_t;

#define MDB_JOB_FIRE 0
#define MDB_JOB_NVE 1
#define MDB_JOB_NVT 2 /* Nose-Hoover */

int mdb_batch_create(const mdb_options_t* opt, mdb_batch_t** out);
int mdb_batch_destroy(mdb_batch_t* b);
/* Add a FIRE quench (minimize_frame semantics). Returns its id in sys_id. */
int mdb_batch_add_fire(mdb_batch_t* b, const mdb_config_t* cfg, const mdb_particle_t* frame,
                       int64_t n, double force_tol, int32_t max_steps,
                       const mdb_fire_params_t* params, int32_t* sys_id);
/* Add an MD segment: nsteps repetitions of step_single_NVE (MDB_JOB_NVE) or
 * step_single_nose_hoover (MDB_JOB_NVT) (src/md_env.cu:1576-1728) from the
 * given frame, with the constructor's initial force evaluation
 * (src/md_env.cu:61-79). g = 2n - 2 uses this system's n. Every system of a
 * batch has the same kind (FIRE, NVE or NVT); mixing returns MDB_ERR_STATE.
 * A system stops after its own nsteps while the others continue. */
int mdb_batch_add_md(mdb_batch_t* b, const mdb_config_t* cfg, const mdb_particle_t* frame,
                     int64_t n, int32_t kind, int64_t nsteps, int32_t* sys_id);
/* Advance every unfinished system by up to `iterations` iterations (FIRE
 * iterations or MD steps); iterations < 0 runs until all are finished. */
int mdb_batch_run(mdb_batch_t* b, int64_t iterations);
/* Number of systems and how many are finished. */
int mdb_batch_progress(mdb_batch_t* b, int32_t* n_systems, int32_t* n_done);
int mdb_batch_system_info(mdb_batch_t* b, int32_t sys_id, int64_t* n, int32_t* done,
                          int64_t* steps);
/* Cell-list rebuilds of one system so far, and its particles whose neighbour
 * list overflowed max_neighbors at the last rebuild (they scan the cell
 * stencil instead). No counterpart in the reference (diagnostics). */
int mdb_batch_system_stats(mdb_batch_t* b, int32_t sys_id, int64_t* rebuilds,
                           int32_t* list_overflow);
int mdb_batch_get_frame(mdb_batch_t* b, int32_t sys_id, mdb_particle_t* out, int64_t n);
int mdb_batch_get_fire_result(mdb_batch_t* b, int32_t sys_id, mdb_minimize_result_t* result,
                              int32_t* energy_steps, double* energy_trace, int64_t trace_cap);
/* cal_total_K / cal_total_U (src/md_env.cu:2141-2146, 2347-2360) and the
 * Nose-Hoover xi of one system, or of every system (arrays of n = number of
 * systems; any pointer may be NULL). */
int mdb_batch_energies(mdb_batch_t* b, int32_t sys_id, double* K, double* U, double* xi);
int mdb_batch_energies_all(mdb_batch_t* b, double* K, double* U, double* xi, int32_t n);
/* Asynchronous form of mdb_batch_run (no counterpart in the reference): issue
 * one chunk of at most `iterations` (< 0: no limit) iterations, ending at the
 * next multiple of 1000, on the batch's stream and return at once; `issued`
 * receives its length (0 when every system has finished). mdb_batch_query
 * reports whether the stream has finished (idle = 1) without waiting;
 * mdb_batch_collect then records finished systems and FIRE energy samples. */
int mdb_batch_issue(mdb_batch_t* b, int64_t iterations, int64_t* issued);
int mdb_batch_query(mdb_batch_t* b, int32_t* idle);
int mdb_batch_collect(mdb_batch_t* b);
/* mdb_sim_partial_U_lambda for every system of a batch (n = number of
 * systems), e.g. the points of a lambda sweep run as one batch. */
int mdb_batch_partial_U_lambda_all(mdb_batch_t* b, double epsilon_lambda, double* out,
                                   int32_t n);
/* Which systems have finished, as of the last run or collect (n = number of
 * systems). */
int mdb_batch_done_flags(mdb_batch_t* b, int32_t* done, int32_t n);
/* Device memory the batch holds (0 before its first run). */
int mdb_batch_device_bytes(mdb_batch_t* b, int64_t* bytes);
/* The schedule of the batch's engine (zeros before its first run). */
int mdb_batch_schedule(mdb_batch_t* b, mdb_schedule_t* out);

/* ---- independent systems over several GPUs (no counterpart in the reference,
 * which runs one system per job: scripts/submit_batches_*.sh) --------------
 * mdb_place_lpt: the greedy longest-processing-time placement of n items of
 * the given costs on nbins bins (largest cost first, each to the least-loaded
 * bin, ties to the lower bin); bin_out[n], load_out[nbins] (optional).
 * A multi-device batch takes systems like mdb_batch_* (one kind per batch),
 * places them at its first run by that rule on particles x steps (FIRE: the
 * iteration cap) over `devices` (a device may be listed more than once), and
 * runs one batch per device concurrently from the calling thread. No data
 * crosses devices; each system's results equal its results alone. */
int mdb_place_lpt(const double* costs, int32_t n, int32_t nbins, int32_t* bin_out,
                  double* load_out);
typedef struct mdb_multibatch mdb_multibatch_t;
int mdb_multibatch_create(const mdb_options_t* opt, const int32_t* devices, int32_t ndev,
                          mdb_multibatch_t** out);
int mdb_multibatch_destroy(mdb_multibatch_t* m);
int mdb_multibatch_add_fire(mdb_multibatch_t* m, const mdb_config_t* cfg,
                            const mdb_particle_t* frame, int64_t n, double force_tol,
                            int32_t max_steps, const mdb_fire_params_t* params, int32_t* sys_id);
int mdb_multibatch_add_md(mdb_multibatch_t* m, const mdb_config_t* cfg,
                          const mdb_particle_t* frame, int64_t n, int32_t kind, int64_t nsteps,
                          int32_t* sys_id);
/* Advance every system by up to `iterations` (< 0: until all are finished). */
int mdb_multibatch_run(mdb_multibatch_t* m, int64_t iterations);
/* The device each system was placed on (n = number of systems). */
int mdb_multibatch_placement(mdb_multibatch_t* m, int32_t* device_of, int32_t n);
int mdb_multibatch_progress(mdb_multibatch_t* m, int32_t* n_systems, int32_t* n_done);
int mdb_multibatch_system_info(mdb_multibatch_t* m, int32_t sys_id, int64_t* n, int32_t* done,
                               int64_t* steps);
int mdb_multibatch_get_frame(mdb_multibatch_t* m, int32_t sys_id, mdb_particle_t* out,
                             int64_t n);
int mdb_multibatch_get_fire_result(mdb_multibatch_t* m, int32_t sys_id,
                                   mdb_minimize_result_t* result, int32_t* energy_steps,
                                   double* energy_trace, int64_t trace_cap);
int mdb_multibatch_energies(mdb_multibatch_t* m, int32_t sys_id, double* K, double* U,
                            double* xi);
int mdb_batch_cuda_stream(mdb_batch_t* b, void** stream);

/* ---- serving: continuous batching of MD and FIRE requests ------------------
 * No counterpart in the reference (which runs one MPI job per simulation). A
 * server owns one worker thread and one device. Requests (an MD segment or a
 * FIRE quench, each with its own config and frame) wait in a queue; while
 * fewer than max_active_batches batches are in flight and the HBM budget
 * allows, the first request in the admission order (MDB_ORDER_*) and the
 * following requests of the same kind in that order are admitted together as
 * a new batch on its own stream, so requests
 * admitted at different times run concurrently. Results (frame and
 * observables) become available as soon as the request's own system
 * finishes; a batch's device memory is released when all of its systems
 * have. A request's result equals that of the same job run alone
 * (mdb_batch_* with one system, or mdb_sim_* / mdb_fire_minimize). All
 * functions are thread-safe. */
typedef struct mdb_server mdb_server_t;

typedef struct mdb_server_options {
  int32_t device;              /* CUDA device ordinal (default 0)               */
  int32_t max_active_batches;  /* batches in flight at once (default 8)         */
  int64_t hbm_budget_bytes;    /* device memory for batches (0: 80% of free)    */
  int64_t max_batch_particles; /* particles per admitted batch (default 1Mi; a
                                  larger request is admitted alone)            */
  int32_t max_batch_systems;   /* systems per admitted batch (default 1024)     */
  int32_t chunk;               /* steps / iterations issued per chunk (500)     */
  double skin;                 /* as mdb_options_t                               */
  int32_t use_graphs;
  int32_t max_neighbors;
  int32_t order;               /* admission order (default MDB_ORDER_SHORTEST)  */
  int32_t max_wait_ms;         /* MDB_ORDER_SHORTEST: requests queued longer
                                  than this go first, oldest first (default
                                  60000; 0: no bound)                           */
  int32_t priorities;          /* 1 (default): a batch's stream priority rises
                                  as its work falls, so the kernels of short
                                  requests are scheduled ahead of long ones;
                                  0: every batch at normal priority             */
  int32_t reserved[5];
} mdb_server_options_t;

/* Admission order of queued requests. FIFO: the oldest request and the
 * following queued requests of its kind. SHORTEST: the request with the least
 * work (particles x steps, or particles x max_steps for FIRE) and the queued
 * requests of its kind in order of work; a request waiting longer than
 * max_wait_ms goes before any that has not. Throughput is the same; SHORTEST
 * lowers the median latency when the queue is long. */
#define MDB_ORDER_FIFO 0
#define MDB_ORDER_SHORTEST 1

typedef struct mdb_request {
  int32_t kind;            /* MDB_JOB_FIRE, MDB_JOB_NVE or MDB_JOB_NVT          */
  int32_t max_steps;       /* FIRE: iteration cap                                */
  int64_t nsteps;          /* NVE/NVT: segment length in steps                   */
  double force_tol;        /* FIRE: stop at max |a| < force_tol                  */
  mdb_fire_params_t fire;  /* FIRE parameters                                    */
} mdb_request_t;

#define MDB_REQ_QUEUED 0
#define MDB_REQ_RUNNING 1
#define MDB_REQ_DONE 2
#define MDB_REQ_FAILED 3

typedef struct mdb_request_result {
  int32_t status;     /* MDB_REQ_*                                              */
  int32_t error;      /* status code of a failed request                         */
  int64_t n;          /* particles                                               */
  int64_t steps;      /* MD steps taken / FIRE iterations (as minimize_frame)    */
  int32_t converged;  /* FIRE                                                    */
  int32_t nonfinite;
  double K, U, xi;    /* final kinetic and potential energy, Nose-Hoover xi      */
  double max_force;   /* FIRE: max |a| at the end                                */
  double t_submit, t_start, t_done; /* seconds since the server was created      */
} mdb_request_result_t;

typedef struct mdb_server_stats {
  int64_t submitted, queued, running, finished, failed;
  int64_t batches_admitted, active_batches;
  int64_t device_bytes;      /* held by batches in flight                        */
  int64_t hbm_budget_bytes;
  double particle_steps;     /* sum of n x steps over finished requests          */
  double elapsed_s;          /* since the server was created                     */
} mdb_server_stats_t;

void mdb_server_options_default(mdb_server_options_t* out);
int mdb_server_create(const mdb_server_options_t* opt, mdb_server_t** out);
/* Stops admitting, lets the chunks in flight end, fails what has not
 * finished, joins the worker and frees everything. */
int mdb_server_destroy(mdb_server_t* s);
/* Queues a request (the frame is copied); its id goes to *id. */
int mdb_server_submit(mdb_server_t* s, const mdb_config_t* cfg, const mdb_particle_t* frame,
                      int64_t n, const mdb_request_t* req, int64_t* id);
/* Waits until the request has finished or failed, or timeout_s seconds
 * (< 0: no limit); *info receives its current record either way. */
int mdb_server_wait(mdb_server_t* s, int64_t id, double timeout_s, mdb_request_result_t* info);
/* The result of a finished request: frame_out (n particles, may be NULL) and
 * *info; releases the request. A failed request returns its error status. */
int mdb_server_result(mdb_server_t* s, int64_t id, mdb_particle_t* frame_out, int64_t n,
                      mdb_request_result_t* info);
int mdb_server_stats(mdb_server_t* s, mdb_server_stats_t* out);

/* ---- single-call kernels (building blocks, used by tests) ------------------
 */
/* li_force_kernel (src/md_cuda_common.cu:151-264) + cal_local_U_kernel
 * (:703-825) + the pair part of cal_local_pressure_scalar_kernel (:591-701)
 * for one frame: acc_out (2n doubles, F/m in the frame's order), U (shifted
 * pair energy) and W = sum_i 1/2 sum_j r.F. periodic_y selects the y image
 * convention (0 for the piston walls' LJ part). */
int mdb_compute_forces(const mdb_config_t* cfg, const mdb_particle_t* frame, int64_t n,
                       double Lx, double Ly, int32_t periodic_y, const mdb_options_t* opt,
                       double* acc_out, double* U_out, double* W_out);
/* The cell binning of the force path: cell = cy*ncx + cx with
 * ncx = max(1, floor(Lx/cell_min)), cx = clamp(trunc(x*(ncx/Lx)), 0, ncx-1)
 * (NaN bins to 0), and perm = the stable sort of particle indices by cell.
 * pos is 2n doubles (x0,y0,x1,y1,...). cell_out and perm_out hold n ints. */
int mdb_cell_build(const double* pos, int64_t n, double Lx, double Ly, double cell_min,
                   int32_t device, int32_t* cell_out, int32_t* perm_out, int32_t* ncx_out,
                   int32_t* ncy_out);

/* ---- forces without allocation ------------------------------------------
 * No counterpart in the reference: an added entry point for callers that
 * cannot allocate device memory — hosts whose own pool or caching allocator
 * owns the device memory and forbids allocations behind its back, and loops
 * that must not stall other streams on the implicit synchronisation of
 * cudaMalloc/cudaFree. It computes what mdb_compute_forces computes, from
 * device buffers the caller owns, on the caller's stream (`stream` is a
 * cudaStream_t; NULL = the legacy default stream), and returns without
 * synchronising. It calls no cudaMalloc, cudaFree or other allocating routine.
 *   pos  device, 2n doubles (x0,y0,x1,y1,...)   type device, n int32
 *   acc  device, 2n doubles out: F/m            uw   device, 2 doubles out:
 *        U (shifted pair energy), W = sum_i 1/2 sum_j r.F
 * Limit: n <= MDB_NOALLOC_MAX_PARTICLES (larger n returns MDB_ERR_CAPACITY
 * before any work), because its scratch memory is one fixed 1 MiB device
 * array inside the library. Every call on a device shares that array: calls
 * ordered on one stream are independent (each clears what must start at
 * zero), calls that overlap on the GPU race and give wrong results. The
 * first call on a device (with that device current) looks the array's
 * address up; make that first call before any stream capture. After a
 * cudaDeviceReset (or with another context current) the next call looks it up
 * again. Cost: a cell holding m particles costs m^2 comparisons to order; a
 * frame with all n particles in one cell (clustered, or non-finite positions)
 * costs n^2 (seconds at n = 65536). */
#define MDB_NOALLOC_MAX_PARTICLES 65536
int mdb_compute_forces_noalloc(const mdb_config_t* cfg, const double* pos, const int32_t* type,
                               int64_t n, double Lx, double Ly, int32_t periodic_y, void* stream,
                               double* acc, double* uw);

/* ---- misc --------------------------------------------------------------- */
/* Copies the last error message of the calling thread (NUL-terminated). */
int mdb_last_error(char* buf, size_t cap);
const char* mdb_version(void);
/* Number of kernel launches this library issued so far (all handles). */
int64_t mdb_kernel_launches(void);

#ifdef __cplusplus
}
#endif

#endif /* MDB200_H */
