/*
 * mdoracle.h — CPU restatement of the MD stepping path of MD_Simulation_CUDA.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker that the CUDA product is
 * compared against, and the CPU baseline bench.py times beside it. Nothing in
 * the product (md_simulation_cuda_b200/) may link, import or call it.
 *
 * Parity status: the reference's physics code cannot be compiled in this
 * container (src/md_cuda_common.cu includes RAFT/RMM, src/md_env.cu needs MPI,
 * gDel2D and delaunator), and the reference ships no golden vectors or
 * known-answer tests for forces or integrators. The physics here is therefore
 * "parity unpinned" against the reference binary; it is pinned instead against
 * analytic known answers (two-particle forces/energies, lattice sums, Newton's
 * third law, FIRE two-particle minimum) in tests/test_oracle.py. The PFRAME
 * and config-JSON formats ARE pinned against the reference's own
 * src/md_common.cpp and src/md_config.cpp, compiled from the reference tree by
 * oracle/build_ref.py into oracle/_ref/ (tests/test_formats.py).
 *
 * Arithmetic modes:
 *  OR_FP64      every operation in double (the truth the force-error bound is
 *               stated against).
 *  OR_REF_MIXED the reference's arithmetic (src/md_cuda_common.cu:207-263): the
 *               FP64 displacement is cast to FP32, minimum image in FP32 with
 *               roundf, FP32 pair term, FP64 accumulation.
 * ws1_halo != 0 additionally reproduces the world-size-1 halo self-duplication
 * of the reference (src/md_env.cu:459-460, 801-805, 964-991;
 * src/md_cuda_common.cu:85-90): every partner within 1.2*cutoff*sigma_max of
 * x=0 or x=Lx is counted a second time. It only explains differences against
 * the reference binary at mpirun -np 1; it is not physics.
 *
 * FP64 integrator steps use explicit fma() with the operation order stated at
 * each function, which the CUDA kernels reproduce operation for operation.
 */
#ifndef MDORACLE_H
#define MDORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OR_FP64 = 0, OR_REF_MIXED = 1 };

typedef struct or_lj {
  double sigma[3];   /* AA, BB, AB */
  double epsilon[3]; /* AA, BB, AB */
  double mass_a;     /* type 0       */
  double mass_b;     /* every other  */
  double cutoff;     /* dimensionless, rc_ij = cutoff * sigma_ij */
} or_lj_t;

/* Forces (acc = F/m), shifted pair energy U and pair virial W, all pairs
 * (O(N^2), the reference's loop). pos: 2n doubles. */
int or_forces_allpairs(const or_lj_t* lj, int64_t n, const double* pos, const int32_t* type,
                       double Lx, double Ly, int32_t periodic_y, int32_t mode, int32_t ws1_halo,
                       double* acc, double* U, double* W, int32_t nthreads);
/* Same quantities through a cell list (cell width >= rc_max). Falls back to
 * all pairs when the grid is narrower than 3 cells. ws1_halo is not supported
 * here. */
int or_forces_cells(const or_lj_t* lj, int64_t n, const double* pos, const int32_t* type,
                    double Lx, double Ly, int32_t periodic_y, int32_t mode, double* acc,
                    double* U, double* W, int32_t nthreads);
/* The all-pairs loop of li_force_kernel for the rows [row0, row0+nrows)
 * only (acc_rows: 2*nrows doubles). A bounded sample of the reference's
 * O(N^2) force pass, used as the timed CPU baseline. */
int or_forces_rows(const or_lj_t* lj, int64_t n, const double* pos, const int32_t* type,
                   double Lx, double Ly, int32_t periodic_y, int32_t mode, int64_t row0,
                   int64_t nrows, double* acc_rows, int32_t nthreads);
/* MDSimulation::cal_partial_U_lambda (src/md_env.cu:2362-2406, kernel
 * src/md_cuda_common.cu:266-377) with the nearest image: out = sum over
 * ordered pairs of 1/2 * (-eps_lambda) * (Fx dx - Fy dy); scale (optional) =
 * the same sum of magnitudes. */
int or_partial_U_lambda(const or_lj_t* lj, int64_t n, const double* pos, const int32_t* type,
                        double Lx, double Ly, int32_t periodic_y, int32_t mode,
                        double epsilon_lambda, double* out, double* scale, int32_t nthreads);
/* get_N_profile at world size 1 (src/md_env.cu:3920-3985): per-type counts
 * in x bins, out[2*nb] = {type 0 | other types}. */
int or_n_profile(int64_t n, const double* pos, const int32_t* type, double Lx, int32_t nb,
                 int32_t* out);
/* get_pressure_profile (src/md_env.cu:3821-3918): Irving-Kirkwood profile
 * in y bins, out[3*nb] = {Pxx | Pyy | Pxy}, all pairs, nearest image. */
int or_pressure_profile(const or_lj_t* lj, int64_t n, const double* pos, const double* vel,
                        const int32_t* type, double Lx, double Ly, int32_t periodic_y,
                        int32_t mode, int32_t nb, double* out);
/* Per-thread values of the reference's block-reduced kernels, each in its
 * own accumulation order, with the same halos as or_forces_allpairs:
 *   OR_SUM_U    cal_local_U_kernel (src/md_cuda_common.cu:703-825)
 *   OR_SUM_P    cal_local_pressure_scalar_kernel (:591-701), m|v|^2 first
 *   OR_SUM_K    cal_local_K_kernel (:554-589)
 *   OR_SUM_DUDL cal_partial_U_lambda_kernel (:266-377) for eps_lambda
 * out: n doubles (thread i's value before the block reduction). */
enum { OR_SUM_U = 0, OR_SUM_P = 1, OR_SUM_K = 2, OR_SUM_DUDL = 3 };
int or_ref_thread_values(const or_lj_t* lj, int64_t n, const double* pos, const double* vel,
                         const int32_t* type, double Lx, double Ly, int32_t periodic_y,
                         int32_t mode, int32_t ws1_halo, int32_t what, double eps_lambda,
                         double* out, int32_t nthreads);
/* The shared-memory tree of those kernels over blocks of `threads` values
 * (threads past n add 0): partials[b] (optional), and their sum in block
 * order as the reference's host loops take it (the return value). */
double or_ref_block_partials(int64_t n, const double* v, int32_t threads, double* partials);
/* Ordered in-cutoff pairs counted through a cell list (large systems). */
int64_t or_count_pairs_cells(const or_lj_t* lj, int64_t n, const double* pos,
                             const int32_t* type, double Lx, double Ly, int32_t nthreads);
/* Number of ordered pairs (i != j) inside their cutoff (FP64 test). */
int64_t or_count_pairs(const or_lj_t* lj, int64_t n, const double* pos, const int32_t* type,
                       double Lx, double Ly, int32_t periodic_y, int32_t nthreads);

/* Project binning (the CUDA cell build must match it bit for bit). */
void or_cell_grid(double Lx, double Ly, double cell_min, int32_t* ncx, int32_t* ncy);
void or_cell_bin(int64_t n, const double* pos, double Lx, double Ly, int32_t ncx, int32_t ncy,
                 int32_t* cell);
void or_cell_sort(int64_t n, const int32_t* cell, int32_t ncells, int32_t* perm,
                  int32_t* cell_start);

double or_pbc_wrap(double x, double L);

/* ---- stateful engine mirroring MDSimulation's hot path ------------------ */
typedef struct or_sim {
  int64_t n;
  double* pos; /* 2n */
  double* vel; /* 2n */
  double* acc; /* 2n */
  int32_t* type;
  or_lj_t lj;
  double dt, Q, T_target;
  int64_t n_global;
  double barostat_mass, k_piston, area_rate_init, hmin_ratio, hmax_ratio;
  double Lx, Ly, Lx0, Ly0;
  double t, xi;
  double nph_area_momentum, nph_aspect_ratio;
  int32_t nph_state_initialized;
  double piston_velocity, piston_force;
  int32_t piston_velocity_initialized, piston_mode_active;
  double last_instant_pressure;
  int32_t mode;      /* OR_FP64 / OR_REF_MIXED */
  int32_t ws1_halo;  /* reproduce the ws=1 halo duplication */
  int32_t use_cells; /* cell list instead of all pairs */
  int32_t nthreads;
  int32_t error;     /* nonzero after an invalid box (reference: MPI_Abort) */
  int32_t ref_threads; /* > 0: K, U, P and wall sums through the reference's
                          block trees of this many threads, then block order
                          (bit-exact with its kernels); 0: sequential sums */
} or_sim_t;

/* Buffers are caller-owned; or_sim_setup fills the derived fields and computes
 * the initial forces (MDSimulation ctor: cal_forces, src/md_env.cu:61-79). */
void or_sim_setup(or_sim_t* s);
void or_sim_cal_forces(or_sim_t* s, int32_t periodic_y);
void or_step_nve(or_sim_t* s);
void or_step_nose_hoover(or_sim_t* s);
void or_step_nph(or_sim_t* s, double p_ext);
void or_step_nph_piston(or_sim_t* s, double p_ext);
double or_total_K(const or_sim_t* s);
double or_total_U(or_sim_t* s);
double or_instant_pressure(or_sim_t* s);
double or_scalar_pressure(or_sim_t* s, int32_t periodic_y);
/* piston_wall_kernel + evaluate_piston_wall_observables (src/md_cuda_common.cu:
 * 498-552, src/md_env.cu:2148-2203): upper-wall force and wall energy, and
 * with update_acc the wall force added to acc.y. */
void or_sim_piston_walls(or_sim_t* s, int32_t update_acc, double* upper, double* energy);

/* One of the reference's integrator kernels (src/md_cuda_common.cu:379-496)
 * in place on n particles (pos, vel: 2n; acc: 2n read only):
 * 0 step_half_vv (dt, Lx, Ly), 1 step_2nd_half_vv (dt),
 * 2 step_half_vv_nh (dt, xi, Lx, Ly), 3 step_2nd_half_vv_nh (dt, xi),
 * 4 step_half_nph_velocity (dt), 5 step_nph_scale_and_drift (dt, lin, vsc,
 * Lx, Ly = the new box), 6 step_half_vv_piston (dt, Lx). */
int or_ref_integrator(int32_t which, int64_t n, double* pos, double* vel, const double* acc,
                      double dt, double xi, double lin, double vsc, double Lx, double Ly);

/* ---- FIRE (EnergyMinimizer::minimize_frame) ----------------------------- */
typedef struct or_fire_params {
  double dt_init, dt_max, alpha0, f_inc, f_dec;
  int32_t N_min;
} or_fire_params_t;

typedef struct or_fire_result {
  int32_t steps, converged;
  double max_force, potential_energy;
  int64_t n_energy_samples;
} or_fire_result_t;

/* pos/vel/acc: 2n in/out (vel/acc overwritten as the reference does). */
int or_fire_minimize(const or_lj_t* lj, int64_t n, double* pos, double* vel, double* acc,
                     const int32_t* type, double Lx, double Ly, double force_tol,
                     int32_t max_steps, const or_fire_params_t* p, int32_t mode,
                     int32_t ws1_halo, int32_t use_cells, int32_t nthreads,
                     or_fire_result_t* res, int32_t* energy_steps, double* energy_trace,
                     int64_t trace_cap);

#ifdef __cplusplus
}
#endif

#endif
