// Internal structures shared by the host engine and the sm_100a kernels.
//
// Data layout in HBM (per batch; a single simulation is a batch of one):
//   particles of all systems are concatenated; system s owns the slots
//   [p0_s, p0_s + n_s) for its whole life. Inside that range the particles are
//   kept sorted by cell (re-sorted at every cell-list rebuild); orig[k] maps a
//   slot back to the caller's particle index.
//   SoA, FP64 state: pos/vel/acc double2 (16 B each), type int32, theta f64.
//   pff  float4 per slot: position as an exact float-float pair (hi, lo) in a
//        biased binade, hi parts' sign bits carry the type class. This is the
//        only array the pair loop gathers (16 B per candidate).
//   sb   float2 per slot: position at the last rebuild (fractional for periodic
//        axes, absolute for the piston's walled y axis).
//   cells: per system a grid of up to ccap_x*ccap_y cells; the global
//        exclusive scan cstart[] of per-cell counts gives each cell's slot
//        range directly because systems are laid out in order.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mdb {

constexpr int kThreads = 256;  // particle kernels: one particle per thread
constexpr double kSkinMD = 0.45;   // automatic list skin: MD systems
constexpr double kSkinFire = 0.2;  // automatic list skin: a handle of FIRE systems only
constexpr double kFireFp64Below = 1e-3;  // FIRE: FP64 pair terms below this max |a|
constexpr int kNP = 6;         // reduction slots per block
constexpr int kScanItems = 4;  // cells per thread in the scan kernels
constexpr int kScanBlock = 512;
constexpr int kScanTile = kScanItems * kScanBlock;
// ncount[] flag: the list needs neither the minimum image nor offset wrapping.
constexpr int32_t kListInterior = 1 << 30;
// Force phase: list rows of the next chunk prefetched into L1 per warp
// (built-in schedule; Dev::pf_rows holds the one in use).
constexpr int kListPrefetchRows = 28;
// With mdb_options_t.lanes = MDB_LANES_SPLIT, small MD systems (n <=
// kLanesMaxN) give each slot kLanes lanes of the force phase, which split its
// pair candidates; a block then covers kThreads / kLanes slots in every
// phase. FIRE systems keep one lane per slot.
constexpr int kLanes = 4;
constexpr int kLanesMaxN = 16384;
// MD calls of at least this many steps use the multi-step kernel where it is
// enabled (one step: 46 us in it against 36 us per phase at N = 4096).
constexpr int kMultiStepMinSteps = 4;

// Force-phase variants.
enum FMode : int32_t {
  FM_INIT = 0,    // acc = F/m (constructor / set_frame / piston entry)
  FM_NVE = 1,     // + second velocity-Verlet half kick
  FM_NH = 2,      // + Nose-Hoover second half kick, K reduction
  FM_NPH = 3,     // + virial, kinetic before/after kick, barostat half step
  FM_PISTON = 4,  // + soft walls, piston half step
  FM_FIRE = 5,    // + full kick, FIRE statistics and control
  FM_OBS = 6,     // no state change: U, virial, kinetic, wall terms
};

// Drift-phase variants.
enum DMode : int32_t { DM_NVE = 0, DM_NH = 1, DM_NPH = 2, DM_PISTON = 3, DM_FIRE = 4 };

// Job kinds of a batch system.
enum Kind : int32_t { K_FIRE = 0, K_NVE = 1, K_NVT = 2 };

struct SysParams {
  int64_t p0;     // first slot
  int64_t c0;     // first cell
  int32_t n;      // particles
  int32_t b0;     // first block of the block table
  int32_t nb;     // blocks
  int32_t items;  // particles per thread (a block covers kThreads*items slots)
  int32_t ccap_x, ccap_y;
  int32_t kind;
  int32_t lanes;  // lanes per slot in the force phase (1, or kLanes for small MD systems)
  float frl2[3];  // neighbour-list radius^2 per pair class: (rc_ij + skin)^2
  double sig[3], eps[3], Vc[3];  // AA, BB, AB
  double massA, massB, cutoff, rc_max, r_cell, skin;
  double dt, Q, T0, g_dof, W, k_piston, hmin, hmax, Lx0, Ly0, rate_init;
  double offx, offy;             // binade offsets of the float-float split
  float fsig2[3], feps24[3], feps4[3], frc2[3];
  // FIRE
  double f_dt_max, f_alpha0, f_inc, f_dec, f_tol;
  double f_hp_below;  // FP64 pair terms once max |a| < f_hp_below (< 0: never)
  int32_t f_Nmin, f_max_steps;
  int64_t target_steps;  // MD segment length (batches)
};

struct SysState {
  double Lx, Ly;
  double xi, K;                       // Nose-Hoover
  double pA, aspect, P_cur, last_P;   // NPH
  double fl, ce;                      // Ly clamp bounds
  double vp, Fp, wallU;               // piston
  double U, Wv, kin, kin2;            // last observable reductions
  double Wani;                        // 1/2 sum (Fx dx - Fy dy) of the last observation
  double p_ext;                       // external pressure of the running call
  double inv_wx, inv_wy, Lx_b, Ly_b;  // cell grid at the last rebuild
  int32_t ncx, ncy, allpairs, periodic_y;
  int32_t clamped, nph_init, piston_active, piston_init;
  uint32_t dmax_x, dmax_y, jump;      // float bits (non-negative)
  int32_t nl_overflow;                // particles whose list overflowed at the last rebuild
  int32_t need_rebuild;
  int32_t nonfinite;
  int32_t err;
  uint32_t counter;
  int32_t done;                        // finished job (batches)
  int64_t steps, rebuilds;
  // FIRE
  double f_dt, f_alpha, f_maxf, f_power;
  int32_t f_streak, f_conv, f_zero_v, f_step;
  int32_t f_conv_step;
  int32_t f_drift;  // the force phase of this iteration ran and did not converge
  int32_t f_fp64;   // FP64 pair terms for this system (FIRE and its observations)
  int32_t f_pad;
  // step (MD) or iteration (FIRE) counter at the last rebuild that the drift
  // asked for; a forced rebuild resets it to kNoRebuildYet
  int64_t rb_last;
};

// SysState::rb_last before any drift-requested rebuild.
constexpr int64_t kNoRebuildYet = -(int64_t(1) << 40);
// A rebuild builds the system's neighbour list only when its previous
// drift-requested rebuild is at least this many steps (iterations) back;
// otherwise its force phase scans the cell stencil until the next rebuild
// (a list rebuilt every step or two costs more than it saves).
constexpr int64_t kListMinReuse = 3;

struct BatchGlobal {
  int32_t any_rebuild;
  uint32_t sys_counter;
  int32_t nsys;
  int32_t all_done;
  int64_t steps_left;  // multi-step kernel: steps of the running call not yet done
  uint32_t bar_count;  // multi-step kernel: grid barrier arrivals
  uint32_t bar_gen;    //   and generation
  int32_t bar_err;     //   a barrier wait ran out of polls
  int32_t forced;      // the pending rebuild was forced (not asked for by a drift)
};

// The NPH driver protocol (run_test_NPH.cpp:137-290) run on the device: its
// parameters, clamped as the host protocol clamps them, and the loop state,
// advanced by a one-thread kernel after each iteration of a graph while loop
// (one decision step, a chunk of quiet steps, or the NPH entry).
struct NphProto {
  int64_t eval, auto_steps, window, stable_req, warm_min, warm_max, prod, hard, cap;
  double tol;
  double W, rate_init;  // barostat mass (>= 1e-12) and initial area rate
  double dt;            // time added per step (advance_time)
  double* win;          // window ring, `window` slots
  void* rec;            // mdb_nph_record_t[cap]
  double P_target, auto_sum, t;
  int64_t step, auto_done, warm_done, prod_done, stable, auto_n, nrec;
  int64_t auto_end, warm_end;
  int64_t win_n, win_head;  // samples in the window ring, slot of the oldest
  int64_t iters;            // while-loop iterations run
  int32_t phase;            // phase of the next step
  int32_t p_valid;          // S.P_cur holds the pressure of the current state
  int32_t nph_init;         // NPH area momentum and aspect initialised
  int32_t forced, finished, err;
  int32_t last_phase, last_sample;  // phase of the last step, whether it was sampled
  int32_t pending;          // what the body of the running iteration does
  int32_t pending_steps;    // its steps (quiet chunks)
  int32_t window_ok;        // stability test of the current window (quiet chunks)
  int32_t pad;
};

// Kernel argument block (passed by value).
struct Dev {
  const int32_t* sys_of_block;
  const int32_t* sysid;  // per slot
  const SysParams* sp;
  SysState* st;
  BatchGlobal* bg;
  double2 *pos, *vel, *acc;
  int32_t* type;
  double* theta;
  int32_t* orig;
  double2 *pos2, *vel2, *acc2;
  int32_t* type2;
  double* theta2;
  int32_t* orig2;
  float4* pff;
  float2* sb;
  int32_t* cell_of;
  int32_t* key;
  int32_t* perm;
  int32_t* nlist;     // neighbour list, offset j - i of entry k of slot i at
  int16_t* nlist16;   //   nlist[k * ntot + i] (int32) or nlist16[...] (int16)
  int32_t* ncount;    // list length per slot (| kListInterior), -1: use the cell stencil
  int32_t max_nbr;
  int32_t nl16;       // 1: 16-bit offsets (every stencil offset fits in int16)
  int32_t* ccount;
  int32_t* ccursor;
  int32_t* cstart;    // ncells + 1
  int32_t* scan_part; // per scan tile
  double* part;       // nblocks * kNP   block partial sums
  double* partm;      // nblocks * 4     block partial maxima
  int32_t nsys;
  int32_t nblocks;
  int64_t ntot;
  int64_t ncells;
  cudaGraphConditionalHandle cond;
  int32_t use_cond;
  int32_t rb_grid;    // grid of the grid-stride rebuild kernels
  int32_t pf_rows;    // force phase: list rows of the next chunk prefetched per warp
};

}  // namespace mdb
