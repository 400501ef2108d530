// Host engine: owns the device memory of a batch of independent systems (a
// single simulation is a batch of one) and issues the step phases.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "mdb200.h"
#include "mdb_internal.h"

namespace mdb {

struct SystemSpec {
  mdb_config_t cfg;
  std::vector<mdb_particle_t> frame;
  int32_t kind = K_NVE;
  mdb_fire_params_t fire{};
  double tol = 0.0;
  int32_t max_steps = 0;
  int64_t target_steps = 0;
  bool fire_prepare = false;  // wrap positions, zero v and a (FIRE entry)
};

class Engine {
 public:
  explicit Engine(const mdb_options_t& opt);
  ~Engine();
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;

  int add_system(SystemSpec&& spec);
  // Allocates and uploads every added system, then builds the cell lists.
  int build();

  int nsys() const { return (int)specs_.size(); }
  int64_t n(int s) const { return (int64_t)specs_[s].frame.size(); }
  const SysParams& params(int s) const { return hsp_[s]; }
  cudaStream_t stream() const { return stream_; }
  bool graphs() const { return use_graphs_; }
  int device() const { return device_; }

  // nsteps x { drift(dm) ; rebuild if needed ; force(fm) }
  int run_md(int dm, int fm, bool py, int64_t nsteps);
  // Same steps issued eagerly with CUDA events around each phase on the
  // engine's stream; ms[0..2] receive the summed drift / rebuild / force time.
  int run_md_timed(int dm, int fm, bool py, int64_t nsteps, double* ms);
  // iters x { force(FIRE) ; drift(FIRE) ; rebuild if needed }
  int run_fire(int64_t iters);
  // One force-phase launch (FM_INIT / FM_OBS).
  int force(int fm, bool py);
  int reduce_K();
  // Flags every system for a rebuild (periodic_y >= 0 also switches the y
  // convention) and runs the rebuild pipeline now.
  int rebuild_now(int periodic_y);
  int set_pext(double p);

  int get_state(int s, SysState* out);
  int get_states(std::vector<SysState>& out);
  int put_state(int s, const SysState& st);
  int get_frame(int s, mdb_particle_t* out);
  int set_frame(int s, const mdb_particle_t* in);
  // Queues the export of system s's frame (caller's particle order) into
  // `host` on the engine's stream and returns without waiting; `host` should
  // be pinned memory for the copy to be asynchronous.
  int export_async(int s, mdb_particle_t* host);
  // Queues the observables of system s (time t and the piston flag come from
  // the caller) into `host` on the engine's stream; does not wait.
  int observables_async(int s, double t, int piston_active, mdb_observables_t* host);
  // Per-type x-bin counts (2*nb ints) and unnormalised Irving-Kirkwood sums
  // in y bins (3*nb doubles: xx | yy | xy) of system s; py selects the y
  // convention of the engine's current cell binning.
  int profiles(int s, int nb, bool py, double* ptens, int32_t* counts);
  // Slot -> original index and slot -> local cell of system s (n entries each).
  int debug_cells(int s, int32_t* orig, int32_t* cell);
  int sync();
  // Whether every issued kernel and copy of the engine's stream has finished
  // (does not wait).
  int idle(bool* out);
  // Device memory the engine holds, in bytes.
  int64_t device_bytes() const { return bytes_; }
  // The schedule in use (built in, or chosen by the autotuner at build).
  const mdb_schedule_t& schedule() const { return schedule_; }

  // Kernel launches issued (eager launches + kernel nodes of launched graphs,
  // counting the rebuild body once per rebuild actually run).
  long long launches_issued() const { return launches_; }
  // Times the host has blocked on the engine's stream (state and frame reads,
  // sync()); the destructor's final wait is not counted.
  long long host_waits() const { return host_waits_; }

  // The NPH driver protocol of a single system in one graph launch. A while
  // node runs one step per iteration; a switch node picks the Nose-Hoover
  // body, the NPH body, or the NPH body preceded by the NPH entry (pressure
  // observation and barostat initialisation); a one-thread kernel takes the
  // protocol's decisions on the device after each step and writes the
  // records; steps between two decision points run as quiet chunks of 64, 8
  // or 1 steps. q holds the parameters and the initial loop state on entry
  // and the final loop state on return; rec receives min(q->nrec, cap)
  // records. The host waits at most twice, both after the last step.
  int run_nph_protocol(NphProto* q, mdb_nph_record_t* rec, int64_t cap);

 private:
  int ensure_device();
  int launch(void* fn, int grid, int block, const Dev& d);
  int launch_rebuild_eager();
  int add_kernel_node(cudaGraph_t g, const cudaGraphNode_t* deps, int ndeps, void* fn, int grid,
                      int block, const Dev& d, cudaGraphNode_t* out);
  int add_rebuild_body(cudaGraph_t body, const Dev& d);
  int add_cond_rebuild(cudaGraph_t g, cudaGraphNode_t dep, cudaGraphConditionalHandle h,
                       cudaGraphNode_t* out);
  int get_graph(int kind, int dm, int fm, bool py, int chunk, cudaGraphExec_t* exec);
  // Times the schedule candidates on the built state (every candidate leaves
  // the state bit for bit as it was) and keeps the fastest; cached per device
  // and workload shape.
  int tune();
  int time_force(int fm, int reps, double* ms);
  int time_rebuild(int reps, double* ms);
  void drop_graphs();
  // The cached protocol graph (built at the first protocol run).
  int proto_graph(cudaGraphExec_t* exec);
  // Whether MD steps run in the multi-step kernel (single system, all
  // blocks resident), and its cached graph per drift/force mode.
  int choose_multi_step();
  int get_steps_graph(int dm, int fm, cudaGraphExec_t* exec);
  void free_proto();
  cudaError_t wait_host() {
    ++host_waits_;
    return cudaStreamSynchronize(stream_);
  }

  int device_ = 0;
  double skin_ = 0.0;
  int max_nbr_ = 48;
  bool use_graphs_ = true;
  bool built_ = false;
  cudaStream_t stream_ = nullptr;
  std::vector<SystemSpec> specs_;
  std::vector<SysParams> hsp_;
  Dev dev_{};
  int64_t ntot_ = 0, ncells_ = 0;
  int nblocks_ = 0;
  int rb_grid_ = 0;
  int scan_grid_ = 0;
  int nlist_grid_ = 0;  // k_rb_nlist: one wave of resident blocks
  int fire_prec_ = MDB_FIRE_AUTO;
  int autotune_ = 0;
  int step_kernel_ = MDB_STEPS_AUTO;
  bool multi_step_ = false;
  bool lanes_ = false;  // some system has several lanes per slot (SysParams::lanes)
  int lanes_opt_ = MDB_LANES_ONE;  // mdb_options_t.lanes (AUTO counts as ONE here)
  int multi_cap_ = 0;  // blocks of the multi-step kernel the device holds at once
  mdb_schedule_t schedule_{};
  int stream_priority_ = 0;  // levels above normal for stream_
  int64_t aos_cap_ = 0;
  void* d_aos_ = nullptr;
  void* d_obs_ = nullptr;  // one mdb_observables_t staging slot
  std::vector<void*> allocs_;
  std::map<std::tuple<int, int, int, int, int>, std::pair<cudaGraph_t, cudaGraphExec_t>> graphs_;
  long long launches_ = 0;
  long long host_waits_ = 0;
  NphProto* d_proto_ = nullptr;  // protocol loop state (address baked into its graph)
  double* proto_win_ = nullptr;
  void* proto_rec_ = nullptr;
  int64_t proto_win_cap_ = 0, proto_rec_cap_ = 0;
  int64_t bytes_ = 0;
  long long last_rebuilds_ = 0;
};

// Kernel of a force phase (FM_*; py: periodic y) and of a drift phase (DM_*);
// ln: the launch holds systems with several lanes per slot.
void* force_fn(int fm, bool py, bool ln);
void* drift_fn(int dm, bool ln);

int reference_initial_frame(const mdb_config_t& cfg, std::vector<mdb_particle_t>& out);

// For the trajectory writer: queue the export of a simulation's frame into
// `host` and record `ev` after it on the simulation's stream.
int sim_export_async(mdb_sim_t* sim, mdb_particle_t* host, cudaEvent_t ev);
int64_t sim_particles(mdb_sim_t* sim);
int sim_device(mdb_sim_t* sim);
// The NPH driver protocol of a simulation in one graph launch (the decisions
// on the device); host_waits receives the host's blocking waits it took.
int sim_run_nph_protocol_graph(mdb_sim_t* sim, const mdb_nph_protocol_t& p,
                               mdb_nph_record_t* rec, int64_t cap, mdb_nph_result_t* res);
// Blocking waits of the host on the simulation's stream so far.
long long sim_host_waits(mdb_sim_t* sim);
// Whether the simulation issues its steps as CUDA graphs.
bool sim_uses_graphs(mdb_sim_t* sim);

}  // namespace mdb
