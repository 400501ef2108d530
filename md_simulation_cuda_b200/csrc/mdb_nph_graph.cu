// The NPH driver protocol of the reference's NPH test driver
// (tests/run_NPH_test/run_test_NPH.cpp:137-290) as one graph launch.
//
// Graph:  while (h_while) {
//           switch (h_case) {
//             NH1 / NPH1:   drift -> if (rebuild) rebuild -> force       (one step)
//             NH8 / NPH8:   8 such steps          (quiet chunks: no sample or
//             NH64 / NPH64: 64 such steps          decision falls inside)
//             ENTER:        force OBS -> k_proto_enter   (NPH entry, no step)
//             other:        nothing (the first iteration)
//           }
//           if (h_obs) force OBS      (AUTO_TARGET sample: cal_instant_pressure)
//           k_proto_step              (the driver's logic, then the next body)
//         }
// k_proto_step first accounts for what the iteration's body did: a decision
// step runs the driver's loop body (pressure sample, phase counters,
// AUTO_TARGET mean, rolling window and its stability test, phase switches,
// record); a quiet chunk advances the counters only, as the host-driven form
// does for the steps between two decision points. It then plans the next body
// with the host-driven form's chunk rule and sets the condition values. Every
// FP64 expression is the one the host protocol evaluates, in the same order
// (the library is built with --fmad=false, so no product is fused into a
// sum), so the two forms give the same bits.
#include <math.h>
#include <string.h>

#include "mdb_engine.h"
#include "mdb_util.h"

namespace mdb {

namespace {

enum { PH_AUTO = 0, PH_WARMUP = 1, PH_PRODUCTION = 2 };
// bodies of the switch node
enum { B_NH1 = 0, B_NPH1, B_NH8, B_NPH8, B_NH64, B_NPH64, B_ENTER, B_COUNT, B_NONE = 255 };
// what the body of the running iteration does
enum { P_NONE = 0, P_ENTER = 1, P_STEP = 2, P_QUIET = 3 };

constexpr int kProtoKey = 2;  // graph cache key kind of the protocol graph

struct ProtoArgs {
  NphProto* q;
  SysState* st;  // the system's state (a single system)
  cudaGraphConditionalHandle h_while, h_case, h_obs;
};

__device__ int64_t lmin(int64_t a, int64_t b) { return a < b ? a : b; }

__device__ double tol_den(double p) {
  // std::max(1e-12, fabs(P_target))
  const double a = fabs(p);
  return (1e-12 < a) ? a : 1e-12;
}

// compute_stats (run_test_NPH.cpp:36-56): window mean and sample standard
// deviation, summed from the oldest sample on.
__device__ void window_stats(const NphProto& q, double* mean, double* sd) {
  *mean = 0.0;
  *sd = 0.0;
  if (q.win_n == 0) return;
  double s = 0.0;
  for (int64_t k = 0; k < q.win_n; ++k) s += q.win[(q.win_head + k) % q.window];
  const double m = s / (double)q.win_n;
  *mean = m;
  if (q.win_n <= 1) return;
  double var = 0.0;
  for (int64_t k = 0; k < q.win_n; ++k) {
    const double d = q.win[(q.win_head + k) % q.window] - m;
    var += d * d;
  }
  *sd = sqrt(var / (double)(q.win_n - 1));
}

__device__ bool window_within(const NphProto& q) {
  double m, sd;
  window_stats(q, &m, &sd);
  const double den = tol_den(q.P_target);
  return fabs(m - q.P_target) / den <= q.tol && sd / den <= q.tol;
}

// The entry of an NPH step after a non-NPH one (mdb_sim_step_nph): the
// scalar pressure of the current state (after the force OBS pass of the
// body) and, once per simulation, init_nph_state_if_needed
// (src/md_env.cu:1757-1778).
__global__ void k_proto_enter(ProtoArgs a) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  NphProto& q = *a.q;
  SysState& S = *a.st;
  if (!q.nph_init) {
    if (!(S.Lx > 0.0) || !(S.Ly > 0.0)) {
      q.err = MDB_ERR_BOX;
      return;
    }
    S.aspect = S.Lx / S.Ly;
    S.pA = q.W * q.rate_init;
    q.nph_init = 1;
  }
  if (!q.p_valid) {
    const double A = S.Lx * S.Ly;
    S.P_cur = (A > 0.0) ? (S.kin + S.Wv) / (2.0 * A) : 0.0;
    q.p_valid = 1;
  }
}

// One step with the driver's loop body after it (run_test_NPH.cpp:160-285).
__device__ void decision_step(NphProto& q, SysState& S) {
  const int used = q.phase;
  const int64_t step = q.step;
  const bool sample = (step % q.eval) == 0;
  double P_inst = 0.0;
  if (sample) {
    if (used == PH_AUTO) {
      // cal_instant_pressure: the force OBS pass of this iteration has run
      const double A = S.Lx * S.Ly;
      S.last_P = (A > 0.0) ? (S.kin + S.Wv) / (2.0 * A) : 0.0;
      S.P_cur = S.last_P;
    }
    P_inst = S.last_P;  // get_last_instant_pressure in the NPH phases
  }
  q.p_valid = (used == PH_AUTO) ? (sample ? 1 : 0) : 1;
  q.t += q.dt;
  if (used == PH_AUTO)
    ++q.auto_done;
  else if (used == PH_WARMUP)
    ++q.warm_done;
  else
    ++q.prod_done;
  if (sample) {
    if (used == PH_AUTO) {
      q.auto_sum += P_inst;
      ++q.auto_n;
    } else if (q.win_n < q.window) {
      q.win[(q.win_head + q.win_n) % q.window] = P_inst;
      ++q.win_n;
    } else {  // push_back, then pop_front
      q.win[q.win_head] = P_inst;
      q.win_head = (q.win_head + 1) % q.window;
    }
  }
  if (used == PH_AUTO && q.auto_done >= q.auto_steps && q.auto_n > 0) {
    q.P_target = q.auto_sum / (double)q.auto_n;
    q.phase = PH_WARMUP;
    q.win_n = 0;
    q.win_head = 0;
    q.stable = 0;
    q.auto_end = step;
  }
  if (used == PH_WARMUP) {
    if (q.warm_done >= q.warm_min && q.win_n >= q.window) {
      q.stable = window_within(q) ? q.stable + 1 : 0;
      if (q.stable >= q.stable_req) {
        q.phase = PH_PRODUCTION;
        q.warm_end = step;
      }
    }
    if (q.phase == PH_WARMUP && q.warm_done >= q.warm_max) {
      q.phase = PH_PRODUCTION;
      q.warm_end = step;
      q.forced = 1;
    }
  }
  if (used == PH_PRODUCTION && q.prod_done >= q.prod) q.finished = 1;
  if (sample && q.nrec < q.cap) {
    mdb_nph_record_t& r = ((mdb_nph_record_t*)q.rec)[q.nrec];
    memset(&r, 0, sizeof(r));
    r.step = step;
    r.phase = used;
    r.P_inst = P_inst;
    r.P_target = q.P_target;
    double m, sd;
    window_stats(q, &m, &sd);
    r.mean = m;
    r.stddev = sd;
    r.rel_err = fabs(m - q.P_target) / tol_den(q.P_target);
    r.t = q.t;
    r.Lx = S.Lx;
    r.Ly = S.Ly;
    r.dA_dt = (used == PH_AUTO) ? 0.0 : S.pA / q.W;
  }
  if (sample) ++q.nrec;
  ++q.step;
  q.last_phase = used;
  q.last_sample = sample ? 1 : 0;
}

// c quiet steps: the counters only (the stability test gives the same answer
// on each of them, the window does not change).
__device__ void quiet_steps(NphProto& q, int64_t c) {
  const int used = q.phase;
  for (int64_t k = 0; k < c; ++k) q.t += q.dt;
  q.step += c;
  if (used == PH_AUTO) {
    q.auto_done += c;
  } else if (used == PH_WARMUP) {
    if (q.warm_done + c >= q.warm_min && q.win_n >= q.window)
      q.stable = q.window_ok ? q.stable + c : 0;
    q.warm_done += c;
  } else {
    q.prod_done += c;
  }
  q.p_valid = (used == PH_AUTO) ? 0 : 1;
  q.last_phase = used;
  q.last_sample = 0;
}

// Steps before the next point where the protocol samples or decides (the
// host-driven form's chunk rule); window_ok receives the warmup test result.
__device__ int64_t quiet_run(const NphProto& q, int* window_ok) {
  const int64_t step = q.step;
  const int64_t next_sample = (step % q.eval == 0) ? step : step + (q.eval - step % q.eval);
  int64_t k = next_sample - step;
  *window_ok = 0;
  if (q.phase == PH_AUTO) {
    k = lmin(k, q.auto_steps - q.auto_done - 1);
  } else if (q.phase == PH_WARMUP) {
    k = lmin(k, q.warm_max - q.warm_done - 1);
    if (q.warm_done + 1 < q.warm_min) {
      k = lmin(k, q.warm_min - q.warm_done - 1);
    } else if (q.win_n >= q.window) {
      *window_ok = window_within(q) ? 1 : 0;
      if (*window_ok) k = lmin(k, q.stable_req - q.stable - 1);
    }
  } else {
    k = lmin(k, q.prod - q.prod_done - 1);
  }
  k = lmin(k, q.hard - step - 1);
  return k > 0 ? k : 0;
}

__global__ void k_proto_step(ProtoArgs a) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  NphProto& q = *a.q;
  SysState& S = *a.st;
  if (q.pending == P_STEP)
    decision_step(q, S);
  else if (q.pending == P_QUIET)
    quiet_steps(q, q.pending_steps);
  ++q.iters;
  if (S.err != 0 && q.err == 0) q.err = S.err;
  const bool more = !q.finished && q.step < q.hard && q.err == 0;
  if (more) {
    const bool nph = q.phase != PH_AUTO;
    int body, obs = 0;
    if (nph) S.p_ext = q.P_target;  // set_pext before every NPH call
    if (nph && (!q.nph_init || !q.p_valid)) {
      q.pending = P_ENTER;
      body = B_ENTER;
    } else {
      int ok;
      const int64_t k = quiet_run(q, &ok);
      if (k > 0) {
        const int c = k >= 64 ? 64 : (k >= 8 ? 8 : 1);
        q.pending = P_QUIET;
        q.pending_steps = c;
        q.window_ok = ok;
        body = (c == 64) ? B_NH64 : (c == 8) ? B_NH8 : B_NH1;
      } else {
        q.pending = P_STEP;
        body = B_NH1;
        obs = (!nph && q.step % q.eval == 0) ? 1 : 0;
      }
      if (nph) body += 1;  // the NPH twin of the Nose-Hoover body
    }
    cudaGraphSetConditional(a.h_case, (unsigned)body);
    cudaGraphSetConditional(a.h_obs, (unsigned)obs);
  } else {
    q.pending = P_NONE;
  }
  cudaGraphSetConditional(a.h_while, more ? 1u : 0u);
}

}  // namespace

int Engine::proto_graph(cudaGraphExec_t* exec) {
  auto key = std::make_tuple(kProtoKey, 0, 0, 1, 0);
  auto it = graphs_.find(key);
  if (it != graphs_.end()) {
    *exec = it->second.second;
    return MDB_OK;
  }
  cudaGraph_t g = nullptr;
  MDB_CUDA(cudaGraphCreate(&g, 0));
  int rc = MDB_OK;
  auto ck = [&](cudaError_t e, const char* what) {
    if (rc == MDB_OK && e != cudaSuccess) rc = cuda_error(e, what);
    return rc == MDB_OK;
  };
  ProtoArgs pa{};
  pa.q = d_proto_;
  pa.st = dev_.st;
  // The first iteration runs no body: k_proto_step plans the first one.
  ck(cudaGraphConditionalHandleCreate(&pa.h_while, g, 1, cudaGraphCondAssignDefault), "handle");
  ck(cudaGraphConditionalHandleCreate(&pa.h_case, g, B_NONE, cudaGraphCondAssignDefault),
     "handle");
  ck(cudaGraphConditionalHandleCreate(&pa.h_obs, g, 0, cudaGraphCondAssignDefault), "handle");
  auto add_cond = [&](cudaGraph_t parent, const cudaGraphNode_t* dep, cudaGraphConditionalHandle h,
                      cudaGraphConditionalNodeType type, unsigned size, cudaGraphNode_t* node,
                      cudaGraph_t* bodies) {
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = type;
    cp.conditional.size = size;
    if (ck(cudaGraphAddNode(node, parent, dep, dep ? 1 : 0, &cp), "cudaGraphAddNode(conditional)"))
      for (unsigned k = 0; k < size; ++k) bodies[k] = cp.conditional.phGraph_out[k];
  };
  auto add_proto_kernel = [&](cudaGraph_t parent, const cudaGraphNode_t* dep, void* fn,
                              cudaGraphNode_t* node) {
    void* args[] = {&pa};
    cudaKernelNodeParams kp = {};
    kp.func = fn;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(32);
    kp.kernelParams = args;
    ck(cudaGraphAddKernelNode(node, parent, dep, dep ? 1 : 0, &kp), "cudaGraphAddKernelNode");
  };
  cudaGraphNode_t nwhile, nswitch, nobs_if, nstep;
  cudaGraph_t body = nullptr, cases[B_COUNT] = {}, obs_body = nullptr;
  add_cond(g, nullptr, pa.h_while, cudaGraphCondTypeWhile, 1, &nwhile, &body);
  if (rc == MDB_OK)
    add_cond(body, nullptr, pa.h_case, cudaGraphCondTypeSwitch, B_COUNT, &nswitch, cases);
  for (int b = 0; b < B_COUNT && rc == MDB_OK; ++b) {
    cudaGraph_t cg = cases[b];
    if (b == B_ENTER) {
      cudaGraphNode_t nobs, nenter;
      rc = add_kernel_node(cg, nullptr, 0, force_fn(FM_OBS, true, lanes_), nblocks_, kThreads, dev_, &nobs);
      if (rc == MDB_OK) add_proto_kernel(cg, &nobs, (void*)k_proto_enter, &nenter);
      continue;
    }
    const bool nph = (b % 2) == 1;
    const int steps = (b < B_NH8) ? 1 : (b < B_NH64) ? 8 : 64;
    cudaGraphNode_t prev = nullptr;
    for (int k = 0; k < steps && rc == MDB_OK; ++k) {
      cudaGraphConditionalHandle hr;
      if (!ck(cudaGraphConditionalHandleCreate(&hr, g, 0, 0), "handle")) break;
      Dev dd = dev_;
      dd.cond = hr;
      dd.use_cond = 1;
      cudaGraphNode_t nd, nc, nf;
      rc = add_kernel_node(cg, prev ? &prev : nullptr, prev ? 1 : 0,
                           drift_fn(nph ? DM_NPH : DM_NH, lanes_), nblocks_, kThreads, dd, &nd);
      if (rc == MDB_OK) rc = add_cond_rebuild(cg, nd, hr, &nc);
      if (rc == MDB_OK)
        rc = add_kernel_node(cg, &nc, 1, force_fn(nph ? FM_NPH : FM_NH, true, lanes_), nblocks_, kThreads,
                             dev_, &nf);
      prev = nf;
    }
  }
  if (rc == MDB_OK)
    add_cond(body, &nswitch, pa.h_obs, cudaGraphCondTypeIf, 1, &nobs_if, &obs_body);
  if (rc == MDB_OK) {
    cudaGraphNode_t nobs;
    rc = add_kernel_node(obs_body, nullptr, 0, force_fn(FM_OBS, true, lanes_), nblocks_, kThreads, dev_,
                         &nobs);
  }
  if (rc == MDB_OK) add_proto_kernel(body, &nobs_if, (void*)k_proto_step, &nstep);
  cudaGraphExec_t ex = nullptr;
  if (rc == MDB_OK) ck(cudaGraphInstantiate(&ex, g, 0), "cudaGraphInstantiate(protocol)");
  if (rc != MDB_OK) {
    cudaGraphDestroy(g);
    return rc;
  }
  graphs_[key] = std::make_pair(g, ex);
  *exec = ex;
  return MDB_OK;
}

int Engine::run_nph_protocol(NphProto* q, mdb_nph_record_t* rec, int64_t cap) {
  if (!built_) return set_error(MDB_ERR_STATE, "engine not built");
  if (nsys() != 1) return set_error(MDB_ERR_STATE, "the NPH protocol runs on a single system");
  if (!q || cap < 0 || (cap > 0 && !rec) || q->window < 1 || q->eval < 1)
    return set_error(MDB_ERR_ARG, "bad protocol arguments");
  MDB_CUDA(cudaSetDevice(device_));
  // device buffers: the loop state (its address is baked into the cached
  // graph), the window ring and the records (grown on demand)
  if (!d_proto_) {
    MDB_CUDA(cudaMalloc((void**)&d_proto_, sizeof(NphProto)));
    bytes_ += sizeof(NphProto);
  }
  if (proto_win_cap_ < q->window) {
    if (proto_win_) {
      MDB_CUDA(wait_host());  // an earlier run may still read the old ring
      cudaFree(proto_win_);
    }
    proto_win_ = nullptr;
    proto_win_cap_ = 0;
    MDB_CUDA(cudaMalloc((void**)&proto_win_, sizeof(double) * (size_t)q->window));
    proto_win_cap_ = q->window;
  }
  const int64_t rc_cap = cap > 0 ? cap : 1;
  if (proto_rec_cap_ < rc_cap) {
    if (proto_rec_) {
      MDB_CUDA(wait_host());
      cudaFree(proto_rec_);
    }
    proto_rec_ = nullptr;
    proto_rec_cap_ = 0;
    MDB_CUDA(cudaMalloc(&proto_rec_, sizeof(mdb_nph_record_t) * (size_t)rc_cap));
    proto_rec_cap_ = rc_cap;
  }
  q->cap = cap;
  q->win = proto_win_;
  q->rec = proto_rec_;
  q->pending = P_NONE;
  q->iters = 0;
  cudaGraphExec_t ex;
  const int grc = proto_graph(&ex);
  if (grc != MDB_OK) return grc;
  MDB_CUDA(cudaMemcpyAsync(d_proto_, q, sizeof(NphProto), cudaMemcpyHostToDevice, stream_));
  MDB_CUDA(cudaGraphLaunch(ex, stream_));
  MDB_CUDA(cudaMemcpyAsync(q, d_proto_, sizeof(NphProto), cudaMemcpyDeviceToHost, stream_));
  MDB_CUDA(wait_host());
  // kernels: two per step, the protocol kernel per iteration (the conditional
  // rebuild bodies and observation passes are not counted, as in run_md)
  launches_ += 2LL * q->step + q->iters;
  count_launches(2LL * q->step + q->iters);
  const int64_t nr = q->nrec < cap ? q->nrec : cap;
  if (nr > 0) {
    MDB_CUDA(cudaMemcpyAsync(rec, proto_rec_, sizeof(mdb_nph_record_t) * (size_t)nr,
                             cudaMemcpyDeviceToHost, stream_));
    MDB_CUDA(wait_host());
  }
  return MDB_OK;
}

void Engine::free_proto() {
  if (d_proto_) cudaFree(d_proto_);
  if (proto_win_) cudaFree(proto_win_);
  if (proto_rec_) cudaFree(proto_rec_);
  d_proto_ = nullptr;
  proto_win_ = nullptr;
  proto_rec_ = nullptr;
  proto_win_cap_ = proto_rec_cap_ = 0;
}

}  // namespace mdb
