// The NPH driver protocol of the reference's NPH test driver
// (tests/run_NPH_test/run_test_NPH.cpp:137-290) as one graph launch.
//
// Graph:  while (h_while) {
//           switch (h_case) {
//             0: drift NH    -> if (rebuild) rebuild -> force NH
//             1: drift NPH   -> if (rebuild) rebuild -> force NPH
//             2: force OBS -> k_proto_enter -> drift NPH -> if (rebuild) ... -> force NPH
//           }
//           if (h_obs) force OBS          (AUTO_TARGET sample: cal_instant_pressure)
//           k_proto_step                  (the driver's per-step logic)
//         }
// k_proto_step runs the loop body of the driver after the step: the pressure
// sample, the phase counters, the AUTO_TARGET mean, the rolling window and its
// stability test, the phase switches and the record. It then sets the three
// condition values for the next iteration. Every FP64 expression is the one
// the host protocol evaluates, in the same order (the library is built with
// --fmad=false, so no product is fused into a sum), so the two give the same
// bits.
#include <math.h>
#include <string.h>

#include "mdb_engine.h"
#include "mdb_util.h"

namespace mdb {

namespace {

enum { PH_AUTO = 0, PH_WARMUP = 1, PH_PRODUCTION = 2 };
// bodies of the per-step switch node
enum { CASE_NH = 0, CASE_NPH = 1, CASE_NPH_ENTER = 2 };

struct ProtoArgs {
  NphProto* q;
  double* win;            // window ring, q->window slots
  mdb_nph_record_t* rec;  // q->cap records
  SysState* st;           // the system's state (a single system)
  cudaGraphConditionalHandle h_while, h_case, h_obs;
};

__device__ double tol_den(double p) {
  // std::max(1e-12, fabs(P_target))
  const double a = fabs(p);
  return (1e-12 < a) ? a : 1e-12;
}

// compute_stats (run_test_NPH.cpp:36-56): window mean and sample standard
// deviation, summed from the oldest sample on.
__device__ void window_stats(const NphProto& q, const double* win, double* mean, double* sd) {
  *mean = 0.0;
  *sd = 0.0;
  if (q.win_n == 0) return;
  double s = 0.0;
  for (int64_t k = 0; k < q.win_n; ++k) s += win[(q.win_head + k) % q.window];
  const double m = s / (double)q.win_n;
  *mean = m;
  if (q.win_n <= 1) return;
  double var = 0.0;
  for (int64_t k = 0; k < q.win_n; ++k) {
    const double d = win[(q.win_head + k) % q.window] - m;
    var += d * d;
  }
  *sd = sqrt(var / (double)(q.win_n - 1));
}

__device__ void set_next(const ProtoArgs& a, const NphProto& q, SysState& S) {
  int c = CASE_NH;
  if (q.phase != PH_AUTO) {
    S.p_ext = q.P_target;  // set_pext before every NPH step
    c = (!q.nph_init || !q.p_valid) ? CASE_NPH_ENTER : CASE_NPH;
  }
  cudaGraphSetConditional(a.h_case, (unsigned)c);
  cudaGraphSetConditional(a.h_obs, (q.phase == PH_AUTO && q.step % q.eval == 0) ? 1u : 0u);
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
      S.err = MDB_ERR_BOX;  // the step's kernels skip the system
      return;
    }
    S.aspect = S.Lx / S.Ly;
    S.pA = q.W * q.rate_init;
    q.nph_init = 1;
  }
  if (!q.p_valid) {
    const double A = S.Lx * S.Ly;
    S.P_cur = (A > 0.0) ? (S.kin + S.Wv) / (2.0 * A) : 0.0;
  }
}

// The driver's loop body after the step of the iteration
// (run_test_NPH.cpp:160-285).
__global__ void k_proto_step(ProtoArgs a) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  NphProto& q = *a.q;
  SysState& S = *a.st;
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
    } else {
      if (q.win_n < q.window) {
        a.win[(q.win_head + q.win_n) % q.window] = P_inst;
        ++q.win_n;
      } else {  // push_back then pop_front
        a.win[q.win_head] = P_inst;
        q.win_head = (q.win_head + 1) % q.window;
      }
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
      double m, sd;
      window_stats(q, a.win, &m, &sd);
      const double den = tol_den(q.P_target);
      const bool ok = fabs(m - q.P_target) / den <= q.tol && sd / den <= q.tol;
      q.stable = ok ? q.stable + 1 : 0;
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
    mdb_nph_record_t& r = a.rec[q.nrec];
    memset(&r, 0, sizeof(r));
    r.step = step;
    r.phase = used;
    r.P_inst = P_inst;
    r.P_target = q.P_target;
    double m, sd;
    window_stats(q, a.win, &m, &sd);
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
  if (S.err != 0 && q.err == 0) q.err = S.err;
  const bool more = !q.finished && q.step < q.hard && q.err == 0;
  set_next(a, q, S);
  cudaGraphSetConditional(a.h_while, more ? 1u : 0u);
}

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

}  // namespace

int Engine::run_nph_protocol(NphProto* q, mdb_nph_record_t* rec, int64_t cap) {
  if (!built_) return set_error(MDB_ERR_STATE, "engine not built");
  if (nsys() != 1) return set_error(MDB_ERR_STATE, "the NPH protocol runs on a single system");
  if (!q || cap < 0 || (cap > 0 && !rec) || q->window < 1 || q->eval < 1)
    return set_error(MDB_ERR_ARG, "bad protocol arguments");
  MDB_CUDA(cudaSetDevice(device_));
  q->cap = cap;
  DevBuf bq, bw, br;
  MDB_CUDA(cudaMalloc(&bq.p, sizeof(NphProto)));
  MDB_CUDA(cudaMalloc(&bw.p, sizeof(double) * (size_t)q->window));
  MDB_CUDA(cudaMalloc(&br.p, sizeof(mdb_nph_record_t) * (size_t)(cap > 0 ? cap : 1)));
  MDB_CUDA(cudaMemcpyAsync(bq.p, q, sizeof(NphProto), cudaMemcpyHostToDevice, stream_));

  ProtoArgs pa{};
  pa.q = (NphProto*)bq.p;
  pa.win = (double*)bw.p;
  pa.rec = (mdb_nph_record_t*)br.p;
  pa.st = dev_.st;

  // Condition values of the first iteration are the handles' defaults.
  int c0 = CASE_NH;
  if (q->phase != PH_AUTO) c0 = (!q->nph_init || !q->p_valid) ? CASE_NPH_ENTER : CASE_NPH;
  const unsigned o0 = (q->phase == PH_AUTO && q->step % q->eval == 0) ? 1u : 0u;

  cudaGraph_t g = nullptr;
  cudaGraphExec_t ex = nullptr;
  MDB_CUDA(cudaGraphCreate(&g, 0));
  int rc = MDB_OK;
  auto ck = [&](cudaError_t e, const char* what) {
    if (rc == MDB_OK && e != cudaSuccess) rc = cuda_error(e, what);
    return rc == MDB_OK;
  };
  cudaGraphConditionalHandle hw, hc, ho;
  ck(cudaGraphConditionalHandleCreate(&hw, g, 1, cudaGraphCondAssignDefault), "handle");
  ck(cudaGraphConditionalHandleCreate(&hc, g, (unsigned)c0, cudaGraphCondAssignDefault), "handle");
  ck(cudaGraphConditionalHandleCreate(&ho, g, o0, cudaGraphCondAssignDefault), "handle");
  pa.h_while = hw;
  pa.h_case = hc;
  pa.h_obs = ho;

  // while node: its body is one protocol step
  cudaGraph_t body = nullptr;
  cudaGraphNode_t nwhile;
  if (rc == MDB_OK) {
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = hw;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    if (ck(cudaGraphAddNode(&nwhile, g, nullptr, 0, &cp), "cudaGraphAddNode(while)"))
      body = cp.conditional.phGraph_out[0];
  }
  // switch node: the step body of the phase
  cudaGraphNode_t nswitch;
  cudaGraph_t cases[3] = {nullptr, nullptr, nullptr};
  if (rc == MDB_OK) {
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = hc;
    cp.conditional.type = cudaGraphCondTypeSwitch;
    cp.conditional.size = 3;
    if (ck(cudaGraphAddNode(&nswitch, body, nullptr, 0, &cp), "cudaGraphAddNode(switch)"))
      for (int k = 0; k < 3; ++k) cases[k] = cp.conditional.phGraph_out[k];
  }
  for (int k = 0; k < 3 && rc == MDB_OK; ++k) {
    cudaGraph_t cg = cases[k];
    cudaGraphNode_t prev = nullptr, nd, nc, nf;
    const bool nph = (k != CASE_NH);
    if (k == CASE_NPH_ENTER) {
      cudaGraphNode_t nobs;
      rc = add_kernel_node(cg, nullptr, 0, force_fn(FM_OBS, true), nblocks_, kThreads, dev_, &nobs);
      if (rc == MDB_OK) {
        void* args[] = {&pa};
        cudaKernelNodeParams kp = {};
        kp.func = (void*)k_proto_enter;
        kp.gridDim = dim3(1);
        kp.blockDim = dim3(32);
        kp.kernelParams = args;
        ck(cudaGraphAddKernelNode(&prev, cg, &nobs, 1, &kp), "cudaGraphAddKernelNode(enter)");
      }
    }
    cudaGraphConditionalHandle hr;
    if (rc == MDB_OK) ck(cudaGraphConditionalHandleCreate(&hr, g, 0, 0), "handle");
    Dev dd = dev_;
    if (rc == MDB_OK) {
      dd.cond = hr;
      dd.use_cond = 1;
      rc = add_kernel_node(cg, prev ? &prev : nullptr, prev ? 1 : 0, drift_fn(nph ? DM_NPH : DM_NH),
                           nblocks_, kThreads, dd, &nd);
    }
    if (rc == MDB_OK) rc = add_cond_rebuild(cg, nd, hr, &nc);
    if (rc == MDB_OK)
      rc = add_kernel_node(cg, &nc, 1, force_fn(nph ? FM_NPH : FM_NH, true), nblocks_, kThreads,
                           dev_, &nf);
  }
  // the AUTO_TARGET sample's observation pass, then the protocol step
  cudaGraphNode_t nobs_if, nstep;
  if (rc == MDB_OK) {
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = ho;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    if (ck(cudaGraphAddNode(&nobs_if, body, &nswitch, 1, &cp), "cudaGraphAddNode(if)")) {
      cudaGraphNode_t nobs;
      rc = add_kernel_node(cp.conditional.phGraph_out[0], nullptr, 0, force_fn(FM_OBS, true),
                           nblocks_, kThreads, dev_, &nobs);
    }
  }
  if (rc == MDB_OK) {
    void* args[] = {&pa};
    cudaKernelNodeParams kp = {};
    kp.func = (void*)k_proto_step;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(32);
    kp.kernelParams = args;
    ck(cudaGraphAddKernelNode(&nstep, body, &nobs_if, 1, &kp), "cudaGraphAddKernelNode(step)");
  }
  if (rc == MDB_OK) ck(cudaGraphInstantiate(&ex, g, 0), "cudaGraphInstantiate(protocol)");
  bool launched = false;
  if (rc == MDB_OK) launched = ck(cudaGraphLaunch(ex, stream_), "cudaGraphLaunch(protocol)");
  if (rc == MDB_OK) {
    ck(cudaMemcpyAsync(q, bq.p, sizeof(NphProto), cudaMemcpyDeviceToHost, stream_), "copy");
    ck(wait_host(), "cudaStreamSynchronize");
  }
  if (rc == MDB_OK) {
    // per step: drift + force + protocol step (like run_md, the conditional
    // rebuild bodies and observation passes are not counted)
    launches_ += 3LL * q->step;
    count_launches(3LL * q->step);
    const int64_t nr = q->nrec < cap ? q->nrec : cap;
    if (nr > 0) {
      ck(cudaMemcpyAsync(rec, br.p, sizeof(mdb_nph_record_t) * (size_t)nr,
                         cudaMemcpyDeviceToHost, stream_),
         "copy");
      ck(wait_host(), "cudaStreamSynchronize");
    }
  }
  if (rc != MDB_OK && launched) cudaStreamSynchronize(stream_);  // before the buffers go
  if (ex) cudaGraphExecDestroy(ex);
  if (g) cudaGraphDestroy(g);
  return rc;
}

}  // namespace mdb
