"""Benchmark of the MD stepping path: particle-steps/s.

Default workload: the Nose-Hoover interface slab, N = 1,048,576 (Lx = 2 Ly at
density 0.8, 90%/10% A stripes, T = 0.7, Q = 1.0, dt = 0.002), FP32 pair terms
with FP64 state. A "step" is one step_single_nose_hoover() of that system.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload nvt_slab|nve_4096|fire_mix]

Multi-GPU (torchrun, one rank per GPU): a single system does not shard, so
every rank advances its own replica (seeded per rank) — weak scaling, no
collective on the data path; time is the max over ranks.

--impl reference times the reference's algorithm for this path on the host
cores: its O(N^2) all-pairs force loop (src/md_cuda_common.cu:151-264) in the
reference's mixed precision, restated by the CPU oracle, on a bounded sample of
rows per step (the reference has no CPU implementation of its own).

The main line also carries `reference_gpu`: the reference's own CUDA kernels
(src/md_cuda_common.cu compiled unmodified into oracle/_ref/libref_kernels.so,
driven by its host step logic at MPI world size 1, self-halo included) timed
on the same GPU for the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L2_BYTES = 126 * 1024 * 1024
FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # 148 SMs x 128 lanes x FMA x 1.965 GHz


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(x: float, dist, device) -> float:
    """The maximum of x over all ranks (x itself without a process group)."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for k, name in enumerate(names):
                if parts[5 + k].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_workload(name, rank):
    from md_simulation_cuda_b200 import workloads as wl

    if name == "nve_4096":
        f, cfg = wl.nve_4096(seed=1 + 1000 * rank)
        return f, cfg, "nve", "NVE velocity Verlet N=4096, rho=0.8, dt=0.001"
    if name == "nph_4m":
        f, cfg = wl.nph_square(seed=3 + 1000 * rank)
        return f, cfg, "nph", ("NPH barostat N=4194304, square box, rho=0.8, 65% A, P_ext=1.0, "
                               "W=10.0, dt=0.001")
    f, cfg = wl.nvt_slab(seed=2 + 1000 * rank)
    return f, cfg, "nh", ("Nose-Hoover interface slab N=1048576, Lx=2Ly, rho=0.8, "
                          "90%/10% A stripes, T=0.7, Q=1.0, dt=0.002")


def step_roofline(per_gpu_value, hbm_gbs, p_ord, bytes_per_step=97.0):
    """Whole-step roofline: particle-steps/s on one GPU against
    min(HBM bandwidth / bytes per particle-step, FP32 peak / (24 flops x
    ordered pairs inside the cutoff per particle)). 97 B is the specified
    algorithmic figure (FP64 pos/vel/force read and written, 1 B type); this
    design moves 173 B (force phase 65 B + drift phase 108 B)."""
    bw_bound = hbm_gbs * 1e9 / bytes_per_step
    fp_bound = FP32_NOMINAL_TFLOPS * 1e12 / (24.0 * p_ord) if p_ord else float("inf")
    bound = min(bw_bound, fp_bound)
    return {"achieved": per_gpu_value, "bound": bound, "unit": "particle-steps/s",
            "bytes_per_particle_step": bytes_per_step,
            "limited_by": "hbm" if bw_bound <= fp_bound else "fp32",
            "frac": per_gpu_value / bound}


def reference_gpu_leg(f, cfg, mode, steps):
    """The reference's own single-GPU build on this GPU: its kernels from
    src/md_cuda_common.cu (compiled unmodified for sm_100a) and its host step
    logic at world size 1, including the self-halo it rebuilds every step.
    Device time (CUDA events around its host-synchronous loop) after one
    untimed step."""
    try:
        from oracle import refkernels as rk

        if not rk.available():
            return {"unavailable": "oracle/_ref/libref_kernels.so not built"}
        kind = {"nh": rk.KIND_NH, "nph": rk.KIND_NPH, "nve": rk.KIND_NVE}[mode]
        p_ext = 1.0 if mode == "nph" else 0.0
        r = rk.RefSim(cfg, f, ws1_halo=True, threads=int(cfg.get("THREADS_PER_BLOCK", 256) or 256))
        r.step(kind, 1, p_ext=p_ext)
        ms = r.time_steps(kind, steps, p_ext=p_ext)
        r.close()
        n = len(f)
        return {"value": n * steps / (ms * 1e-3), "unit": "particle-steps/s",
                "ms_per_step": ms / steps, "steps": steps,
                "build": "src/md_cuda_common.cu unmodified, nvcc -O3 for sm_100a "
                         "(oracle/build_ref.py); host step logic of src/md_env.cu at world "
                         "size 1 restated in oracle/ref_kernels.cu",
                "how": "CUDA events on the default stream around the host-synchronous "
                       "step loop, after 1 untimed step"}
    except Exception as e:  # noqa: BLE001
        return {"unavailable": f"reference kernels failed: {e}"}


def cpu_cell_baseline(f, cfg, mode_name, budget_s=20.0):
    """The oracle's cell-list step on all host cores (the fair CPU baseline)."""
    from oracle import pyoracle as po

    s = po.Sim(cfg, f["pos"], f["vel"], f["type"], mode=po.OR_REF_MIXED, use_cells=True)
    if mode_name == "nh":
        step = s.step_nose_hoover
    elif mode_name == "nph":
        step = lambda n: s.step_nph(1.0, n)  # noqa: E731
    else:
        step = s.step_nve
    t0 = time.perf_counter()
    n = 0
    while True:
        step(1)
        n += 1
        if time.perf_counter() - t0 > budget_s / 2 or n >= 50:
            break
    dt = time.perf_counter() - t0
    return {"value": len(f) * n / dt, "unit": "particle-steps/s", "cores": os.cpu_count(),
            "kind": "port",
            "sample": f"{n} full steps of the oracle's cell-list "
                      f"{dict(nh='Nose-Hoover', nph='NPH', nve='NVE')[mode_name]} step "
                      f"(reference mixed-precision pair arithmetic, OpenMP on all cores)"}


def measure_fire_mix(dev, warm_iters, iters, plain_sample=32, to_completion=False, shard=None,
                     dist=None):
    """C4: the 512-system FIRE mix as ONE batch vs the same systems run one at
    a time through the single-system path (a stratified sample of
    `plain_sample` systems, each as a batch of one). particle-iterations are
    counted per system from its own iteration counter, so systems that
    converge stop counting. Wall clock around synchronous runs."""
    import numpy as np

    import md_simulation_cuda_b200 as mdb
    from md_simulation_cuda_b200 import workloads as wl

    S = wl.FIRE_SETTINGS
    params = wl.fire_params()
    systems = wl.fire_mix(512)
    if shard is not None:
        # this rank's systems: the library's LPT placement on particles x
        # iteration cap (the same on every rank; no collective on the data path)
        rank, ws = shard
        owner, _ = mdb.place_lpt([len(f) * S["max_steps"] for f, _ in systems], ws)
        systems = [x for x, r in zip(systems, owner) if r == rank]
    sizes = np.array([len(f) for f, _ in systems])

    def steps_of(b, ids):
        return np.array([b.system_info(i)[2] for i in ids], dtype=np.int64)

    b = mdb.Batch(device=dev, autotune=True)
    ids = [b.add_fire(cfg, f, S["force_tol"], S["max_steps"], params) for f, cfg in systems]
    t_build = time.perf_counter()
    b.run(warm_iters)
    schedule = b.schedule()
    t_build = time.perf_counter() - t_build
    s0 = steps_of(b, ids)
    import torch

    # (an NVTX range around the timed window: `ncu --nvtx --nvtx-include timed/`
    # profiles exactly these launches)
    torch.cuda.nvtx.range_push("timed")
    t0 = time.perf_counter()
    b.run(-1 if to_completion else iters)
    t_batch = max_over_ranks(time.perf_counter() - t0, dist, dev)
    torch.cuda.nvtx.range_pop()
    s1 = steps_of(b, ids)
    # non-finite systems (none are expected: FP32 pair terms are floored at
    # r^2 = 1e-5 sigma^2) do not count as work
    finite = np.array([not b.fire_result(i, with_frame=False).nonfinite for i in ids])
    work = float((sizes * (s1 - s0) * finite).sum())
    if dist is not None:
        import torch

        tw = torch.tensor([work], device=dev, dtype=torch.float64)
        dist.all_reduce(tw)
        work = float(tw.item())
    done = int(b.progress()[1])
    converged = sum(1 for i in ids if b.system_info(i)[1] and b.system_info(i)[2] < S["max_steps"])
    del b
    # plain path: the same window for a stratified sample, one system at a time
    order = np.argsort(sizes)
    pick = order[:: max(1, len(order) // plain_sample)][:plain_sample]
    p_work, p_time = 0.0, 0.0
    for k in pick:
        f, cfg = systems[k]
        one = mdb.Batch(device=dev)
        one.add_fire(cfg, f, S["force_tol"], S["max_steps"], params)
        one.run(warm_iters)
        a0 = one.system_info(0)[2]
        t1 = time.perf_counter()
        one.run(-1 if to_completion else iters)
        p_time += time.perf_counter() - t1
        p_work += float(sizes[k] * (one.system_info(0)[2] - a0))
        del one
    plain = p_work / p_time if p_time > 0 else None
    value = work / t_batch
    return {"metric": "particle-iterations/s", "value": value, "unit": "particle-iterations/s",
            "systems": len(systems), "particles": int(sizes.sum()),
            "ranks": 1 if shard is None else shard[1],
            "window": ("to completion" if to_completion else f"iterations {warm_iters}.."
                       f"{warm_iters + iters}"),
            "seconds": t_batch, "build_and_warmup_s": t_build,
            "finished_systems": done, "converged_systems": converged,
            "nonfinite_systems": int((~finite).sum()),
            "schedule": schedule,
            "plain_path": {"value": plain, "unit": "particle-iterations/s",
                           "sample": f"{len(pick)} systems (every {max(1, len(order) // plain_sample)}"
                                     f"th by N), each alone as a batch of one, same window"},
            "ratio_vs_plain": (value / plain) if plain else None}


def run_fire_mix(args):
    """The 512-system FIRE mix; with N ranks the systems are split by LPT on
    their size, each rank runs its share as one batch, and the aggregate is
    the total work over the slowest rank's time."""
    import torch

    ws, rank, local = _dist()
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = local if ws > 1 else 0
    torch.cuda.set_device(dev)
    clocks = ClockSampler(dev)
    clocks.start()
    res = measure_fire_mix(dev, args.warmup, args.steps, to_completion=args.to_completion,
                           shard=(rank, ws) if ws > 1 else None, dist=dist,
                           plain_sample=32 // ws)
    clk = clocks.stop()
    if rank == 0:
        out = {"metric": res["metric"], "value": res["value"], "unit": res["unit"], "n_gpus": ws,
               "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
               "scaling": "strong", "vs_baseline": None, "dtype": "fp32-pair/fp64-state",
               "data": "synthetic (seeded uniform-random starts)",
               "config": {"workload": "batched FIRE, 512 systems, N log-uniform [256, 16384], "
                                      "f_A ~ U(0.2,0.8), rho ~ U(0.6,1.0), square periodic "
                                      "boxes, uniform-random positions; dt_init 0.001, dt_max "
                                      "0.01, alpha0 0.1, f_inc 1.1, f_dec 0.5, tol 1e-6, 20000 "
                                      "its", "parallelism": f"systems sharded by LPT over {ws}"},
               "batched": res, "clocks": clk}
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def run_served(args):
    """C5: the served mixed stream through mdb.Server (continuous batching).
    Requests are submitted at their Poisson arrival times by one thread while
    a pool of threads builds their frames ahead of time; latency is measured
    from the scheduled arrival to the result being available on the host."""
    import queue
    import threading
    from concurrent.futures import ThreadPoolExecutor

    import numpy as np
    import torch

    import md_simulation_cuda_b200 as mdb
    from md_simulation_cuda_b200 import workloads as wl

    ws, rank, local = _dist()
    if rank != 0:
        return 0
    torch.cuda.set_device(0)
    specs = wl.served_stream(n_requests=args.requests)
    params = wl.fire_params()
    S = wl.FIRE_SETTINGS
    pool = ThreadPoolExecutor(max_workers=8)
    futures = [pool.submit(wl.served_frame, sp) for sp in specs[:64]]
    nxt = len(futures)
    srv = (mdb.Server(device=0, order=mdb.ORDER_FIFO, priorities=False) if args.server_fifo
           else mdb.Server(device=0))
    host_t0 = time.perf_counter()  # the server clock starts at creation
    ids = queue.Queue()
    clocks = ClockSampler(0)
    clocks.start()
    start = time.perf_counter()
    lag = []
    for k, sp in enumerate(specs):
        f, cfg = futures[k].result()
        futures[k] = None
        if nxt < len(specs):
            futures.append(pool.submit(wl.served_frame, specs[nxt]))
            nxt += 1
        delay = start + sp["arrival"] - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        lag.append(max(0.0, -delay))
        if sp["fire"]:
            rid = srv.submit_fire(cfg, f, S["force_tol"], S["max_steps"], params)
        else:
            rid = srv.submit_md(cfg, f, sp["steps"], nose_hoover=True)
        ids.put((k, rid))
    ids.put(None)
    results = {}
    while True:
        item = ids.get()
        if item is None:
            break
        k, rid = item
        srv.wait(rid)
        r = srv.result(rid)
        r.frame = None
        results[k] = r
    clk = clocks.stop()
    st = srv.stats()
    srv.close()
    pool.shutdown()
    offset = start - host_t0
    lat = np.array([results[k].t_done - (offset + specs[k]["arrival"]) for k in results])
    lat_fire = np.array([lat[i] for i, k in enumerate(results) if specs[k]["fire"]])
    lat_md = np.array([lat[i] for i, k in enumerate(results) if not specs[k]["fire"]])
    work = sum(results[k].n * results[k].steps for k in results)
    t_first = offset + specs[0]["arrival"]
    t_last = max(results[k].t_done for k in results)
    agg = work / (t_last - t_first)
    out = {"metric": "served particle-steps/s (p50/p99 latency)", "value": agg,
           "unit": "particle-steps/s", "n_gpus": 1, "steps": len(specs), "warmup": 0,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "fp32-pair/fp64-state", "data": "synthetic (seeded jittered lattices)",
           "config": {"workload": f"served stream: {len(specs)} requests, Poisson 200/s, 70% NVT "
                                  "(N log-uniform [1024, 262144], 1000-20000 steps, T ~ U(0.5,1.2)) "
                                  "/ 30% FIRE quench (same N law, tol 1e-6, 20000 its)",
                      "server": ("mdb.Server, 8 batches in flight of up to 1Mi particles, 80% of free HBM, " +
                                 ("oldest first, normal stream priority" if args.server_fifo else
                                  "least work first with a 60 s aging bound, stream priority by batch work"))},
           "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                         "max": float(lat.max()),
                         "nvt_p50": float(np.percentile(lat_md, 50)) if len(lat_md) else None,
                         "fire_p50": float(np.percentile(lat_fire, 50)) if len(lat_fire) else None,
                         "from": "scheduled arrival to result on the host"},
           "arrival_lag_s": {"p50": float(np.percentile(lag, 50)), "max": float(max(lag))},
           "requests": {"finished": int(st.finished), "failed": int(st.failed),
                        "batches_admitted": int(st.batches_admitted)},
           "wall_s": t_last - t_first, "clocks": clk}
    print(json.dumps(out), flush=True)
    return 0


def run_reference(args):
    """Reference arm: the O(N^2) all-pairs force loop, bounded row sample."""
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    from oracle import pyoracle as po

    f, cfg, mode, desc = make_workload(args.workload, 0)
    N = len(f)
    Lx, Ly = cfg["box_w_global"], cfg["box_h_global"]
    cores = os.cpu_count()
    # calibrate rows/s, then size each step for ~budget/(K+W) seconds
    t0 = time.perf_counter()
    po.forces_rows(cfg, f["pos"], f["type"], Lx, Ly, 0, 16)
    rate = 16 / (time.perf_counter() - t0)
    budget = 90.0
    rows = max(8, min(N, int(rate * budget / max(1, args.steps + args.warmup))))
    for w in range(args.warmup):
        po.forces_rows(cfg, f["pos"], f["type"], Lx, Ly, (w * rows) % (N - rows + 1), rows)
    t0 = time.perf_counter()
    for k in range(args.steps):
        po.forces_rows(cfg, f["pos"], f["type"], Lx, Ly, (k * rows) % (N - rows + 1), rows)
    dt = time.perf_counter() - t0
    value = rows * args.steps / dt
    out = {"impl": "reference", "metric": "particle-steps/s", "value": value,
           "unit": "particle-steps/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "fp32-pair/fp64-accumulate", "data": "synthetic",
           "config": {"workload": desc, "N": N},
           "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": cores,
                            "kind": "port",
                            "sample": f"{rows} rows of the O(N^2) force loop over all {N} "
                                      f"particles per step (rows x 1 step = particle-steps)"},
           "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return 0


def run_ours(args):
    import numpy as np
    import torch

    import md_simulation_cuda_b200 as mdb

    ws, rank, local = _dist()
    if ws > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        dist = None
    dev = local if ws > 1 else 0
    torch.cuda.set_device(dev)
    f, cfg, mode, desc = make_workload(args.workload, rank)
    N = len(f)
    sim = mdb.MDSimulation(cfg, frame=f, device=dev, autotune=True)
    schedule = sim.schedule()
    if mode == "nh":
        step = lambda n: sim.step_single_nose_hoover(nsteps=n)  # noqa: E731
    elif mode == "nph":
        step = lambda n: sim.step_single_NPH(1.0, nsteps=n)  # noqa: E731
    else:
        step = lambda n: sim.step_single_NVE(nsteps=n)  # noqa: E731
    stream = torch.cuda.ExternalStream(sim.cuda_stream(), device=dev)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)
    step(args.warmup)
    sim.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- device-timed region: K steps, L2 flushed between steps -------------
    clocks = ClockSampler(dev)
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    o0 = sim.observables()
    l0 = mdb.kernel_launches()
    barrier()
    torch.cuda.synchronize(dev)
    sim.synchronize()
    torch.cuda.nvtx.range_push("timed")  # `ncu --nvtx --nvtx-include timed/`
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()  # evict the state from L2 (outside the step's events)
            ev[k][0].record(stream)
        step(1)
        ev[k][1].record(stream)
    sim.synchronize()
    torch.cuda.synchronize(dev)
    torch.cuda.nvtx.range_pop()
    barrier()
    clk = clocks.stop()
    o1 = sim.observables()
    # graph launches are counted as drift + force per step; the conditional
    # rebuild body (11 kernels) runs only on the steps that rebuild
    launches = mdb.kernel_launches() - l0 + 11 * (o1.rebuilds - o0.rebuilds)
    t_ms = sum(a.elapsed_time(b) for a, b in ev)
    t_max = max_over_ranks(t_ms / 1e3, dist, dev)
    value = N * ws * args.steps / t_max

    # ---- the dominant kernel: per-phase CUDA events on the launching stream --
    nph = 20
    ms = sim.phase_times(nph, nose_hoover=(mode == "nh"), nph=(mode == "nph"))
    t_force = ms[2] / nph / 1e3
    t_drift = ms[0] / nph / 1e3
    hbm_peak, peak_kind = _peaks()
    force_bytes = 65.0 * N   # read pos(ff) 16 + type 1 + vel 16; write acc 16 + vel 16
    step_bytes = 97.0 * N    # per particle-step, whole step
    prof = os.path.join(ROOT, "profiles", "force_kernel_traffic.json")
    traffic = None
    if os.path.exists(prof):
        pj = json.load(open(prof))
        traffic = pj.get("dram_bytes_per_particle", None)
        traffic = traffic * N if traffic else None
    from oracle import pyoracle as po

    p_ord = None
    cpu = None
    if rank == 0 and ws == 1:
        p_ord = po.count_pairs_cells(cfg, f["pos"], f["type"], cfg["box_w_global"],
                                     cfg["box_h_global"]) / N
        cpu = cpu_cell_baseline(f, cfg, mode)

    # ---- end to end through the C ABI with host buffers ----------------------
    K2 = max(10, args.steps)
    pinned = torch.empty(N * 64, dtype=torch.uint8, pin_memory=True)
    host = pinned.numpy().view(mdb.PARTICLE_DTYPE)
    host[:] = f
    out_pinned = torch.empty(N * 64, dtype=torch.uint8, pin_memory=True)
    out_host = out_pinned.numpy().view(mdb.PARTICLE_DTYPE)
    import ctypes

    obs_size = ctypes.sizeof(mdb._lib.MDBObservables)
    ring = torch.empty(K2 * obs_size, dtype=torch.uint8, pin_memory=True)
    ring_ptr = ring.data_ptr()
    barrier()
    sim.synchronize()
    t0 = time.perf_counter()
    sim.set_frame(host)                      # H2D of the step inputs
    for k in range(K2):
        step(1)
        sim.observables_async(ring_ptr + k * obs_size)  # D2H of the step's result
    mdb._lib.check(mdb._lib.lib().mdb_sim_get_frame(sim._h, mdb._lib.frame_ptr(out_host), N))
    e2e_t = max_over_ranks(time.perf_counter() - t0, dist, dev)
    last = mdb._lib.MDBObservables.from_address(ring_ptr + (K2 - 1) * obs_size)
    first = mdb._lib.MDBObservables.from_address(ring_ptr)
    assert last.steps - first.steps == K2 - 1 and last.n == N  # every step's record arrived
    e2e = {"value": N * ws * K2 / e2e_t, "unit": "particle-steps/s",
           "h2d_bytes_per_step": int(64 * N / K2) + 8,
           "d2h_bytes_per_step": int(64 * N / K2) + obs_size,
           "steps": K2,
           "how": "set_frame from pinned host memory, K steps each followed by an "
                  "asynchronous observables read into pinned memory, get_frame; wall clock"}

    # ---- one call of K steps (a driver that asks for many steps at once) -------
    # For a system small enough for the multi-step kernel this runs all K
    # steps in cooperative launches that return only for rebuilds; the L2 is
    # not flushed inside the call (the state of such a system fits in it).
    long_call = None
    if schedule.get("multi_step"):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        sim.synchronize()
        with torch.cuda.stream(stream):
            flush.zero_()
            a.record(stream)
        step(args.steps)
        b.record(stream)
        sim.synchronize()
        t_call = max_over_ranks(a.elapsed_time(b) / 1e3, dist, dev)
        long_call = {"value": N * ws * args.steps / t_call, "unit": "particle-steps/s",
                     "steps_per_call": args.steps, "us_per_step": t_call / args.steps * 1e6,
                     "how": "one step call of K steps (multi-step kernel), CUDA events, "
                            "L2 flushed once before the call"}

    # ---- C4: the 512-system FIRE mix, batched vs one system at a time --------
    batched = None
    if rank == 0 and ws == 1 and args.workload == "nvt_slab":
        batched = measure_fire_mix(dev, 100, 2000)

    # ---- the reference's own CUDA build on this GPU (rank 0, N = 1) ---------
    reference_gpu = None
    if rank == 0 and ws == 1:
        del sim
        sim = None
        torch.cuda.empty_cache()
        ref_steps = {"nh": 3, "nph": 1, "nve": 1000}[mode]
        reference_gpu = reference_gpu_leg(f, cfg, mode, ref_steps)
        if "value" in reference_gpu:
            reference_gpu["ours_over_reference"] = value / reference_gpu["value"]
            reference_gpu["ours_e2e_over_reference"] = e2e["value"] / reference_gpu["value"]

    if rank == 0:
        achieved = force_bytes / t_force / 1e9
        out = {
            "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32-pair/fp64-state", "data": "synthetic (seeded jittered lattice)",
            "config": {"workload": desc, "N": N, "parallelism": f"replicas x{ws}",
                       "l2": "flushed between timed steps (256 MiB write outside the events)"},
            "roofline": {"bound": "hbm", "kernel": {
                             "nh": "k_force<FM_NH> (pair force + NH kick + K)",
                             "nph": "k_force<FM_NPH> (pair force + virial + kick + barostat)",
                             "nve": "k_force<FM_NVE> (pair force + kick)"}[mode],
                         "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "peak_source": peak_kind,
                         "traffic": traffic,
                         "algorithmic_bytes_per_particle": 65,
                         "force_ms": t_force * 1e3, "drift_ms": t_drift * 1e3,
                         "step_GBps_97B": step_bytes * value / ws / N / 1e9 if N else None,
                         "fp32": {"achieved_tflops": (24.0 * p_ord * N / t_force / 1e12)
                                  if p_ord else None,
                                  "peak_tflops": FP32_NOMINAL_TFLOPS, "peak_source": "nominal",
                                  "frac": (24.0 * p_ord * N / t_force / 1e12 / FP32_NOMINAL_TFLOPS)
                                  if p_ord else None,
                                  "pairs_per_particle": p_ord},
                         # whole step: per-GPU particle-steps/s over the step's bound,
                         # min(HBM peak / 97 B, FP32 peak / (24 flops x P_ord))
                         "step": step_roofline(value / ws, hbm_peak, p_ord),
                         "step_design": step_roofline(value / ws, hbm_peak, p_ord, 173.0)},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(launches),
            "clocks": clk,
            "batched": batched,
            "reference_gpu": reference_gpu,
            "schedule": schedule,
            "long_call": long_call,
        }
        print(json.dumps(out), flush=True)
    del sim
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="nvt_slab",
                    choices=["nvt_slab", "nve_4096", "nph_4m", "fire_mix", "served"])
    ap.add_argument("--to-completion", action="store_true",
                    help="fire_mix: run every system until it converges or hits 20000 its")
    ap.add_argument("--requests", type=int, default=2000, help="served: number of requests")
    ap.add_argument("--server-fifo", action="store_true",
                    help="served: oldest-first admission, no stream priorities")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "fire_mix":
        return run_fire_mix(args)
    if args.workload == "served":
        return run_served(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
