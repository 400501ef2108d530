"""The NPH driver protocol (tests/run_NPH_test/run_test_NPH.cpp:137-290 of the
reference) without a GPU: the library's chunked run (mdb_nph_protocol_dry_run)
takes every decision on the same step as a literal per-step transcription of
the reference's loop, for scripted pressure sequences."""
import math

import numpy as np
import pytest

import md_simulation_cuda_b200 as mdb
from md_simulation_cuda_b200._lib import MDBNphProtocol


def literal(q, pressures):
    """The reference driver's loop, one step per iteration."""
    eval_i = max(1, q.eval_interval)
    auto_steps = max(1, q.auto_steps)
    window = max(2, q.window_samples)
    stable_req = max(1, q.stable_required)
    warm_min = max(0, q.warmup_min_steps)
    warm_max = max(warm_min + 1, q.warmup_max_steps)
    prod = max(1, q.production_steps)
    hard = auto_steps + warm_max + prod + 50000
    phase = 0 if q.auto_target else 1
    P_target = 0.0 if q.auto_target else q.P_target
    auto_done = warm_done = prod_done = stable = 0
    auto_samples, win, recs = [], [], []
    auto_end = warm_end = -1
    forced = False
    finished = False
    step = 0

    def stats(v):
        if not v:
            return 0.0, 0.0
        m = sum_seq(v) / len(v)  # std::accumulate order
        if len(v) <= 1:
            return m, 0.0
        var = 0.0
        for x in v:
            var += (x - m) * (x - m)
        return m, math.sqrt(var / (len(v) - 1))

    def sum_seq(v):
        s = 0.0
        for x in v:
            s += x
        return s

    while step < hard and not finished:
        used = phase
        P_inst = pressures[step]
        if used == 0:
            auto_done += 1
        elif used == 1:
            warm_done += 1
        else:
            prod_done += 1
        if step % eval_i == 0:
            if used == 0:
                auto_samples.append(P_inst)
            else:
                win.append(P_inst)
                while len(win) > window:
                    win.pop(0)
        if used == 0 and auto_done >= auto_steps and auto_samples:
            P_target = sum_seq(auto_samples) / len(auto_samples)
            phase = 1
            win = []
            stable = 0
            auto_end = step
        if used == 1:
            if warm_done >= warm_min and len(win) >= window:
                m, sd = stats(win)
                den = max(1e-12, abs(P_target))
                ok = abs(m - P_target) / den <= q.tolerance_rel and sd / den <= q.tolerance_rel
                stable = stable + 1 if ok else 0
                if stable >= stable_req:
                    phase = 2
                    warm_end = step
            if phase == 1 and warm_done >= warm_max:
                phase = 2
                warm_end = step
                forced = True
        if used == 2 and prod_done >= prod:
            finished = True
        if step % eval_i == 0:
            m, sd = stats(win)
            recs.append((step, used, P_inst, P_target, m, sd))
        step += 1
    return dict(P_target=P_target, auto_end=auto_end, warm_end=warm_end, forced=forced,
                finished=finished, total=step, recs=recs)


def protocol(**kw):
    q = MDBNphProtocol()
    q.auto_target = 1
    q.P_target = 0.0
    q.auto_steps = 300
    q.eval_interval = 20
    q.window_samples = 6
    q.stable_required = 45
    q.warmup_min_steps = 130
    q.warmup_max_steps = 2000
    q.production_steps = 250
    q.tolerance_rel = 0.05
    for k, v in kw.items():
        setattr(q, k, v)
    return q


def scripts():
    rng = np.random.default_rng(3)
    n = 60000
    settle = 1.0 + 0.5 * np.exp(-np.arange(n) / 400.0) + 0.01 * rng.standard_normal(n)
    noisy = 1.0 + 0.3 * rng.standard_normal(n)  # never stable: forced switch
    flicker = 1.0 + 0.02 * np.sign(np.sin(np.arange(n) / 37.0))
    return {"settle": settle, "noisy": noisy, "flicker": flicker}


@pytest.mark.parametrize("name", ["settle", "noisy", "flicker"])
@pytest.mark.parametrize("auto", [1, 0])
def test_chunked_protocol_equals_per_step_loop(built, name, auto):
    p = scripts()[name]
    q = protocol(auto_target=auto, P_target=1.0)
    ref = literal(q, p)
    res, recs, chunks = mdb.nph_protocol_dry_run(q, p)
    assert res.P_target == ref["P_target"]
    assert res.auto_end_step == ref["auto_end"]
    assert res.warmup_end_step == ref["warm_end"]
    assert bool(res.forced_switch) == ref["forced"]
    assert bool(res.finished) == ref["finished"]
    assert res.total_steps == ref["total"]
    got = [(r.step, r.phase, r.P_inst, r.P_target, r.mean, r.stddev) for r in recs]
    assert got == ref["recs"]
    assert chunks < res.total_steps / 5  # steps run in chunks, not one by one


def test_protocol_from_config(built):
    cfg = mdb.MDConfigManager()
    cfg.apply_override("pressure_eval_interval_steps", "50")
    cfg.apply_override("nph_steps", "1234")
    q = mdb.nph_protocol_from_config(cfg)
    assert q.auto_target == 1  # pressure_target_mode defaults to "auto_initial"
    assert q.eval_interval == 50 and q.production_steps == 1234
    assert q.window_samples == 50 and q.tolerance_rel == 0.05


@pytest.mark.parametrize("kw", [
    dict(eval_interval=1, window_samples=1, stable_required=1),       # every step sampled, clamps
    dict(auto_steps=1, warmup_min_steps=0, warmup_max_steps=1),      # shortest phases
    dict(warmup_min_steps=500, warmup_max_steps=100),                # max below min: clamped
    dict(eval_interval=7, window_samples=3, stable_required=2, production_steps=1),
    dict(eval_interval=0, auto_steps=0, stable_required=0, production_steps=0),  # zeros: clamped
])
def test_protocol_edge_parameters(built, kw):
    """Degenerate and clamped parameters take the same decisions chunked as in
    the per-step loop."""
    p = scripts()["settle"]
    q = protocol(**kw)
    ref = literal(q, p)
    res, recs, _ = mdb.nph_protocol_dry_run(q, p)
    assert (res.P_target, res.auto_end_step, res.warmup_end_step, bool(res.forced_switch),
            bool(res.finished), res.total_steps) == (
        ref["P_target"], ref["auto_end"], ref["warm_end"], ref["forced"], ref["finished"],
        ref["total"])
    got = [(r.step, r.phase, r.P_inst, r.P_target, r.mean, r.stddev) for r in recs]
    assert got == ref["recs"]
