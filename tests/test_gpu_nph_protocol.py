"""The NPH driver protocol on a real system: the library's chunked run gives
the same pressure samples, target and phase switches, bit for bit, as the
reference driver's per-step loop written against the public step API."""
import pytest

import md_simulation_cuda_b200 as mdb
from md_simulation_cuda_b200 import workloads as wl

from tests.test_nph_protocol import protocol

pytestmark = pytest.mark.gpu


def _system():
    f, Lx, Ly = wl.lattice_frame(900, 0.8, 1.0, 0.65, 0.9, seed=21, jitter=0.1)
    return f, wl.config_dict(900, Lx, Ly, dt=0.002, T=0.9, barostat_mass=10.0)


def per_step(cfg, f, q):
    """run_test_NPH.cpp:137-290, one step at a time through the public API."""
    sim = mdb.MDSimulation(cfg, frame=f)
    phase, P_target = 0, 0.0
    auto_done = warm_done = prod_done = stable = 0
    auto_samples, win, samples = [], [], []
    warm_end = -1
    step = 0
    while True:
        used = phase
        if used == 0:
            sim.step_single_nose_hoover()
        else:
            sim.step_single_NPH(P_target)
        if used == 0:
            auto_done += 1
        elif used == 1:
            warm_done += 1
        else:
            prod_done += 1
        if step % q.eval_interval == 0:
            P = sim.cal_instant_pressure() if used == 0 else sim.get_last_instant_pressure()
            samples.append((step, used, P))
            (auto_samples if used == 0 else win).append(P)
            while len(win) > q.window_samples:
                win.pop(0)
        if used == 0 and auto_done >= q.auto_steps and auto_samples:
            s = 0.0
            for x in auto_samples:
                s += x
            P_target, phase, win, stable = s / len(auto_samples), 1, [], 0
        if used == 1:
            if warm_done >= q.warmup_min_steps and len(win) >= q.window_samples:
                s = 0.0
                for x in win:
                    s += x
                m = s / len(win)
                var = 0.0
                for x in win:
                    var += (x - m) * (x - m)
                sd = (var / (len(win) - 1)) ** 0.5
                den = max(1e-12, abs(P_target))
                ok = abs(m - P_target) / den <= q.tolerance_rel and sd / den <= q.tolerance_rel
                stable = stable + 1 if ok else 0
                if stable >= q.stable_required:
                    phase, warm_end = 2, step
            if phase == 1 and warm_done >= q.warmup_max_steps:
                phase, warm_end = 2, step
        step += 1
        if used == 2 and prod_done >= q.production_steps:
            break
    return P_target, warm_end, step, samples, sim


def test_protocol_matches_per_step_driver(built):
    f, cfg = _system()
    q = protocol(auto_steps=60, eval_interval=10, window_samples=4, stable_required=5,
                 warmup_min_steps=20, warmup_max_steps=200, production_steps=50,
                 tolerance_rel=0.3)
    P_target, warm_end, total, samples, ref_sim = per_step(cfg, f, q)
    sim = mdb.MDSimulation(cfg, frame=f)
    res, recs = sim.run_nph_protocol(q)
    assert res.finished and res.total_steps == total
    assert res.P_target == P_target and res.auto_end_step == 59
    assert res.warmup_end_step == warm_end
    assert [(r.step, r.phase, r.P_inst) for r in recs] == samples
    assert sim.get_Lx() == ref_sim.get_Lx() and sim.get_Ly() == ref_sim.get_Ly()
