"""The NPH driver protocol on a real system.

The library runs the protocol as one graph launch with the decisions on the
device (a while node over the steps, a switch node choosing the Nose-Hoover or
NPH body, the window statistics in a one-thread kernel), or host-driven with
the decisions on the host between captured step chunks. Both give the same
pressure samples, target and phase switches, bit for bit, as the reference
driver's per-step loop written against the public step API, and the same
records and final state as each other. The device form waits on the host only
after the last step."""
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


def _q_default():
    return protocol(auto_steps=60, eval_interval=10, window_samples=4, stable_required=5,
                    warmup_min_steps=20, warmup_max_steps=200, production_steps=50,
                    tolerance_rel=0.3)


REC_FIELDS = ("step", "t", "phase", "P_inst", "P_target", "mean", "stddev", "rel_err", "Lx",
              "Ly", "dA_dt")


def _rec_tuple(r):
    return tuple(getattr(r, k) for k in REC_FIELDS)


def _state(sim):
    sim.sample_collect()
    fr = sim.get_host_particles()
    o = sim.observables()
    return (fr["pos"].tobytes(), fr["vel"].tobytes(), fr["acc"].tobytes(), o.t, o.Lx, o.Ly,
            o.nph_area_momentum, o.last_instant_pressure, o.steps)


def test_protocol_matches_per_step_driver(built):
    f, cfg = _system()
    q = _q_default()
    P_target, warm_end, total, samples, ref_sim = per_step(cfg, f, q)
    sim = mdb.MDSimulation(cfg, frame=f)
    res, recs = sim.run_nph_protocol(q)
    assert res.finished and res.total_steps == total
    assert res.P_target == P_target and res.auto_end_step == 59
    assert res.warmup_end_step == warm_end
    assert [(r.step, r.phase, r.P_inst) for r in recs] == samples
    assert sim.get_Lx() == ref_sim.get_Lx() and sim.get_Ly() == ref_sim.get_Ly()
    # one graph launch: no host wait between the pressure samples
    assert len(samples) > 10 and res.host_waits <= 2
    assert _state(sim) == _state(ref_sim)


@pytest.mark.parametrize("case", ["auto", "auto_ends_on_sample", "fixed_target", "forced",
                                  "resumed"])
def test_device_protocol_equals_host_driven(built, case):
    """Every record field, the result and the final state bit for bit."""
    f, cfg = _system()
    q = _q_default()
    if case == "fixed_target":  # starts in NPH_WARMUP: the first step enters NPH
        q.auto_target = 0
        q.P_target = 1.7
    elif case == "auto_ends_on_sample":  # the NPH entry finds the pressure current
        q.auto_steps = 61
    elif case == "forced":  # the window never settles: the warmup ends at its limit
        q.tolerance_rel = 1e-9
        q.warmup_max_steps = 120
    elif case == "resumed":  # NPH initialised and the pressure current: no entry pass
        q.auto_target = 0
        q.P_target = 1.6
    runs = []
    for host in (True, False):
        sim = mdb.MDSimulation(cfg, frame=f)
        if case == "resumed":  # NPH already initialised, the pressure current
            sim.step_single_NPH(1.5, nsteps=7)
            sim.step_single_nose_hoover(nsteps=3)
            sim.cal_instant_pressure()
        res, recs = sim.run_nph_protocol(q, host_driven=host)
        runs.append((res, [_rec_tuple(r) for r in recs], _state(sim)))
    (rh, ch, sh), (rd, cd, sd) = runs
    for k in ("P_target", "auto_end_step", "warmup_end_step", "total_steps", "n_records",
              "forced_switch", "finished"):
        assert getattr(rh, k) == getattr(rd, k), k
    assert ch == cd
    assert sh == sd
    assert rd.finished == 1
    if case == "forced":
        assert rd.forced_switch == 1
    assert rh.host_waits >= rh.n_records  # the host reads every sample
    assert rd.host_waits <= 2


def test_device_protocol_record_cap_and_continuation(built):
    """Records beyond the cap are counted, not written; the simulation steps on
    from the protocol's end like after the host-driven run."""
    f, cfg = _system()
    q = _q_default()
    out = []
    for host in (True, False):
        sim = mdb.MDSimulation(cfg, frame=f)
        res, recs = sim.run_nph_protocol(q, record_cap=5, host_driven=host)
        assert len(recs) == 5 and res.n_records > 5
        sim.step_single_NPH(res.P_target, nsteps=20)
        sim.step_single_nose_hoover(nsteps=10)
        out.append(([_rec_tuple(r) for r in recs], _state(sim), sim.cal_instant_pressure()))
    assert out[0] == out[1]
