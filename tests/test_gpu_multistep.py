"""The multi-step kernel (mdb_options_t.step_kernel).

A single system whose blocks all fit on the device at once runs its MD steps
in one cooperative kernel: the drift and force phases of each step with grid
barriers between them, returning to the graph around it only for a cell-list
rebuild. The phases are the per-phase kernels' own block functions over the
same blocks, so the trajectory, the thermostat and barostat variables and the
step and rebuild counts are bit for bit those of one launch per phase.
"""
import pytest

import md_simulation_cuda_b200 as mdb
from md_simulation_cuda_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _system(N, seed=21):
    f, Lx, Ly = wl.lattice_frame(N, 0.8, 1.0, 0.65, 0.9, seed=seed, jitter=0.1)
    return f, wl.config_dict(N, Lx, Ly, dt=0.002, T=0.9, barostat_mass=10.0)


def _state(sim):
    sim.sample_collect()
    fr = sim.get_host_particles()
    o = sim.observables()
    return (fr["pos"].tobytes(), fr["vel"].tobytes(), fr["acc"].tobytes(), o.t, o.Lx, o.Ly,
            o.xi, o.nph_area_momentum, o.last_instant_pressure, o.steps, o.rebuilds)


def _drive(sim):
    out = []
    sim.step_single_nose_hoover(nsteps=1)
    sim.step_single_nose_hoover(nsteps=257)
    out.append(_state(sim))
    sim.step_single_NVE(nsteps=131)
    out.append((_state(sim), sim.cal_total_K(), sim.cal_total_U()))
    sim.step_single_NPH(1.4, nsteps=90)
    sim.step_single_NPH(1.4, nsteps=7)
    out.append((_state(sim), sim.cal_instant_pressure()))
    sim.step_single_nose_hoover(nsteps=33)
    out.append(_state(sim))
    return out


@pytest.mark.parametrize("N", [900, 4096, 30000])
def test_multi_step_bit_identical(built, N):
    f, cfg = _system(N)
    per = mdb.MDSimulation(cfg, frame=f, step_kernel=mdb.STEPS_PER_PHASE)
    multi = mdb.MDSimulation(cfg, frame=f, step_kernel=mdb.STEPS_MULTI)
    assert per.schedule()["multi_step"] == 0
    assert multi.schedule()["multi_step"] == 1
    a, b = _drive(per), _drive(multi)
    assert a == b
    # rebuilds happened inside the run (the graph's rebuild branch ran)
    assert a[-1][-1] > 5


def test_multi_step_default_choice(built):
    small, cfg = _system(4096)
    s = mdb.MDSimulation(cfg, frame=small).schedule()
    assert s["multi_step"] == 1 and s["multi_step_blocks"] >= 148
    big, cfg = _system(262144)
    assert mdb.MDSimulation(cfg, frame=big).schedule()["multi_step"] == 0


def test_multi_step_short_and_repeated_calls(built):
    f, cfg = _system(2000, seed=3)
    a = mdb.MDSimulation(cfg, frame=f, step_kernel=mdb.STEPS_PER_PHASE)
    b = mdb.MDSimulation(cfg, frame=f, step_kernel=mdb.STEPS_MULTI)
    for sim in (a, b):
        sim.step_single_NVE(nsteps=0)
        for k in range(40):
            sim.step_single_nose_hoover(nsteps=1 + (k % 5))
    assert _state(a) == _state(b)
