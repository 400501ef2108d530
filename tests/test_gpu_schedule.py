"""The engine-schedule autotuner (mdb_options_t.autotune).

It times schedule candidates at build (the list prefetch depth of the force
phase, the list-build grid, the grid of the other rebuild kernels) and keeps
the fastest, cached per device and workload shape in MDB_SCHEDULE_CACHE. None
of those knobs changes what is computed, so a tuned handle gives bit for bit
the results of an untuned one.
"""
import numpy as np
import pytest

import md_simulation_cuda_b200 as mdb
from md_simulation_cuda_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _frames_equal(a, b):
    a.sample_collect()
    b.sample_collect()
    fa, fb = a.get_host_particles(), b.get_host_particles()
    return (np.array_equal(fa["pos"], fb["pos"]) and np.array_equal(fa["vel"], fb["vel"])
            and np.array_equal(fa["acc"], fb["acc"]))


@pytest.mark.parametrize("case", ["nve_4096", "slab_40k"])
def test_tuned_schedule_is_bit_identical(built, tmp_path, monkeypatch, case):
    cache = tmp_path / "schedule.txt"
    monkeypatch.setenv("MDB_SCHEDULE_CACHE", str(cache))
    if case == "nve_4096":
        f, cfg = wl.nve_4096()
    else:
        f, cfg = wl.nvt_slab(N=40000, seed=5)
    plain = mdb.MDSimulation(cfg, frame=f)
    tuned = mdb.MDSimulation(cfg, frame=f, autotune=True)
    sp, st = plain.schedule(), tuned.schedule()
    assert sp["tuned"] == 0 and st["tuned"] == 1 and st["from_cache"] == 0
    assert cache.exists() and cache.read_text().count("\n") == 1
    for sim in (plain, tuned):
        sim.step_single_nose_hoover(nsteps=150)
        sim.step_single_NVE(nsteps=50)
    assert _frames_equal(plain, tuned)
    assert plain.cal_total_K() == tuned.cal_total_K()
    assert plain.cal_total_U() == tuned.cal_total_U()
    assert plain.xi == tuned.xi
    # a second handle of the same shape reads the choice from the cache
    again = mdb.MDSimulation(cfg, frame=f, autotune=True)
    sa = again.schedule()
    assert sa["from_cache"] == 1 and sa["tuned"] == 1
    for k in ("list_prefetch_rows", "nlist_grid", "rebuild_grid"):
        assert sa[k] == st[k]


def test_tuned_fire_batch_is_bit_identical(built, tmp_path, monkeypatch):
    monkeypatch.setenv("MDB_SCHEDULE_CACHE", str(tmp_path / "schedule.txt"))
    systems = wl.fire_mix(6, seed=9, n_min=64, n_max=900)
    params = mdb.FireParams(dt_init=0.001, dt_max=0.01)
    res = []
    for tune in (False, True):
        b = mdb.Batch(autotune=tune)
        for f, cfgd in systems:
            b.add_fire(cfgd, f, 1e-6, 300, params)
        b.run()
        assert b.schedule()["tuned"] == (1 if tune else 0)
        res.append([b.fire_result(k) for k in range(len(systems))])
    for a, b in zip(*res):
        assert a.steps == b.steps and a.converged == b.converged
        assert np.array_equal(a.frame["pos"], b.frame["pos"])
        assert np.array_equal(a.energy_trace, b.energy_trace)
