"""Independent systems over several devices (mdb_multibatch_*).

The GPU machine of the test run has one GPU, so the device list names device
0 twice: the systems are placed on two sub-batches (two engines, two streams)
by the library's LPT rule and run concurrently. Each system's results must be
bit for bit those of the same system in one plain batch, since a batch
evolves every system as it would run alone.
"""
import numpy as np
import pytest

import md_simulation_cuda_b200 as mdb
from md_simulation_cuda_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def test_fire_systems_over_two_sub_batches(built):
    systems = wl.fire_mix(10, seed=12, n_min=64, n_max=1200)
    params = mdb.FireParams(dt_init=0.001, dt_max=0.01)
    one = mdb.Batch()
    multi = mdb.MultiBatch(devices=[0, 0])
    for f, cfgd in systems:
        one.add_fire(cfgd, f, 1e-6, 500, params)
        multi.add_fire(cfgd, f, 1e-6, 500, params)
    one.run()
    multi.run()
    place = multi.placement()
    assert place.tolist() == [0] * len(systems)  # device ids (both sub-batches on device 0)
    assert multi.progress() == (len(systems), len(systems))
    for k in range(len(systems)):
        a, b = one.fire_result(k), multi.fire_result(k)
        assert a.steps == b.steps and a.converged == b.converged
        assert np.array_equal(a.frame["pos"], b.frame["pos"])
        assert np.array_equal(a.energy_trace, b.energy_trace)


def test_md_segments_over_two_sub_batches(built):
    specs = [wl.lattice_frame(n, 0.8, 1.0, 0.6, 1.0, seed=40 + n) for n in (300, 900, 2000, 700)]
    one = mdb.Batch()
    multi = mdb.MultiBatch(devices=[0, 0])
    steps = [120, 40, 80, 200]
    for (f, Lx, Ly), st in zip(specs, steps):
        cfgd = wl.config_dict(len(f), Lx, Ly, dt=0.001, T=1.0)
        one.add_md(cfgd, f, mdb.JOB_NVT, st)
        multi.add_md(cfgd, f, mdb.JOB_NVT, st)
    one.run()
    multi.run()
    for k, st in enumerate(steps):
        assert multi.system_info(k)[2] == st
        assert np.array_equal(one.frame(k)["pos"], multi.frame(k)["pos"])
        assert one.energies(k) == multi.energies(k)
