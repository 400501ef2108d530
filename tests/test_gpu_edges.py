"""Edge cases of the force and step paths against the oracle: a single
particle, neighbour lists that overflow (the stencil fallback), no lists at
all, 32-bit list offsets (a very elongated box), and a batch mixing a
one-particle system with ordinary ones."""
import numpy as np
import pytest

import md_simulation_cuda_b200 as mdb
from md_simulation_cuda_b200 import workloads as wl
from oracle import pyoracle as po
from tests.helpers import rel_err, rel_l2

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5


def test_single_particle(built):
    L = 12.0
    cfg = wl.config_dict(1, L, L, dt=0.01)
    f = mdb.make_frame(1)
    f["pos"] = [[3.0, 4.0]]
    f["vel"] = [[0.5, -0.25]]
    sim = mdb.MDSimulation(cfg, frame=f)
    sim.step_single_NVE(nsteps=100)
    sim.sample_collect()
    g = sim.get_host_particles()
    assert np.allclose(g["pos"][0], [(3.0 + 0.5) % L, (4.0 - 0.25) % L], atol=1e-12)
    assert sim.cal_total_U() == 0.0 and np.all(g["acc"] == 0.0)
    res = mdb.EnergyMinimizer(dict(cfg, n_cap=1)).minimize_frame(
        f, 1e-6, 100, mdb.FireParams.from_config(cfg))
    assert res.converged and res.max_force == 0.0


@pytest.mark.parametrize("max_neighbors", [6, -1])
def test_list_overflow_and_no_lists(built, max_neighbors):
    """max_neighbors 6: most lists overflow and those particles scan their
    stencil; -1: no lists. Forces stay on the FP64 oracle, and a short
    trajectory on the one computed with full lists (the stencil and the list
    visit the partners in different orders, so the FP32 sums differ in their
    last bits; over 50 steps that grows to a few 1e-9)."""
    f, cfg = wl.nve_4096(seed=9)
    Lx, Ly = cfg["box_w_global"], cfg["box_h_global"]
    acc, U, W = mdb.compute_forces(cfg, f, Lx, Ly, max_neighbors=max_neighbors)
    ref, U0, W0 = po.forces(cfg, f["pos"], f["type"], Lx, Ly, mode=po.OR_FP64)
    assert rel_l2(acc, ref) <= FORCE_TOL
    assert rel_err(U, U0) <= 1e-6 and rel_err(W, W0) <= 1e-6
    a = mdb.MDSimulation(cfg, frame=f)
    b = mdb.MDSimulation(cfg, frame=f, max_neighbors=max_neighbors)
    a.step_single_NVE(nsteps=50)
    b.step_single_NVE(nsteps=50)
    a.sample_collect()
    b.sample_collect()
    d = a.get_host_particles()["pos"] - b.get_host_particles()["pos"]
    assert np.max(np.abs(d)) < 1e-8


def test_int32_list_offsets(built):
    """A 3-cell-high strip with ~13,000 particles per cell row: list offsets
    exceed 16 bits and the engine keeps 32-bit lists."""
    N, rho, Ly = 40000, 0.8, 9.0
    Lx = N / (rho * Ly)
    f, _, _ = wl.lattice_frame(N, rho, Lx / Ly, 0.65, 1.0, seed=13, jitter=0.1)
    cfg = wl.config_dict(N, Lx, Ly, dt=0.001)
    acc, U, W = mdb.compute_forces(cfg, f, Lx, Ly)
    ref, U0, W0 = po.forces(cfg, f["pos"], f["type"], Lx, Ly, mode=po.OR_FP64, cells=True)
    assert rel_l2(acc, ref) <= FORCE_TOL
    assert rel_err(U, U0) <= 1e-6 and rel_err(W, W0) <= 1e-6


def test_batch_with_a_single_particle_system(built):
    systems = []
    for k, N in enumerate([1, 700, 2500]):
        if N == 1:
            L = 10.0
            f = mdb.make_frame(1)
            f["pos"] = [[1.0, 2.0]]
            f["vel"] = [[0.1, 0.2]]
            cfg = wl.config_dict(1, L, L, dt=0.002, T=0.5)
        else:
            f, Lx, Ly = wl.lattice_frame(N, 0.8, 1.0, 0.65, 0.9, seed=70 + k, jitter=0.1)
            cfg = wl.config_dict(N, Lx, Ly, dt=0.002, T=0.9)
        systems.append((f, cfg))
    b = mdb.Batch()
    for f, cfg in systems:
        b.add_md(cfg, f, mdb.JOB_NVE, 80)
    b.run(-1)
    for sid, (f, cfg) in enumerate(systems):
        # the batch's setting: one lane per particle
        sim = mdb.MDSimulation(cfg, frame=f, lanes=mdb.LANES_ONE)
        sim.step_single_NVE(nsteps=80)
        sim.sample_collect()
        assert np.array_equal(b.frame(sid)["pos"], sim.get_host_particles()["pos"])
