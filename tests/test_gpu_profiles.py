"""Density and Irving-Kirkwood pressure-tensor profiles (get_N_profile,
get_density_profile, get_pressure_profile; src/md_env.cu:3821-4104) on the GPU
against the oracle: counts bit for bit; pressure bins within 1e-5 of the
largest bin against the FP64 oracle (FP32 pair terms); sums reproducible bit
for bit (fixed-point accumulation)."""
import numpy as np
import pytest

import md_simulation_cuda_b200 as mdb
from md_simulation_cuda_b200 import workloads as wl
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def _slab(N=3000, seed=11):
    f, Lx, Ly = wl.lattice_frame(N, 0.8, 2.0, lambda s: np.where(s < 0.5, 0.9, 0.1), 0.8,
                                 seed=seed, jitter=0.1)
    return f, Lx, Ly, wl.config_dict(N, Lx, Ly, dt=0.002, T=0.8)


def test_n_and_density_profiles_bit_exact(built):
    f, Lx, Ly, cfg = _slab()
    sim = mdb.MDSimulation(cfg, frame=f)
    sim.step_single_nose_hoover(nsteps=50)
    sim.sample_collect()
    g = sim.get_host_particles()
    nb = 16
    a, b = po.n_profile(g["pos"], g["type"], sim.get_Lx(), nb)
    got = sim.get_N_profile(nb)
    assert np.array_equal(got[:nb], a) and np.array_equal(got[nb:], b)
    dens = sim.get_density_profile(nb)
    s = a + b
    ref = np.where(s > 0, (a - b) / np.maximum(s, 1), 0.0)
    assert np.array_equal(dens, ref)
    assert dens[1] > 0.5 and dens[nb - 2] < -0.5  # A-rich then B-rich stripe


def test_pressure_profile_vs_fp64(built):
    f, Lx, Ly, cfg = _slab(seed=12)
    sim = mdb.MDSimulation(cfg, frame=f)
    sim.step_single_nose_hoover(nsteps=30)
    sim.sample_collect()
    g = sim.get_host_particles()
    nb = 12
    got = sim.get_pressure_profile(nb)
    xx, yy, xy = po.pressure_profile(cfg, g["pos"], g["vel"], g["type"], sim.get_Lx(),
                                     sim.get_Ly(), nb)
    ref = np.concatenate([xx, yy, xy])
    assert np.max(np.abs(got - ref)) <= 1e-5 * np.max(np.abs(ref))
    again = sim.get_pressure_profile(nb)
    assert np.array_equal(got, again)  # order-independent sums


def test_pressure_profile_matches_scalar_pressure(built):
    """Bin sums give back the scalar pressure: mean over bins of
    (Pxx + Pyy) / 2 = P (src/md_env.cu:2205-2266)."""
    f, cfg = wl.nve_4096(seed=4)
    sim = mdb.MDSimulation(cfg, frame=f)
    sim.step_single_NVE(nsteps=20)
    nb = 8
    p = sim.get_pressure_profile(nb)
    P = sim.cal_instant_pressure()
    assert abs((p[:nb].mean() + p[nb:2 * nb].mean()) / 2 - P) <= 1e-6 * (1 + abs(P))
