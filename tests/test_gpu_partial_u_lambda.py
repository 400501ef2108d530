"""cal_partial_U_lambda (the lambda derivative of the area-preserving
deformation, src/md_env.cu:2362-2406) on the GPU against the FP64 oracle:
|dU/dlambda - oracle| <= 1e-6 * sum of |Fx dx| + |Fy dy| (the sum cancels for
an isotropic liquid, so the bound is stated against its magnitude)."""
import numpy as np
import pytest

import md_simulation_cuda_b200 as mdb
from md_simulation_cuda_b200 import workloads as wl
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

EPS = 0.01


@pytest.mark.parametrize("N,aspect,seed", [(2000, 2.0, 1), (3000, 1.0, 2)])
def test_partial_U_lambda_vs_fp64(built, N, aspect, seed):
    f, Lx, Ly = wl.lattice_frame(N, 0.85, aspect, 0.6, 1.0, seed=seed, jitter=0.15)
    cfg = wl.config_dict(N, Lx, Ly, dt=0.001)
    sim = mdb.MDSimulation(cfg, frame=f)
    got = sim.cal_partial_U_lambda(EPS)
    ref, scale = po.partial_U_lambda(cfg, f["pos"], f["type"], Lx, Ly, EPS)
    assert abs(got - ref) <= 1e-6 * scale


def test_partial_U_lambda_two_particles(built):
    L = 10.0
    cfg = wl.config_dict(2, L, L, dt=0.001, SIGMA_BB=1.0, SIGMA_AB=1.0, EPSILON_BB=1.0,
                         EPSILON_AB=1.0)
    for r in (0.97, 1.1, 1.5):
        tmp = 24 * (2 * r ** -14 - r ** -8)
        f = mdb.make_frame(2)
        f["pos"] = [[9.8, 5.0], [(9.8 + r) % L, 5.0]]  # across the periodic x edge
        v = mdb.MDSimulation(cfg, frame=f).cal_partial_U_lambda(EPS)
        assert abs(v + EPS * tmp * r * r) <= 1e-5 * EPS * abs(tmp) * r * r


def test_partial_U_lambda_piston_convention(built):
    """In piston mode the y axis is not periodic (src/md_env.cu:2369)."""
    f, Lx, Ly = wl.lattice_frame(1500, 0.8, 2.0, 0.65, 0.8, seed=4, jitter=0.1)
    cfg = wl.config_dict(1500, Lx, Ly, dt=0.001, barostat_mass=10.0, k_piston=100.0)
    sim = mdb.MDSimulation(cfg, frame=f)
    sim.step_single_NPH_piston(1.0, nsteps=5)
    frame = sim.get_host_particles()
    got = sim.cal_partial_U_lambda(EPS)
    ref, scale = po.partial_U_lambda(cfg, frame["pos"], frame["type"], sim.get_Lx(),
                                     sim.get_Ly(), EPS, periodic_y=0)
    assert abs(got - ref) <= 1e-6 * scale


def test_partial_U_lambda_batch_equals_solo(built):
    b = mdb.Batch()
    solos = []
    for k, T in enumerate((0.6, 0.9, 1.2)):  # a temperature sweep as one batch
        f, Lx, Ly = wl.lattice_frame(1200, 0.8, 1.0, 0.65, T, seed=60 + k, jitter=0.1)
        cfg = wl.config_dict(1200, Lx, Ly, dt=0.002, T=T)
        b.add_md(cfg, f, mdb.JOB_NVT, 100)
        # the batch's setting: one lane per particle
        sim = mdb.MDSimulation(cfg, frame=f, lanes=mdb.LANES_ONE)
        sim.step_single_nose_hoover(nsteps=100)
        solos.append(sim.cal_partial_U_lambda(EPS))
    b.run(-1)
    assert np.array_equal(b.partial_U_lambda(EPS), np.array(solos))
