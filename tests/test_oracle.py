"""The CPU oracle pinned against analytic known answers (the reference ships no
golden vectors for forces or integrators; see oracle/mdoracle.h)."""
import math

import numpy as np
import pytest

from md_simulation_cuda_b200 import workloads as wl
from oracle import pyoracle as po
from tests.helpers import rel_l2

CFG1 = dict(SIGMA_AA=1.0, SIGMA_BB=1.0, SIGMA_AB=1.0, EPSILON_AA=1.0, EPSILON_BB=1.0,
            EPSILON_AB=1.0, MASS_A=1.0, MASS_B=1.0, cutoff=2.5, dt=1e-3, Q=1.0, T_target=1.0)


@pytest.mark.parametrize("mode,tol", [(po.OR_FP64, 1e-12), (po.OR_REF_MIXED, 2e-6)])
@pytest.mark.parametrize("r", [0.9, 1.0, 2 ** (1 / 6), 1.7, 2.49])
def test_two_particle_force_energy_virial(mode, tol, r):
    pos = np.array([[5.0, 5.0], [5.0 + r, 5.0]])
    acc, U, W = po.forces(CFG1, pos, [0, 0], 10.0, 10.0, mode=mode)
    F = 24 * (2 * r ** -13 - r ** -7)
    Vc = 4 * (2.5 ** -12 - 2.5 ** -6)
    assert abs(acc[0, 0] + F) <= tol * max(1, abs(F))
    assert abs(acc[1, 0] - F) <= tol * max(1, abs(F))
    assert abs(U - (4 * (r ** -12 - r ** -6) - Vc)) <= tol * max(1, abs(U))
    assert abs(W - F * r) <= tol * max(1, abs(W))


def test_cutoff_is_strict_and_per_pair_type():
    cfg = dict(wl.LJ, dt=1e-3, Q=1.0, T_target=1.0)
    # AB cutoff = 2.5 * 0.8 = 2.0: just inside / outside
    for r, expect in ((1.999, True), (2.001, False)):
        acc, _, _ = po.forces(cfg, [[1, 1], [1 + r, 1]], [0, 1], 20, 20)
        assert (acc[0, 0] != 0) == expect
    # BB cutoff = 2.2
    acc, _, _ = po.forces(cfg, [[1, 1], [3.1, 1]], [1, 1], 20, 20)
    assert acc[0, 0] != 0
    acc, _, _ = po.forces(cfg, [[1, 1], [3.3, 1]], [1, 1], 20, 20)
    assert acc[0, 0] == 0


def test_periodic_images():
    pos = np.array([[0.2, 5.0], [9.5, 5.0]])  # 0.7 apart through x = 0
    acc, U, _ = po.forces(CFG1, pos, [0, 0], 10.0, 10.0)
    acc2, U2, _ = po.forces(CFG1, [[5.0, 5.0], [5.7, 5.0]], [0, 0], 10.0, 10.0)
    # particle 0 sits to the right of particle 1 through the boundary
    assert acc[0, 0] == pytest.approx(-acc2[0, 0], rel=1e-11)
    assert U == pytest.approx(U2, rel=1e-12)


def test_square_lattice_energy():
    """Perfect square lattice (spacing a): per-particle energy is the lattice
    sum over neighbour shells inside the cutoff."""
    a, m = 1.1, 20
    L = a * m
    g = (np.stack(np.meshgrid(np.arange(m), np.arange(m)), -1).reshape(-1, 2) + 0.5) * a
    acc, U, _ = po.forces(CFG1, g, np.zeros(m * m, np.int32), L, L)
    Vc = 4 * (2.5 ** -12 - 2.5 ** -6)
    e = 0.0
    for i in range(-3, 4):
        for j in range(-3, 4):
            if i == 0 and j == 0:
                continue
            r = a * math.hypot(i, j)
            if r < 2.5:
                e += 0.5 * (4 * (r ** -12 - r ** -6) - Vc)
    assert U / (m * m) == pytest.approx(e, rel=1e-12)
    assert np.abs(acc).max() < 1e-10


def test_cells_equal_allpairs():
    f, cfg = wl.nve_4096()
    L = cfg["box_w_global"]
    for mode in (po.OR_FP64, po.OR_REF_MIXED):
        a1, U1, W1 = po.forces(cfg, f["pos"], f["type"], L, L, mode=mode)
        a2, U2, W2 = po.forces(cfg, f["pos"], f["type"], L, L, mode=mode, cells=True)
        assert np.abs(a1 - a2).max() <= 1e-12 * np.abs(a1).max()
        assert U1 == pytest.approx(U2, rel=1e-13)
        assert W1 == pytest.approx(W2, rel=1e-13)


def test_reference_mixed_precision_error():
    """The reference's own arithmetic meets the 1e-5 force bound on the NVE
    workload (its error is dominated by the FP32 cast of the unwrapped
    periodic displacement)."""
    f, cfg = wl.nve_4096()
    L = cfg["box_w_global"]
    a64, _, _ = po.forces(cfg, f["pos"], f["type"], L, L, mode=po.OR_FP64)
    amx, _, _ = po.forces(cfg, f["pos"], f["type"], L, L, mode=po.OR_REF_MIXED)
    e = rel_l2(amx, a64)
    assert 1e-8 < e < 1e-5


def test_ws1_halo_duplication():
    """At world size 1 the reference counts partners in the x-boundary strips
    twice (H1); interior particles far from both strips are unaffected."""
    cfg = dict(CFG1)
    L = 30.0
    pos = np.array([[15.0, 5.0], [16.1, 5.0], [0.5, 5.0], [29.4, 5.0]])
    a0, U0, _ = po.forces(cfg, pos, [0] * 4, L, L)
    a1, U1, _ = po.forces(cfg, pos, [0] * 4, L, L, ws1_halo=1)
    assert np.allclose(a0[:2], a1[:2])  # pair (0,1) far from the strips
    assert np.allclose(a1[2:], 2 * a0[2:])  # the boundary pair counted twice
    assert U1 == pytest.approx(1.5 * U0, rel=1e-12)  # 3 pair energies instead of 2


def test_newton_and_momentum_conservation_nve():
    f, cfg = wl.nve_4096(seed=3)
    s = po.Sim(cfg, f["pos"], f["vel"], f["type"])
    p0 = s.vel.sum(0)
    s.step_nve(20)
    assert np.abs(s.vel.sum(0) - p0).max() < 1e-10


def test_binning_stable_and_complete():
    rng = np.random.default_rng(0)
    pos = rng.uniform(0, 40, (5000, 2))
    cell, perm, ncx, ncy = po.cell_build(pos, 40.0, 40.0, 2.8)
    assert ncx == ncy == 14
    assert sorted(perm.tolist()) == list(range(5000))
    c = cell[perm]
    assert np.all(np.diff(c) >= 0)
    same = np.diff(c) == 0
    assert np.all(np.diff(perm)[same] > 0)  # stable


def test_fire_two_particles_reach_minimum():
    r = po.fire_minimize(CFG1, [[1.0, 1.0], [3.0, 1.0]], [0, 0], 10.0, 10.0, 1e-8, 20000,
                         dict(dt_init=1e-3, dt_max=5e-3, alpha0=0.1, f_inc=1.1, f_dec=0.5,
                              N_min=5))
    assert r["converged"]
    d = r["pos"][1] - r["pos"][0]
    assert abs(np.hypot(*d) - 2 ** (1 / 6)) < 1e-8


def test_nh_thermostat_holds_temperature():
    f, Lx, Ly = wl.lattice_frame(400, 0.7, 1.0, 0.6, 1.5, seed=4)
    cfg = wl.config_dict(400, Lx, Ly, dt=0.002, T=0.8, Q=1.0)
    s = po.Sim(cfg, f["pos"], f["vel"], f["type"])
    ts = []
    for _ in range(150):
        s.step_nose_hoover(10)
        ts.append(2 * s.total_K() / (2 * 400 - 2))
    assert abs(np.mean(ts[50:]) - 0.8) < 0.08


def test_partial_U_lambda_two_particles():
    """dU/dlambda of the area-preserving stretch: a pair along x contributes
    -eps_lambda * tmp * r^2 (both ordered pairs, each halved), along y the
    opposite sign (src/md_cuda_common.cu:345-355)."""
    from md_simulation_cuda_b200 import workloads as wl

    cfg = wl.config_dict(2, 10.0, 10.0, dt=0.001, SIGMA_BB=1.0, SIGMA_AB=1.0, EPSILON_BB=1.0,
                         EPSILON_AB=1.0)
    for r in (0.97, 1.1, 1.5, 2.3):
        tmp = 24 * (2 * r ** -14 - r ** -8)
        for mode in (po.OR_FP64, po.OR_REF_MIXED):
            vx, _ = po.partial_U_lambda(cfg, np.array([[9.8, 5.0], [(9.8 + r) % 10, 5.0]]),
                                        [0, 0], 10.0, 10.0, 0.01, mode=mode)
            vy, _ = po.partial_U_lambda(cfg, np.array([[5.0, 1.0], [5.0, 1.0 + r]]), [0, 0],
                                        10.0, 10.0, 0.01, mode=mode)
            # the mixed mode casts the unwrapped FP64 difference across the
            # periodic edge to FP32 (the reference's own error, ~2e-5 here)
            tol = 1e-12 if mode == po.OR_FP64 else 1e-4
            assert abs(vx + 0.01 * tmp * r * r) <= tol * abs(tmp * r * r) * 0.01 + 1e-14
            assert abs(vy - 0.01 * tmp * r * r) <= tol * abs(tmp * r * r) * 0.01 + 1e-14


def test_pressure_profile_sum_rule():
    """Summed over the bins, the Irving-Kirkwood profile gives back the scalar
    pressure's parts: sum (Pxx + Pyy) * bin area = sum m v^2 + W, with
    W = 1/2 sum over ordered pairs of r.F (src/md_cuda_common.cu:873-1030 vs
    :591-701)."""
    from md_simulation_cuda_b200 import workloads as wl

    f, Lx, Ly = wl.lattice_frame(400, 0.8, 1.0, 0.65, 1.0, seed=1)
    cfg = wl.config_dict(400, Lx, Ly, dt=0.001)
    nb = 10
    xx, yy, xy = po.pressure_profile(cfg, f["pos"], f["vel"], f["type"], Lx, Ly, nb)
    kin = float((f["vel"] ** 2).sum())  # unit masses
    _, _, W = po.forces(cfg, f["pos"], f["type"], Lx, Ly, mode=po.OR_FP64)
    total = (xx.sum() + yy.sum()) * (Lx * Ly / nb)
    assert abs(total - (kin + W)) <= 1e-9 * (kin + abs(W))
    a, b = po.n_profile(f["pos"], f["type"], Lx, nb)
    assert a.sum() + b.sum() == 400 and a.sum() == int((f["type"] == 0).sum())
