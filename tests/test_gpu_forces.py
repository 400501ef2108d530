"""Force/energy/virial parity of the sm_100a pair kernel against the CPU oracle.

Tolerance (the accuracy bound): relative force error ||F_gpu - F_fp64|| /
||F_fp64|| <= 1e-5 against the FP64 oracle. Energies and virials are FP64
reductions of FP32 pair terms: relative 1e-6.
"""
import numpy as np
import pytest

import md_simulation_cuda_b200 as mdb
from md_simulation_cuda_b200 import workloads as wl
from oracle import pyoracle as po
from tests.helpers import rel_err, rel_l2

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5


def _frame(pos, types):
    f = mdb.make_frame(len(types))
    f["pos"] = pos
    f["type"] = types
    return f


def test_forces_nve4096_vs_fp64(built):
    f, cfg = wl.nve_4096()
    Lx, Ly = cfg["box_w_global"], cfg["box_h_global"]
    acc, U, W = mdb.compute_forces(cfg, f, Lx, Ly)
    ref, U0, W0 = po.forces(cfg, f["pos"], f["type"], Lx, Ly, mode=po.OR_FP64)
    assert rel_l2(acc, ref) <= FORCE_TOL
    assert rel_err(U, U0) <= 1e-6
    assert rel_err(W, W0) <= 1e-6


def test_forces_more_accurate_than_reference_mixed(built):
    """The float-float displacement keeps the periodic pairs exact, which the
    reference's FP32 cast of the unwrapped difference does not."""
    f, cfg = wl.nve_4096(seed=5)
    Lx, Ly = cfg["box_w_global"], cfg["box_h_global"]
    acc, _, _ = mdb.compute_forces(cfg, f, Lx, Ly)
    ref64, _, _ = po.forces(cfg, f["pos"], f["type"], Lx, Ly, mode=po.OR_FP64)
    mixed, _, _ = po.forces(cfg, f["pos"], f["type"], Lx, Ly, mode=po.OR_REF_MIXED)
    e_gpu = rel_l2(acc, ref64)
    e_ref = rel_l2(mixed, ref64)
    assert e_gpu <= FORCE_TOL and e_ref <= FORCE_TOL
    assert e_gpu < e_ref
    assert rel_l2(acc, mixed) <= FORCE_TOL


@pytest.mark.parametrize("N,aspect,seed", [(2000, 2.0, 1), (5000, 0.5, 2), (700, 1.0, 3)])
def test_forces_random_lattices(built, N, aspect, seed):
    f, Lx, Ly = wl.lattice_frame(N, 0.85, aspect, 0.5, 1.0, seed=seed, jitter=0.15)
    cfg = wl.config_dict(N, Lx, Ly, dt=0.001)
    acc, U, W = mdb.compute_forces(cfg, f, Lx, Ly)
    ref, U0, W0 = po.forces(cfg, f["pos"], f["type"], Lx, Ly, mode=po.OR_FP64)
    assert rel_l2(acc, ref) <= FORCE_TOL
    assert rel_err(U, U0) <= 1e-6
    assert rel_err(W, W0) <= 1e-6


def test_forces_other_types_use_ab(built):
    """Types other than 0/1 pair with everything through the AB parameters and
    take MASS_B (src/md_cuda_common.cu:218-229, 261)."""
    rng = np.random.default_rng(7)
    f, Lx, Ly = wl.lattice_frame(1500, 0.8, 1.0, 0.5, 1.0, seed=7)
    f["type"] = rng.integers(0, 4, len(f))
    cfg = wl.config_dict(len(f), Lx, Ly, dt=0.001, MASS_B=2.0)
    acc, U, W = mdb.compute_forces(cfg, f, Lx, Ly)
    ref, U0, W0 = po.forces(cfg, f["pos"], f["type"], Lx, Ly, mode=po.OR_FP64)
    assert rel_l2(acc, ref) <= FORCE_TOL
    assert rel_err(U, U0) <= 1e-6


def test_forces_small_box_all_pairs(built):
    """Boxes narrower than three cells use the all-pairs loop with the nearest
    image, as the reference's O(N^2) kernel does."""
    rng = np.random.default_rng(3)
    L = 6.0
    pos = rng.uniform(0, L, (24, 2))
    types = rng.integers(0, 2, 24)
    f = _frame(pos, types)
    cfg = wl.config_dict(24, L, L, dt=0.001)
    acc, U, W = mdb.compute_forces(cfg, f, L, L)
    ref, U0, W0 = po.forces(cfg, pos, types, L, L, mode=po.OR_FP64)
    assert rel_l2(acc, ref) <= FORCE_TOL
    assert rel_err(U, U0) <= 1e-6


def test_forces_nonperiodic_y(built):
    """periodic_y = 0 (the LJ part of the piston walls): no y images."""
    f, Lx, Ly = wl.lattice_frame(3000, 0.8, 2.0, 0.65, 1.0, seed=9)
    cfg = wl.config_dict(3000, Lx, Ly, dt=0.001)
    acc, U, W = mdb.compute_forces(cfg, f, Lx, Ly, periodic_y=False)
    ref, U0, W0 = po.forces(cfg, f["pos"], f["type"], Lx, Ly, periodic_y=0, mode=po.OR_FP64)
    assert rel_l2(acc, ref) <= FORCE_TOL
    assert rel_err(U, U0) <= 1e-6


def test_two_particle_analytic(built):
    """F = 24 eps (2 r^-13 - r^-7) along the separation, U = 4(r^-12-r^-6) - V_c,
    across the periodic boundary too."""
    L = 10.0
    cfg = wl.config_dict(2, L, L, dt=0.001, SIGMA_BB=1.0, SIGMA_AB=1.0, EPSILON_BB=1.0,
                         EPSILON_AB=1.0)
    Vc = 4 * (2.5 ** -12 - 2.5 ** -6)
    for r in (0.95, 1.1, 1.5, 2.4):
        for x0 in (1.0, 9.5):  # second case straddles x = 0
            pos = np.array([[x0, 5.0], [(x0 + r) % L, 5.0]])
            acc, U, W = mdb.compute_forces(cfg, _frame(pos, [0, 0]), L, L)
            F = 24 * (2 * r ** -13 - r ** -7)
            # FP32 pair term; near the minimum 2 sr^12 - sr^6 cancels ~8x
            assert abs(acc[0, 0] + F) <= 1e-5 * abs(F) + 1e-6
            assert abs(acc[1, 0] - F) <= 1e-5 * abs(F) + 1e-6
            U0 = 4 * (r ** -12 - r ** -6) - Vc
            assert abs(U - U0) <= 1e-6 * (1.0 + abs(U0))  # FP32 pair energy
    # beyond the cutoff: nothing
    pos = np.array([[1.0, 5.0], [3.6, 5.0]])
    acc, U, W = mdb.compute_forces(cfg, _frame(pos, [0, 0]), L, L)
    assert np.all(acc == 0.0) and U == 0.0


def test_newton_third_law(built):
    f, cfg = wl.nve_4096(seed=8)
    acc, _, _ = mdb.compute_forces(cfg, f, cfg["box_w_global"], cfg["box_h_global"])
    net = acc.sum(axis=0)  # unit masses
    assert np.all(np.abs(net) <= 1e-9 * np.abs(acc).sum())
