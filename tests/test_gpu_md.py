"""Integrator parity (NVE, Nose-Hoover, NPH, piston) of the CUDA path against
the CPU oracle, through the C ABI (MDSimulation mirror).

The GPU pair term is FP32 (relative force error ~1e-7..1e-6 against FP64), so
single trajectories separate slowly (chaos); short horizons are compared per
particle, long horizons through collective quantities.
"""
import numpy as np
import pytest

import md_simulation_cuda_b200 as mdb
from md_simulation_cuda_b200 import workloads as wl
from oracle import pyoracle as po
from tests.helpers import min_image, rel_err

pytestmark = pytest.mark.gpu


def _pair(frame, cfg, mode=po.OR_FP64, **kw):
    sim = mdb.MDSimulation(cfg, frame=frame, **kw)
    orc = po.Sim(cfg, frame["pos"], frame["vel"], frame["type"], mode=mode)
    return sim, orc


def _maxdx(sim, orc, L):
    sim.sample_collect()
    g = sim.get_host_particles()
    return float(np.abs(min_image(g["pos"] - orc.pos, L)).max()), g


def test_nve_short_horizon_per_particle(built):
    f, cfg = wl.nve_4096()
    L = np.array([cfg["box_w_global"], cfg["box_h_global"]])
    sim, orc = _pair(f, cfg)
    sim.step_single_NVE(nsteps=10)
    orc.step_nve(10)
    dx, g = _maxdx(sim, orc, L)
    assert dx < 1e-8
    assert np.abs(g["vel"] - orc.vel).max() < 1e-6
    assert np.abs(g["acc"] - orc.acc).max() < 1e-5 * np.abs(orc.acc).max()


def test_nve_1000_steps_energies(built):
    """Config NVE N=4096, dt=0.001, 1000 steps: per-step KE/PE against the
    FP64 oracle, and total-energy drift."""
    f, cfg = wl.nve_4096()
    sim, orc = _pair(f, cfg)
    E0 = sim.cal_total_K() + sim.cal_total_U()
    for block in range(10):
        sim.step_single_NVE(nsteps=100)
        orc.step_nve(100)
        K, U = sim.cal_total_K(), sim.cal_total_U()
        K0, U0 = orc.total_K(), orc.total_U()
        assert rel_err(K, K0) < 1e-5, (block, K, K0)
        assert rel_err(U, U0) < 1e-5, (block, U, U0)
    E1 = sim.cal_total_K() + sim.cal_total_U()
    assert abs(E1 - E0) / abs(E0) < 2e-4
    assert abs(sim.t - 1.0) < 1e-12


def test_nose_hoover_slab(built):
    f, Lx, Ly = wl.lattice_frame(4096, 0.8, 2.0, lambda s: np.where(s < 0.5, 0.9, 0.1), 0.7,
                                 seed=21)
    cfg = wl.config_dict(4096, Lx, Ly, dt=0.002, T=0.7, Q=1.0)
    sim, orc = _pair(f, cfg)
    for _ in range(5):
        sim.step_single_nose_hoover(nsteps=20)
        orc.step_nose_hoover(20)
        assert rel_err(sim.xi, orc.xi) < 1e-5 or abs(sim.xi - orc.xi) < 1e-8
        assert rel_err(sim.cal_total_K(), orc.total_K()) < 1e-6
    dx, _ = _maxdx(sim, orc, np.array([Lx, Ly]))
    assert dx < 1e-6


def test_nph_barostat(built):
    f, Lx, Ly = wl.lattice_frame(2048, 0.8, 1.0, 0.65, 1.0, seed=31)
    cfg = wl.config_dict(2048, Lx, Ly, dt=0.001, T=1.0, barostat_mass=10.0)
    sim, orc = _pair(f, cfg)
    p0 = sim.cal_instant_pressure()
    assert rel_err(p0, orc.instant_pressure()) < 1e-6
    for _ in range(5):
        sim.step_single_NPH(1.0, nsteps=20)
        orc.step_nph(1.0, 20)
        o = sim.observables()
        assert rel_err(o.Lx, orc.s.Lx) < 1e-9
        assert rel_err(o.Ly, orc.s.Ly) < 1e-9
        assert abs(o.nph_area_momentum - orc.s.nph_area_momentum) < 1e-6 * (1 + abs(orc.s.nph_area_momentum))
        assert rel_err(o.last_instant_pressure, orc.s.last_instant_pressure) < 1e-5
    assert sim.get_Lx() != Lx  # the box moved


def test_nph_clamp(built):
    """A strong external pressure drives Ly to the lower clamp; p_A is then
    zeroed when it keeps pushing inward (src/md_env.cu:1907-1914)."""
    f, Lx, Ly = wl.lattice_frame(512, 0.8, 1.0, 0.65, 1.0, seed=32)
    cfg = wl.config_dict(512, Lx, Ly, dt=0.001, T=1.0, barostat_mass=0.05,
                         barostat_height_min_ratio=0.97)
    sim, orc = _pair(f, cfg)
    sim.step_single_NPH(3000.0, nsteps=60)
    orc.step_nph(3000.0, 60)
    o = sim.observables()
    assert abs(orc.s.Ly - 0.97 * Ly) < 1e-12 * Ly  # the oracle sits on the clamp
    assert rel_err(o.Ly, orc.s.Ly) < 1e-12
    assert o.nph_area_momentum == 0.0 and orc.s.nph_area_momentum == 0.0


def test_piston_walls(built):
    """step_single_NPH_piston on the reference's piston test geometry
    (N=512, 80x20, eps_AB=0.25), started from the reference-style lattice."""
    mgr = mdb.MDConfigManager()
    c = mgr.config
    for k, v in dict(n_particles_global=512, n_particles_type0=256, box_w_global=80.0,
                     box_h_global=20.0, T_init=0.9, T_target=0.9, EPSILON_AB=0.25, dt=0.001,
                     barostat_mass=10000.0, k_piston=100.0, rank_size=1).items():
        setattr(c, k, v)
    sim = mdb.MDSimulation(mgr)
    sim.sample_collect()
    f = sim.get_host_particles()
    cfgd = {k: getattr(c, k) for k in ("SIGMA_AA", "SIGMA_BB", "SIGMA_AB", "EPSILON_AA",
                                        "EPSILON_BB", "EPSILON_AB", "MASS_A", "MASS_B", "cutoff",
                                        "dt", "Q", "T_target", "n_particles_global",
                                        "barostat_mass", "k_piston", "box_w_global",
                                        "box_h_global")}
    orc = po.Sim(cfgd, f["pos"], f["vel"], f["type"], mode=po.OR_FP64)
    for _ in range(4):
        sim.step_single_NPH_piston(0.5, nsteps=25)
        orc.step_nph_piston(0.5, 25)
        o = sim.observables()
        assert rel_err(o.Ly, orc.s.Ly) < 1e-9
        assert abs(o.nph_piston_velocity - orc.s.piston_velocity) < 1e-7
        assert abs(o.nph_piston_force - orc.s.piston_force) < 1e-5 * (1 + abs(orc.s.piston_force))
    assert rel_err(sim.cal_total_U(), orc.total_U()) < 1e-6
    assert abs(sim.cal_instant_pressure() - orc.instant_pressure()) < 1e-6


def test_reference_lattice_init(built):
    """MDSimulation(cfg) without a file: two lattices, K = (2N-2) T_init / 2,
    zero net momentum (src/md_env.cu:1276-1445)."""
    mgr = mdb.MDConfigManager()
    c = mgr.config
    for k, v in dict(n_particles_global=2048, n_particles_type0=1024, box_w_global=143.10835056,
                     box_h_global=23.85139176, T_init=0.9, T_target=0.9, rank_size=1).items():
        setattr(c, k, v)
    sim = mdb.MDSimulation(mgr)
    sim.sample_collect()
    f = sim.get_host_particles()
    assert (f["type"] == 0).sum() == 1024
    K = sim.cal_total_K()
    assert abs(K - (2 * 2048 - 2) * 0.5 * 0.9) < 1e-9 * K
    assert np.abs(f["vel"].sum(axis=0)).max() < 1e-9
    a = f[f["type"] == 0]["pos"][:, 0]
    # type 0 occupies the central band of width devide_p * Lx
    assert a.min() > 0.25 * 143.10835056 - 1.0 and a.max() < 0.75 * 143.10835056 + 1.0


def test_mode_switches_and_frames(built, tmp_path):
    f, Lx, Ly = wl.lattice_frame(1024, 0.8, 1.0, 0.65, 1.0, seed=41)
    cfg = wl.config_dict(1024, Lx, Ly, dt=0.001, T=1.0, barostat_mass=10.0)
    sim, orc = _pair(f, cfg)
    sim.step_single_NVE(nsteps=5)
    orc.step_nve(5)
    sim.step_single_nose_hoover(nsteps=5)
    orc.step_nose_hoover(5)
    sim.step_single_NPH(1.0, nsteps=5)
    orc.step_nph(1.0, 5)
    sim.step_single_NPH_piston(1.0, nsteps=5)
    orc.step_nph_piston(1.0, 5)
    sim.step_single_NVE(nsteps=5)
    orc.step_nve(5)
    o = sim.observables()
    assert rel_err(o.Ly, orc.s.Ly) < 1e-9
    dx, g = _maxdx(sim, orc, np.array([o.Lx, o.Ly]))
    assert dx < 1e-7
    # save_env / constructor from file
    path = str(tmp_path / "traj.bin")
    sim.save_env(path, 25)
    sim.save_env(path, 26)
    sim2 = mdb.MDSimulation(cfg, None, path, 26)
    sim2.sample_collect()
    assert np.array_equal(sim2.get_host_particles()["pos"], g["pos"])
    assert mdb.FileReader(path).n_frames == 2


def test_rebuild_stress(built):
    """Hot, dilute system with a small skin: many cell-list rebuilds, results
    still match the oracle."""
    f, Lx, Ly = wl.lattice_frame(1500, 0.4, 1.0, 0.5, 3.0, seed=51)
    cfg = wl.config_dict(1500, Lx, Ly, dt=0.004, T=3.0)
    sim, orc = _pair(f, cfg, skin=0.05)
    sim.step_single_NVE(nsteps=200)
    orc.step_nve(200)
    o = sim.observables()
    assert o.rebuilds > 10
    assert rel_err(sim.cal_total_U(), orc.total_U()) < 1e-5


def test_observables_async_matches_sync(built):
    """mdb_sim_observables_async delivers, per step and without waiting, the
    record mdb_sim_observables returns."""
    import ctypes

    import torch

    from md_simulation_cuda_b200 import _lib

    f, cfg = wl.nve_4096(seed=6)
    sim = mdb.MDSimulation(cfg, frame=f)
    size = ctypes.sizeof(_lib.MDBObservables)
    ring = torch.zeros(5 * size, dtype=torch.uint8, pin_memory=True)
    sync = []
    for k in range(5):
        sim.step_single_nose_hoover(nsteps=3)
        sim.observables_async(ring.data_ptr() + k * size)
    sim.synchronize()
    ref = mdb.MDSimulation(cfg, frame=f)
    for k in range(5):
        ref.step_single_nose_hoover(nsteps=3)
        sync.append(ref.observables())
    for k in range(5):
        a = _lib.MDBObservables.from_address(ring.data_ptr() + k * size)
        b = sync[k]
        assert (a.t, a.Lx, a.Ly, a.xi, a.n, a.steps) == (b.t, b.Lx, b.Ly, b.xi, b.n, b.steps)
