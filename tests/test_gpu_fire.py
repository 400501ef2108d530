"""FIRE minimiser parity (EnergyMinimizer::minimize_frame) and batching."""
import numpy as np
import pytest

import md_simulation_cuda_b200 as mdb
from md_simulation_cuda_b200 import workloads as wl
from oracle import pyoracle as po
from tests.helpers import min_image, rel_err

pytestmark = pytest.mark.gpu


def _mgr(**kw):
    m = mdb.MDConfigManager()
    for k, v in kw.items():
        setattr(m.config, k, v)
    return m


def test_two_particle_smoke(built):
    """The reference's RUN_MINIMIZER_SMOKE case (tests/run_test/run_test.cpp:
    107-148): 2 particles at (1,1), (3,1), box 10x10, tol 1e-3, 200 steps."""
    mgr = _mgr(box_w_global=10.0, box_h_global=10.0, dt=1e-3, cutoff=2.5, SIGMA_BB=1.0,
               SIGMA_AB=1.0, EPSILON_AB=1.0, n_particles_global=2, n_local=2, n_cap=16,
               THREADS_PER_BLOCK=128, rank_size=1)
    f = mdb.make_frame(2)
    f["pos"] = [[1.0, 1.0], [3.0, 1.0]]
    params = mdb.FireParams.from_config(mgr)
    res = mdb.EnergyMinimizer(mgr).minimize_frame(f, 1e-3, 200, params)
    cfgd = dict(SIGMA_AA=1.0, SIGMA_BB=1.0, SIGMA_AB=1.0, EPSILON_AA=1.0, EPSILON_BB=1.0,
                EPSILON_AB=1.0, MASS_A=1.0, MASS_B=1.0, cutoff=2.5)
    ref = po.fire_minimize(cfgd, f["pos"], f["type"], 10.0, 10.0, 1e-3, 200,
                           dict(dt_init=1e-3, dt_max=5e-3, alpha0=0.1, f_inc=1.1, f_dec=0.5,
                                N_min=5), mode=po.OR_FP64)
    assert res.steps == ref["steps"] and res.converged == ref["converged"]
    assert rel_err(res.max_force, ref["max_force"]) < 1e-5
    assert np.abs(res.frame["pos"] - ref["pos"]).max() < 1e-7
    assert res.energy_steps == ref["energy_steps"]


def test_minimizer_errors(built):
    mgr = _mgr(box_w_global=10.0, box_h_global=10.0, n_cap=0)
    with pytest.raises(RuntimeError):
        mdb.EnergyMinimizer(mgr)
    mgr.config.n_cap = 1
    em = mdb.EnergyMinimizer(mgr)
    with pytest.raises(RuntimeError):
        em.minimize_frame(mdb.make_frame(2), 1e-3, 10, mdb.FireParams.from_config(mgr))
    with pytest.raises(RuntimeError):
        em.minimize_frame(mdb.make_frame(1), 1e-3, 0, mdb.FireParams.from_config(mgr))


def _hex_crystal(nx, ny, a, jitter, seed):
    """Triangular lattice (the 2D LJ ground state) with uniform jitter."""
    rng = np.random.default_rng(seed)
    Lx, Ly = nx * a, ny * a * np.sqrt(3) / 2
    i, j = np.meshgrid(np.arange(nx), np.arange(ny), indexing="xy")
    x = (i + 0.5 * (j % 2) + 0.25) * a
    y = (j + 0.5) * a * np.sqrt(3) / 2
    f = mdb.make_frame(nx * ny)
    f["pos"] = np.stack([x.ravel(), y.ravel()], 1) + rng.uniform(-jitter, jitter, (nx * ny, 2))
    return f, Lx, Ly


def _mgr_from(cfgd, n_cap):
    mgr = mdb.MDConfigManager(mdb._lib.MDBConfigC())
    for k, v in cfgd.items():
        setattr(mgr.config, k, v)
    mgr.config.n_cap = n_cap
    return mgr


FIRE_P = dict(dt_init=0.001, dt_max=0.01, alpha0=0.1, f_inc=1.1, f_dec=0.5, N_min=5)


def test_fire_crystal_quench_vs_oracle(built):
    """A jittered triangular crystal relaxes to the unique nearby minimum:
    final energy and positions agree with the FP64 oracle, and the CUDA path
    reaches max|F| < 1e-5 (where the reference's FP32 arithmetic stalls)."""
    f, Lx, Ly = _hex_crystal(20, 24, 1.12, 0.05, seed=62)
    cfgd = wl.config_dict(len(f), Lx, Ly, dt=0.001)
    res = mdb.EnergyMinimizer(_mgr_from(cfgd, 1000)).minimize_frame(
        f, 1e-5, 20000, mdb.FireParams(dt_init=0.001, dt_max=0.01))
    ref = po.fire_minimize(cfgd, f["pos"], f["type"], Lx, Ly, 1e-5, 20000, FIRE_P,
                           mode=po.OR_FP64)
    assert ref["converged"]
    assert res.converged, res.max_force
    # FP32 pair energies carry ~1e-7 relative noise (as the reference's do)
    assert rel_err(res.potential_energy, ref["potential_energy"]) < 1e-7
    _, U_at_gpu, _ = po.forces(cfgd, res.frame["pos"], res.frame["type"], Lx, Ly)
    assert rel_err(res.potential_energy, U_at_gpu) < 1e-7
    d = min_image(res.frame["pos"] - ref["pos"], np.array([Lx, Ly]))
    assert np.abs(d - d.mean(0)).max() < 1e-4


def test_fire_short_horizon_vs_oracle(built):
    """Before chaos separates FIRE paths, iterate-by-iterate agreement."""
    f, Lx, Ly = wl.lattice_frame(400, 0.9, 1.0, 0.6, 0.0, seed=61, jitter=0.2)
    cfgd = wl.config_dict(400, Lx, Ly, dt=0.001)
    res = mdb.EnergyMinimizer(_mgr_from(cfgd, 1000)).minimize_frame(
        f, 1e-6, 60, mdb.FireParams(dt_init=0.001, dt_max=0.01))
    ref = po.fire_minimize(cfgd, f["pos"], f["type"], Lx, Ly, 1e-6, 60, FIRE_P, mode=po.OR_FP64)
    assert res.steps == ref["steps"] == 60
    d = min_image(res.frame["pos"] - ref["pos"], np.array([Lx, Ly]))
    assert np.abs(d).max() < 5e-6
    assert rel_err(res.potential_energy, ref["potential_energy"]) < 1e-6
    assert res.energy_steps == ref["energy_steps"]


def test_batch_equals_solo(built):
    """Each system of a batch gives bit-identical results to running it alone
    (per-system cell rebuilds, reductions and FIRE control)."""
    systems = wl.fire_mix(6, seed=9, n_min=64, n_max=900)
    params = mdb.FireParams(dt_init=0.001, dt_max=0.01)
    b = mdb.Batch()
    for f, cfgd in systems:
        b.add_fire(cfgd, f, 1e-6, 400, params)
    b.run()
    n, done = b.progress()
    assert n == 6 and done == 6
    for k, (f, cfgd) in enumerate(systems):
        mgr = mdb.MDConfigManager(mdb._lib.MDBConfigC())
        for kk, v in cfgd.items():
            setattr(mgr.config, kk, v)
        mgr.config.n_cap = len(f)
        solo = mdb.EnergyMinimizer(mgr).minimize_frame(f, 1e-6, 400, params)
        rb = b.fire_result(k)
        # bit-identical, NaN included (FP32 overflow at r < 0.0023 sigma in a
        # random start makes a system non-finite, as in the reference)
        assert rb.steps == solo.steps and rb.converged == solo.converged
        assert np.array_equal([rb.max_force], [solo.max_force], equal_nan=True)
        assert np.array_equal(rb.frame["pos"], solo.frame["pos"], equal_nan=True)
        assert np.array_equal(rb.energy_trace, solo.energy_trace, equal_nan=True)
        assert rb.nonfinite == solo.nonfinite
        # every system was binned at build and rebuilt on its own schedule after
        rebuilds, overflow = b.system_stats(k)
        assert 1 <= rebuilds <= rb.steps + 1 and overflow >= 0


def test_fire_reaches_1e6_from_random_starts(built):
    """Random starts as in the 512-system mix (uniform positions, 20,000
    iteration cap, tolerance 1e-6). FP32 pair terms (the reference's
    arithmetic, fire_precision=FIRE_FP32) leave a noise floor near 1e-5 in
    max|a|, so those runs stall at the cap; with the automatic switch to FP64
    pair terms below max|a| = 1e-3 the GPU converges about as often as the
    FP64 oracle. FIRE from a random start is chaotic, so the GPU and oracle
    runs reach different minima after different iteration counts; each GPU
    result is checked to be a minimum by the oracle's own FP64 forces, with
    the energy the oracle gives that frame."""
    systems = wl.fire_mix(8, seed=7, n_min=256, n_max=1024)
    params = mdb.FireParams(dt_init=0.001, dt_max=0.01)
    runs = {}
    for prec in (mdb.FIRE_AUTO, mdb.FIRE_FP32):
        b = mdb.Batch(fire_precision=prec)
        for f, cfgd in systems:
            b.add_fire(cfgd, f, 1e-6, 20000, params)
        b.run()
        runs[prec] = [b.fire_result(k) for k in range(len(systems))]
    n_ref = 0
    for f, cfgd in systems:
        L = cfgd["box_w_global"]
        ref = po.fire_minimize(cfgd, f["pos"], f["type"], L, L, 1e-6, 20000, FIRE_P,
                               mode=po.OR_FP64)
        n_ref += int(ref["converged"])
    n_auto = 0
    for (f, cfgd), res in zip(systems, runs[mdb.FIRE_AUTO]):
        L = cfgd["box_w_global"]
        assert not res.nonfinite
        if not res.converged:
            continue
        n_auto += 1
        assert res.max_force < 1e-6 and res.steps < 20000
        acc, U, _ = po.forces(cfgd, res.frame["pos"], res.frame["type"], L, L, cells=True)
        assert np.abs(acc).max() < 2e-6
        assert rel_err(res.potential_energy, U) < 1e-9
    n_fp32 = sum(int(r.converged) for r in runs[mdb.FIRE_FP32])
    assert n_ref >= 6
    assert n_auto >= max(5, int(0.7 * n_ref))
    assert n_fp32 <= 1 < n_auto


def test_fire_fp32_mode_is_the_reference_arithmetic(built):
    """fire_precision=FIRE_FP32 keeps FP32 pair terms throughout: the same
    iterates as the automatic mode until the switch point (max|a| > 1e-3
    here, 60 iterations from a jittered lattice)."""
    f, Lx, Ly = wl.lattice_frame(400, 0.9, 1.0, 0.6, 0.0, seed=61, jitter=0.2)
    cfgd = wl.config_dict(400, Lx, Ly, dt=0.001)
    p = mdb.FireParams(dt_init=0.001, dt_max=0.01)
    a = mdb.EnergyMinimizer(_mgr_from(cfgd, 1000)).minimize_frame(f, 1e-6, 60, p)
    b = mdb.EnergyMinimizer(_mgr_from(cfgd, 1000),
                            fire_precision=mdb.FIRE_FP32).minimize_frame(f, 1e-6, 60, p)
    assert a.max_force > 1e-3
    assert np.array_equal(a.frame["pos"], b.frame["pos"])


def test_fire_crystal_fp64_matches_oracle_to_1e9(built):
    """A jittered crystal quench has one nearby minimum: with FP64 pair terms
    from the first iteration (FIRE_FP64) the GPU's energy and positions agree
    with the FP64 oracle's at max|a| < 1e-6."""
    f, Lx, Ly = _hex_crystal(20, 24, 1.12, 0.05, seed=62)
    cfgd = wl.config_dict(len(f), Lx, Ly, dt=0.001)
    em = mdb.EnergyMinimizer(_mgr_from(cfgd, 1000), fire_precision=mdb.FIRE_FP64)
    res = em.minimize_frame(f, 1e-6, 20000, mdb.FireParams(dt_init=0.001, dt_max=0.01))
    ref = po.fire_minimize(cfgd, f["pos"], f["type"], Lx, Ly, 1e-6, 20000, FIRE_P,
                           mode=po.OR_FP64)
    assert ref["converged"] and res.converged
    assert rel_err(res.potential_energy, ref["potential_energy"]) < 1e-9
    d = min_image(res.frame["pos"] - ref["pos"], np.array([Lx, Ly]))
    assert np.abs(d - d.mean(0)).max() < 1e-5


def test_fire_close_pair_stays_finite(built):
    """A pair 0.001 sigma apart (random starts have such pairs): the FP32 pair
    term would overflow to inf/NaN, as the reference's does; here it is
    taken at r^2 = 1e-5 sigma^2 and the quench stays finite."""
    f, L = wl.random_frame(200, 0.8, 0.5, 11)
    f["pos"][1] = f["pos"][0] + np.array([0.001, 0.0])
    f["type"][0] = f["type"][1] = 0
    cfgd = wl.config_dict(len(f), L, L, dt=0.001)
    res = mdb.EnergyMinimizer(_mgr_from(cfgd, 1000)).minimize_frame(
        f, 1e-6, 1, mdb.FireParams(dt_init=0.001, dt_max=0.01))
    assert not res.nonfinite
    assert np.isfinite(res.frame["acc"]).all() and np.isfinite(res.energy_trace).all()
    # the pair's own term at the floor, in FP64 (the FP32 value is within 1e-6)
    r2 = 1e-5
    sr2 = 1.0 / r2
    tmp = 24.0 * (2.0 * sr2 ** 6 - sr2 ** 3) / r2
    assert abs(res.frame["acc"][0, 0] / (tmp * 0.001) + 1.0) < 1e-4


def _wrap_ref(x, L):
    """pbc_wrap_hd (include/md_cuda_common.hpp:20-29) in host arithmetic:
    C fmod is exact, then + L for a negative remainder."""
    import math

    if 0.0 <= x < L:
        return x
    if L <= x < 2.0 * L:
        return x - L
    if -L <= x < 0.0:
        return x + L
    r = math.fmod(x, L)
    return r + L if r < 0.0 else r


def test_fire_entry_wraps_far_positions_exactly(built):
    """The FIRE entry wraps every position into the box; positions many box
    lengths out (a random start's overlapping pair can throw a particle
    2^90 box lengths in one step) wrap bit for bit as the host's exact fmod
    does."""
    rng = np.random.default_rng(11)
    n = 64
    L = 9.87654321
    f = mdb.make_frame(n)
    far = [1e25, -3.7e18, 5.5 * L + 1e-9, -1e300, 2.0 ** 90 + 0.5, -(2.0 ** 60) * L,
           7.0 * L, -7.0 * L, 1e-300, 3e8 * L + 0.25, -1.5 * L, 1.999 * L]
    xs = np.concatenate([far, rng.uniform(-1e40, 1e40, n - len(far))])
    ys = rng.uniform(-1e12, 1e12, n)
    f["pos"][:, 0] = xs
    f["pos"][:, 1] = ys
    f["type"] = rng.integers(0, 2, n)
    cfgd = wl.config_dict(n, L, L, dt=0.001)
    mgr = mdb.MDConfigManager(mdb._lib.MDBConfigC())
    for k, v in cfgd.items():
        setattr(mgr.config, k, v)
    mgr.config.n_cap = n
    res = mdb.EnergyMinimizer(mgr).minimize_frame(f, 1e300, 1,
                                               mdb.FireParams(dt_init=0.001, dt_max=0.01))
    got = res.frame["pos"]
    want = np.array([[_wrap_ref(float(x), L), _wrap_ref(float(y), L)] for x, y in zip(xs, ys)])
    assert np.array_equal(got, want)
