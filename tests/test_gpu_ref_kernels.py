"""The product against the reference's own CUDA kernels, run on the same GPU.

oracle/_ref/libref_kernels.so is the reference's unmodified
src/md_cuda_common.cu with its host step logic restated at world size 1
(oracle/ref_kernels.cu). These tests run it beside libmdb200.so:

* the oracle's reference-arithmetic mode reproduces the reference kernels bit
  for bit at the configurations' sizes (live, beyond the committed fixtures);
* the product's forces are within the accuracy bound (relative L2 1e-5) of
  the reference kernel's and closer than them to the FP64 truth;
* energies, pressure and dU/dlambda agree; the NVE, Nose-Hoover, NPH and
  piston steps track the reference's steps.
"""
import numpy as np
import pytest

import md_simulation_cuda_b200 as mdb
from md_simulation_cuda_b200 import workloads as wl
from oracle import pyoracle as po
from oracle import refkernels as rk
from tests.helpers import min_image, rel_err, rel_l2

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5


def _bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return np.array_equal(a.view(np.int64), b.view(np.int64))


def _ref(cfg, f, **kw):
    return rk.RefSim(cfg, f, **kw)


def test_reference_kernels_equal_oracle_at_4096(built):
    """li_force_kernel, U, pressure and K at N = 4096 (the NVE configuration)
    equal the oracle's restatement bit for bit, with and without the
    world-size-1 self-halo."""
    f, cfg = wl.nve_4096()
    L = cfg["box_w_global"]
    for ws1 in (0, 1):
        r = _ref(cfg, f, ws1_halo=bool(ws1))
        acc, _, _ = po.forces(cfg, f["pos"], f["type"], L, L, mode=po.OR_REF_MIXED,
                              ws1_halo=ws1)
        assert _bits_equal(r.frame()["acc"], acc)
        for what, fn in ((po.OR_SUM_U, r.total_U), (po.OR_SUM_P, r.pressure_sum),
                         (po.OR_SUM_K, r.total_K)):
            tot_ref, part_ref = fn()
            v = po.ref_thread_values(cfg, f["pos"], f["vel"], f["type"], L, L, what,
                                     ws1_halo=ws1)
            tot, part = po.ref_block_partials(v, 256)
            assert _bits_equal(part, part_ref) and _bits_equal([tot], [tot_ref])
        r.close()


def test_product_forces_vs_reference_kernel(built):
    """At N = 4096 and on a dense random start: the product is within 1e-5 of
    the reference kernel's forces and closer than them to the FP64 truth."""
    cases = [wl.nve_4096(seed=5)]
    fr, L = wl.random_frame(3000, 0.9, 0.5, 17)
    fr["pos"] = np.array(fr["pos"])
    cases.append((fr, wl.config_dict(3000, L, L, dt=0.001)))
    for f, cfg in cases:
        Lx, Ly = cfg["box_w_global"], cfg["box_h_global"]
        r = _ref(cfg, f)
        ref_acc = r.frame()["acc"]
        r.close()
        acc, _, _ = mdb.compute_forces(cfg, f, Lx, Ly)
        truth, _, _ = po.forces(cfg, f["pos"], f["type"], Lx, Ly, mode=po.OR_FP64, cells=True)
        mask = np.isfinite(ref_acc).all(1)  # a random start can overflow the reference
        assert rel_l2(acc[mask], ref_acc[mask]) <= FORCE_TOL
        assert rel_l2(acc, truth) <= rel_l2(ref_acc[mask], truth[mask]) * 1.0001


def test_product_observables_vs_reference_kernels(built):
    """cal_total_U, the scalar pressure and cal_partial_U_lambda of the
    product against the reference's kernels (FP32 pair terms on both sides,
    summed in different orders): relative 1e-6."""
    f, cfg = wl.nve_4096(seed=3)
    L = cfg["box_w_global"]
    r = _ref(cfg, f)
    U_ref, _ = r.total_U()
    Psum_ref, _ = r.pressure_sum()
    dudl_ref, _ = r.partial_U_lambda(0.7)
    r.close()
    sim = mdb.MDSimulation(cfg, frame=f)
    assert rel_err(sim.cal_total_U(), U_ref) < 1e-6
    # the pressure is a difference of the kinetic and virial terms (about 3x
    # cancellation); the reference's FP32 cast of the unwrapped displacement
    # costs its periodic pairs ~1e-6 each, so both are held to the FP64 truth
    P_ref = Psum_ref / (2 * L * L)
    orc = po.Sim(cfg, f["pos"], f["vel"], f["type"], mode=po.OR_FP64)
    P64 = orc.instant_pressure()
    P = sim.cal_instant_pressure()
    assert rel_err(P, P_ref) < 2e-5
    assert abs(P - P64) <= abs(P_ref - P64) + 1e-7 * abs(P64)
    assert rel_err(sim.cal_partial_U_lambda(0.7), dudl_ref) < 1e-5


def test_nve_1000_steps_vs_reference_kernels(built):
    """The NVE configuration (N = 4096, dt = 0.001, 1000 steps) through the
    product and through the reference's own kernels: K and U agree at every
    100th step (relative 1e-5), and the energy drift of each is small. The
    drifts against the FP64 oracle's are printed for the record."""
    f, cfg = wl.nve_4096()
    r = _ref(cfg, f)
    K_ref, U_ref = r.step(rk.KIND_NVE, 1000, trace=True)
    g_ref = r.frame()
    r.close()
    sim = mdb.MDSimulation(cfg, frame=f)
    E0 = sim.cal_total_K() + sim.cal_total_U()
    for block in range(10):
        sim.step_single_NVE(nsteps=100)
        k = 100 * block + 99
        assert rel_err(sim.cal_total_K(), K_ref[k]) < 1e-5
        assert rel_err(sim.cal_total_U(), U_ref[k]) < 1e-5
    E1 = sim.cal_total_K() + sim.cal_total_U()
    orc = po.Sim(cfg, f["pos"], f["vel"], f["type"], mode=po.OR_FP64)
    E0o = orc.total_K() + orc.total_U()
    orc.step_nve(1000)
    E1o = orc.total_K() + orc.total_U()
    r0 = _ref(cfg, f)
    E0r = r0.total_K()[0] + r0.total_U()[0]
    r0.close()
    E1r = K_ref[-1] + U_ref[-1]
    drift = {"product": (E1 - E0) / abs(E0), "reference": (E1r - E0r) / abs(E0r),
             "fp64_oracle": (E1o - E0o) / abs(E0o)}
    print("NVE 1000-step relative energy drift:", drift)
    assert abs(drift["product"]) < 2e-4 and abs(drift["reference"]) < 2e-4
    assert abs(drift["product"] - drift["fp64_oracle"]) < 2e-5
    # no further from the FP64 drift than the reference's own build (measured:
    # product -3.120e-5, reference -3.115e-5, FP64 oracle -3.123e-5)
    assert (abs(drift["product"] - drift["fp64_oracle"])
            <= abs(drift["reference"] - drift["fp64_oracle"]) + 1e-7)
    sim.sample_collect()
    g = sim.get_host_particles()
    # chaos amplifies the FP32 differences over 1000 steps; still well inside a cell
    L = np.array([cfg["box_w_global"], cfg["box_h_global"]])
    assert np.abs(min_image(g["pos"] - g_ref["pos"], L)).max() < 1e-2


def test_nose_hoover_vs_reference_kernels(built):
    f, Lx, Ly = wl.lattice_frame(4096, 0.8, 2.0, lambda s: np.where(s < 0.5, 0.9, 0.1), 0.7,
                                 seed=21)
    cfg = wl.config_dict(4096, Lx, Ly, dt=0.002, T=0.7, Q=1.0)
    r = _ref(cfg, f)
    sim = mdb.MDSimulation(cfg, frame=f)
    for _ in range(4):
        r.step(rk.KIND_NH, 25)
        sim.step_single_nose_hoover(nsteps=25)
        st = r.state()
        # xi integrates (2K - g T)/Q with g = 8190: 1e-7 relative differences
        # of K (FP32 pair terms summed in different orders) add up in xi
        assert abs(sim.xi - st["xi"]) < 1e-5 * (1 + abs(st["xi"]))
        assert rel_err(sim.cal_total_K(), r.total_K()[0]) < 1e-6
    sim.sample_collect()
    g = sim.get_host_particles()
    assert np.abs(min_image(g["pos"] - r.frame()["pos"], np.array([Lx, Ly]))).max() < 1e-5
    r.close()


def test_nph_vs_reference_kernels(built):
    f, Lx, Ly = wl.lattice_frame(2048, 0.8, 1.0, 0.65, 1.0, seed=31)
    cfg = wl.config_dict(2048, Lx, Ly, dt=0.001, T=1.0, barostat_mass=10.0)
    r = _ref(cfg, f)
    sim = mdb.MDSimulation(cfg, frame=f)
    for _ in range(4):
        r.step(rk.KIND_NPH, 25, p_ext=1.0)
        sim.step_single_NPH(1.0, nsteps=25)
        st = r.state()
        o = sim.observables()
        assert rel_err(o.Lx, st["Lx"]) < 1e-9 and rel_err(o.Ly, st["Ly"]) < 1e-9
        assert rel_err(o.last_instant_pressure, st["last_P"]) < 1e-5
    r.close()


def test_piston_vs_reference_kernels(built):
    f, Lx, Ly = wl.lattice_frame(1024, 0.32, 4.0, 0.5, 0.9, seed=35)
    f["pos"][:4, 1] = [-0.05, -0.3, Ly + 0.02, Ly + 0.4]
    cfg = wl.config_dict(1024, Lx, Ly, dt=0.001, T=0.9, barostat_mass=10.0, k_piston=100.0)
    r = _ref(cfg, f)
    sim = mdb.MDSimulation(cfg, frame=f)
    for _ in range(4):
        r.step(rk.KIND_PISTON, 25, p_ext=0.5)
        sim.step_single_NPH_piston(0.5, nsteps=25)
        st = r.state()
        o = sim.observables()
        assert rel_err(o.Ly, st["Ly"]) < 1e-9
        assert abs(o.nph_piston_velocity - st["piston_velocity"]) < 1e-7
        assert rel_err(o.nph_piston_force, st["piston_force"]) < 1e-5
    r.close()
