"""The CPU oracle pinned against outputs of the reference's own CUDA kernels.

tests/golden/ref_physics.{npz,json} hold what the reference's unmodified
src/md_cuda_common.cu computed on a GPU (li_force_kernel, cal_local_U_kernel,
cal_local_pressure_scalar_kernel, cal_local_K_kernel,
cal_partial_U_lambda_kernel, piston_wall_kernel, the seven integrator kernels
and whole NVE / Nose-Hoover / NPH / piston steps driven by the reference's
host step logic at world size 1), recorded by tests/golden/make_ref_physics.py.
The oracle's reference-arithmetic mode (OR_REF_MIXED, all pairs, the
reference's block-tree sums) must reproduce every one of them bit for bit,
with and without the world-size-1 self-halo. No GPU is needed here.
"""
import json
import os

import numpy as np
import pytest

from oracle import pyoracle as po

HERE = os.path.dirname(os.path.abspath(__file__))
Z = np.load(os.path.join(HERE, "golden", "ref_physics.npz"))
M = json.load(open(os.path.join(HERE, "golden", "ref_physics.json")))
EPS_LAMBDA = 0.7
STATIC = ["lat512", "slab512", "dense256", "edge64", "piston512"]
TRAJ = ["nve_lat512", "nve_lat512_ws1", "nh_slab512", "nph_lat512", "piston_traj512"]


def bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.int64), b.view(np.int64))


def _frame(name):
    return Z[f"{name}/frame_pos"], Z[f"{name}/frame_vel"], Z[f"{name}/frame_type"]


def _threads(name):
    return [int(k.split("_t")[1]) for k in M[name] if k.startswith("ws0_t")]


@pytest.mark.parametrize("name", STATIC)
@pytest.mark.parametrize("ws1", [0, 1])
def test_forces_bit_exact(built, name, ws1):
    m = M[name]
    pos, _, typ = _frame(name)
    for th in _threads(name):
        acc, _, _ = po.forces(m["cfg"], pos, typ, m["Lx"], m["Ly"], periodic_y=m["periodic_y"],
                              mode=po.OR_REF_MIXED, ws1_halo=ws1)
        assert bits_equal(acc, Z[f"{name}/ws{ws1}_t{th}/acc"])


@pytest.mark.parametrize("name", STATIC)
@pytest.mark.parametrize("ws1", [0, 1])
def test_block_sums_bit_exact(built, name, ws1):
    """U, pressure numerator, K and dU/dlambda: every block partial and the
    host's block-order total."""
    m = M[name]
    pos, vel, typ = _frame(name)
    for th in _threads(name):
        tag = f"ws{ws1}_t{th}"
        for what, key, tot_key in ((po.OR_SUM_U, "U", "U"), (po.OR_SUM_P, "P", "Psum"),
                                   (po.OR_SUM_K, "K", "K"), (po.OR_SUM_DUDL, "dUdl", "dUdl")):
            v = po.ref_thread_values(m["cfg"], pos, vel, typ, m["Lx"], m["Ly"], what,
                                     periodic_y=m["periodic_y"], ws1_halo=ws1,
                                     eps_lambda=EPS_LAMBDA)
            tot, part = po.ref_block_partials(v, th)
            assert bits_equal(part, Z[f"{name}/{tag}/{key}_partials"]), key
            if what == po.OR_SUM_U and not m["periodic_y"]:
                continue  # the reference adds the wall energy to this total
            assert bits_equal([tot], [m[tag][tot_key]]), key


def test_piston_walls_bit_exact(built):
    """The piston geometry (walled y, particles above Ly and below 0): LJ
    forces without the y image, U with the wall energy, and piston_wall_kernel
    with the acceleration update, its upper-wall force and wall energy."""
    m = M["piston512"]
    pos, vel, typ = _frame("piston512")
    sim = po.Sim(m["cfg"], pos, vel, typ, mode=po.OR_REF_MIXED, use_cells=False,
                 ref_threads=256)
    sim.cal_forces(periodic_y=0)
    assert bits_equal(sim.acc, Z["piston512/ws0_t256/acc"])
    sim.s.piston_mode_active = 1
    assert bits_equal([sim.total_U()], [m["ws0_t256"]["U"]])
    up, en = sim.piston_walls(update_acc=True)
    assert bits_equal(sim.acc, Z["piston512/wall_acc"])
    assert bits_equal([up, en], [m["wall_upper"], m["wall_energy"]])


@pytest.mark.parametrize("key", ["half_vv", "second_half_vv", "half_vv_nh", "second_half_vv_nh",
                                 "half_nph_vel", "nph_scale_drift", "half_vv_piston"])
def test_integrator_kernels_bit_exact(built, key):
    which = dict(half_vv=0, second_half_vv=1, half_vv_nh=2, second_half_vv_nh=3, half_nph_vel=4,
                 nph_scale_drift=5, half_vv_piston=6)[key]
    mi = M["integ256"]
    kw = dict(mi["calls"][key])
    Lx = kw.pop("Lx_new", mi["L"])
    Ly = kw.pop("Ly_new", mi["L"])
    p, v = po.ref_integrator(which, Z["integ256/frame_pos"], Z["integ256/frame_vel"],
                             Z["integ256/frame_acc"], Lx=Lx, Ly=Ly, **kw)
    assert bits_equal(p, Z[f"integ256/{key}/pos"])
    assert bits_equal(v, Z[f"integ256/{key}/vel"])


@pytest.mark.parametrize("name", TRAJ)
def test_trajectories_bit_exact(built, name):
    """Whole steps (the constructor's force evaluation, then nsteps steps),
    with cal_total_K / cal_total_U after every step."""
    m = M[name]
    pos, vel, typ = _frame(m["start"])
    sim = po.Sim(m["cfg"], pos, vel, typ, mode=po.OR_REF_MIXED, ws1_halo=m["ws1_halo"],
                 use_cells=False, ref_threads=256)
    K, U = [], []
    for _ in range(m["nsteps"]):
        if m["kind"] == 0:
            sim.step_nve()
        elif m["kind"] == 1:
            sim.step_nose_hoover()
        elif m["kind"] == 2:
            sim.step_nph(m["p_ext"])
        else:
            sim.step_nph_piston(m["p_ext"])
        K.append(sim.total_K())
        U.append(sim.total_U())
    assert bits_equal(sim.pos, Z[f"{name}/final_pos"])
    assert bits_equal(sim.vel, Z[f"{name}/final_vel"])
    assert bits_equal(sim.acc, Z[f"{name}/final_acc"])
    assert bits_equal(K, Z[f"{name}/K_trace"])
    assert bits_equal(U, Z[f"{name}/U_trace"])
    st = m["state"]
    for ref_key, key in (("xi", "xi"), ("Lx", "Lx"), ("Ly", "Ly"),
                         ("nph_area_momentum", "nph_area_momentum"),
                         ("piston_velocity", "piston_velocity"), ("piston_force", "piston_force"),
                         ("last_P", "last_instant_pressure"), ("t", "t")):
        assert bits_equal([getattr(sim.s, key)], [st[ref_key]]), ref_key


def test_reference_force_error_vs_fp64(built):
    """The reference's own arithmetic against the FP64 truth (the figure the
    product's 1e-5 bound is compared with): its FP32 cast of the FP64
    displacement costs it accuracy at the periodic edges."""
    errs = {}
    for name in ("lat512", "slab512", "dense256"):
        m = M[name]
        pos, _, typ = _frame(name)
        truth, _, _ = po.forces(m["cfg"], pos, typ, m["Lx"], m["Ly"], mode=po.OR_FP64)
        ref = Z[f"{name}/ws0_t256/acc"]
        errs[name] = float(np.linalg.norm(ref - truth) / np.linalg.norm(truth))
    assert all(e < 1e-5 for e in errs.values()), errs
