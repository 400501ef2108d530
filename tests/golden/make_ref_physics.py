"""Records the outputs of the reference's own CUDA kernels as golden fixtures.

The reference's src/md_cuda_common.cu (unmodified) is compiled with
oracle/ref_kernels.cu, a restatement of its host step logic at world size 1,
into oracle/_ref/libref_kernels.so by oracle/build_ref.py. This script runs
those kernels on a GPU on small seeded inputs and writes

  ref_physics.npz    inputs and outputs (arrays, float64 / int32)
  ref_physics.json   case parameters and scalar outputs

so that tests/test_ref_pinned.py can check the CPU oracle against the
reference's own arithmetic without a GPU. The inputs are this project's seeded
frames, stored in the fixture, so nothing is regenerated when checking.

Run on a machine with a GPU, from the repository root:
    python tests/golden/make_ref_physics.py [--out DIR]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from md_simulation_cuda_b200 import workloads as wl  # noqa: E402
from md_simulation_cuda_b200._lib import PARTICLE_DTYPE  # noqa: E402
from oracle import refkernels as rk  # noqa: E402

EPS_LAMBDA = 0.7


def min_pair_distance(pos, L):
    d = pos[:, None, :] - pos[None, :, :]
    d -= L * np.round(d / L)
    r2 = (d ** 2).sum(-1)
    np.fill_diagonal(r2, np.inf)
    return math.sqrt(r2.min())


def dense_frame(n, rho, seed):
    """Uniform random start (a FIRE quench's) whose closest pair is >= 0.15."""
    for s in range(seed, seed + 1000):
        f, L = wl.random_frame(n, rho, 0.5, s)
        if min_pair_distance(f["pos"], np.array([L, L])) >= 0.15:
            rng = np.random.default_rng(s)
            f["vel"] = rng.normal(0.0, 1.0, (n, 2))
            return f, L, s
    raise RuntimeError("no seed found")


def edge_frame(seed):
    """64 particles at the periodic edges and at the pair cutoff."""
    rng = np.random.default_rng(seed)
    L = 12.0
    pts = []
    for k in range(16):  # pairs straddling x = 0 / L
        y = 0.5 + 0.7 * k
        pts.append((1e-9 * (k + 1), y))
        pts.append((L - 0.9 - 0.05 * k, y + 0.01))
    for k in range(8):  # A-A pairs at r = rc (1 + (k - 3.5) 2e-8)
        x0, y0 = 3.0 + 0.2 * k, 6.0 + 0.6 * k
        r = 2.5 * (1.0 + (k - 3.5) * 2e-8)
        pts.append((x0, y0))
        pts.append((x0 + r, y0))
    k = 0
    while len(pts) < 64:  # along y = L (minus a hair), at least 0.3 from the rest
        k += 1
        p = (rng.uniform(0, L), L - 1e-10 * k)
        d = np.array(pts) - np.array(p)
        d -= L * np.round(d / L)
        if (d ** 2).sum(-1).min() >= 0.09:
            pts.append(p)
    pos = np.array(pts)
    f = np.zeros(len(pos), dtype=PARTICLE_DTYPE)
    f["pos"] = pos
    f["vel"] = rng.normal(0.0, 1.0, (len(pos), 2))
    f["type"] = np.where(np.arange(len(pos)) < 48, 0, 1)
    return f, L


def integ_frame(n, L, seed):
    rng = np.random.default_rng(seed)
    f = np.zeros(n, dtype=PARTICLE_DTYPE)
    f["pos"] = rng.uniform(-0.01 * L, 1.01 * L, (n, 2))
    f["pos"][:8, 0] = [0.0, -0.0, L, -1e-17, L - 1e-15, 2 * L + 0.25, -L - 0.25, 1e-300]
    f["vel"] = rng.normal(0.0, 1.0, (n, 2))
    f["acc"] = rng.normal(0.0, 10.0, (n, 2))
    f["type"] = (rng.random(n) < 0.4).astype(np.int32)
    return f


def cfg_of(n, Lx, Ly, **kw):
    c = wl.config_dict(n, Lx, Ly, dt=kw.pop("dt", 0.001), T=kw.pop("T", 1.0), Q=kw.pop("Q", 1.0))
    c.update(kw)
    return c


def record_static(name, cfg, frame, periodic_y, arrays, meta, threads=(256,)):
    """Forces, U, pressure, K, dU/dlambda (and walls) on one frame."""
    m = {"n": len(frame), "Lx": cfg["box_w_global"], "Ly": cfg["box_h_global"],
         "periodic_y": periodic_y, "cfg": cfg}
    arrays[f"{name}/frame_pos"] = frame["pos"].copy()
    arrays[f"{name}/frame_vel"] = frame["vel"].copy()
    arrays[f"{name}/frame_type"] = frame["type"].astype(np.int32)
    for ws1 in (0, 1):
        for th in threads:
            tag = f"{name}/ws{ws1}_t{th}"
            s = rk.RefSim(cfg, frame, ws1_halo=bool(ws1), threads=th, init_forces=False)
            s.cal_forces(periodic_y)
            arrays[f"{tag}/acc"] = s.frame()["acc"].copy()
            st = s.state()
            m[f"ws{ws1}_halo_counts"] = [st["n_halo_left"], st["n_halo_right"]]
            if not periodic_y:
                s.set_state(piston_active=1)
            U, Up = s.total_U()
            P, Pp = s.pressure_sum(periodic_y)
            K, Kp = s.total_K()
            L, Lp = s.partial_U_lambda(EPS_LAMBDA, periodic_y)
            arrays[f"{tag}/U_partials"] = Up
            arrays[f"{tag}/P_partials"] = Pp
            arrays[f"{tag}/K_partials"] = Kp
            arrays[f"{tag}/dUdl_partials"] = Lp
            m[f"ws{ws1}_t{th}"] = {"U": U, "Psum": P, "K": K, "dUdl": L}
            if not periodic_y and ws1 == 0 and th == threads[0]:
                up, en = s.piston_wall(update_acc=True)
                arrays[f"{name}/wall_acc"] = s.frame()["acc"].copy()
                m["wall_upper"] = up
                m["wall_energy"] = en
            s.close()
    meta[name] = m


def record_traj(name, start, cfg, frame, kind, nsteps, p_ext, arrays, meta, ws1=0):
    """nsteps of one step kind from the frame of static case `start`."""
    s = rk.RefSim(cfg, frame, ws1_halo=bool(ws1), threads=256, init_forces=True)
    K, U = s.step(kind, nsteps, p_ext=p_ext, trace=True)
    f = s.frame()
    arrays[f"{name}/K_trace"] = K
    arrays[f"{name}/U_trace"] = U
    arrays[f"{name}/final_pos"] = f["pos"].copy()
    arrays[f"{name}/final_vel"] = f["vel"].copy()
    arrays[f"{name}/final_acc"] = f["acc"].copy()
    meta[name] = {"kind": kind, "nsteps": nsteps, "p_ext": p_ext, "ws1_halo": ws1,
                  "cfg": cfg, "state": s.state(), "start": start}
    s.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    if rk.device_count() < 1:
        raise SystemExit("needs a GPU")
    arrays, meta = {}, {}

    f, Lx, Ly = wl.lattice_frame(512, 0.8, 1.0, 0.65, 1.0, seed=31)
    c_lat = cfg_of(512, Lx, Ly, dt=0.001, T=1.0, barostat_mass=10.0)
    record_static("lat512", c_lat, f, 1, arrays, meta, threads=(256, 128))
    fs, Lxs, Lys = wl.lattice_frame(512, 0.8, 2.0, lambda s: np.where(s < 0.5, 0.9, 0.1), 0.7,
                                    seed=32)
    c_slab = cfg_of(512, Lxs, Lys, dt=0.002, T=0.7, Q=1.0)
    record_static("slab512", c_slab, fs, 1, arrays, meta)
    fd, Ld, seed_d = dense_frame(256, 0.8, 33)
    c_dense = cfg_of(256, Ld, Ld)
    record_static("dense256", c_dense, fd, 1, arrays, meta)
    meta["dense256"]["seed"] = seed_d
    fe, Le = edge_frame(34)
    c_edge = cfg_of(len(fe), Le, Le)
    record_static("edge64", c_edge, fe, 1, arrays, meta)
    fp, Lxp, Lyp = wl.lattice_frame(512, 0.32, 4.0, 0.5, 0.9, seed=35)
    fp["pos"][:6, 1] = [-0.05, -0.3, Lyp + 0.02, Lyp + 0.4, -1e-3, Lyp + 1e-3]
    c_pis = cfg_of(512, Lxp, Lyp, dt=0.001, T=0.9, barostat_mass=10.0, k_piston=100.0)
    record_static("piston512", c_pis, fp, 0, arrays, meta)

    # integrator kernels, one at a time on a fresh copy
    Li = 20.0
    fi = integ_frame(256, Li, 36)
    c_int = cfg_of(256, Li, Li)
    arrays["integ256/frame_pos"] = fi["pos"].copy()
    arrays["integ256/frame_vel"] = fi["vel"].copy()
    arrays["integ256/frame_acc"] = fi["acc"].copy()
    arrays["integ256/frame_type"] = fi["type"].astype(np.int32)
    icalls = {
        "half_vv": (rk.HALF_VV, dict(dt=0.003)),
        "second_half_vv": (rk.SECOND_HALF_VV, dict(dt=0.003)),
        "half_vv_nh": (rk.HALF_VV_NH, dict(dt=0.003, xi=0.37)),
        "second_half_vv_nh": (rk.SECOND_HALF_VV_NH, dict(dt=0.003, xi=-0.21)),
        "half_nph_vel": (rk.HALF_NPH_VEL, dict(dt=0.003)),
        "nph_scale_drift": (rk.NPH_SCALE_DRIFT,
                            dict(dt=0.003, lin=1.000317, vsc=1.0 / 1.000317,
                                 Lx_new=Li * 1.000317, Ly_new=Li * 1.000317)),
        "half_vv_piston": (rk.HALF_VV_PISTON, dict(dt=0.003)),
    }
    meta["integ256"] = {"L": Li, "calls": {k: v[1] for k, v in icalls.items()}}
    for key, (which, kw) in icalls.items():
        s = rk.RefSim(c_int, fi, threads=256, init_forces=False)
        s.integrator(which, **kw)
        g = s.frame()
        arrays[f"integ256/{key}/pos"] = g["pos"].copy()
        arrays[f"integ256/{key}/vel"] = g["vel"].copy()
        s.close()

    # trajectories
    record_traj("nve_lat512", "lat512", c_lat, f, rk.KIND_NVE, 40, 0.0, arrays, meta)
    record_traj("nve_lat512_ws1", "lat512", c_lat, f, rk.KIND_NVE, 10, 0.0, arrays, meta, ws1=1)
    record_traj("nh_slab512", "slab512", c_slab, fs, rk.KIND_NH, 40, 0.0, arrays, meta)
    record_traj("nph_lat512", "lat512", c_lat, f, rk.KIND_NPH, 20, 1.0, arrays, meta)
    record_traj("piston_traj512", "piston512", c_pis, fp, rk.KIND_PISTON, 20, 0.5, arrays, meta)

    os.makedirs(a.out, exist_ok=True)
    np.savez_compressed(os.path.join(a.out, "ref_physics.npz"), **arrays)
    with open(os.path.join(a.out, "ref_physics.json"), "w") as fh:
        json.dump(meta, fh, indent=1, sort_keys=True)
    print("wrote", len(arrays), "arrays to", a.out)


if __name__ == "__main__":
    main()
