"""ctypes binding of the CPU oracle (oracle/mdoracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
as the checker and by bench.py's CPU-baseline leg. The product package never
imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libmdoracle.so")
_lock = threading.Lock()
_lib = None

OR_FP64 = 0
OR_REF_MIXED = 1


class OrLJ(C.Structure):
    _fields_ = [
        ("sigma", C.c_double * 3),
        ("epsilon", C.c_double * 3),
        ("mass_a", C.c_double),
        ("mass_b", C.c_double),
        ("cutoff", C.c_double),
    ]


class OrSim(C.Structure):
    _fields_ = [
        ("n", C.c_int64),
        ("pos", C.POINTER(C.c_double)),
        ("vel", C.POINTER(C.c_double)),
        ("acc", C.POINTER(C.c_double)),
        ("type", C.POINTER(C.c_int32)),
        ("lj", OrLJ),
        ("dt", C.c_double),
        ("Q", C.c_double),
        ("T_target", C.c_double),
        ("n_global", C.c_int64),
        ("barostat_mass", C.c_double),
        ("k_piston", C.c_double),
        ("area_rate_init", C.c_double),
        ("hmin_ratio", C.c_double),
        ("hmax_ratio", C.c_double),
        ("Lx", C.c_double),
        ("Ly", C.c_double),
        ("Lx0", C.c_double),
        ("Ly0", C.c_double),
        ("t", C.c_double),
        ("xi", C.c_double),
        ("nph_area_momentum", C.c_double),
        ("nph_aspect_ratio", C.c_double),
        ("nph_state_initialized", C.c_int32),
        ("piston_velocity", C.c_double),
        ("piston_force", C.c_double),
        ("piston_velocity_initialized", C.c_int32),
        ("piston_mode_active", C.c_int32),
        ("last_instant_pressure", C.c_double),
        ("mode", C.c_int32),
        ("ws1_halo", C.c_int32),
        ("use_cells", C.c_int32),
        ("nthreads", C.c_int32),
        ("error", C.c_int32),
        ("ref_threads", C.c_int32),
    ]


class OrFireParams(C.Structure):
    _fields_ = [
        ("dt_init", C.c_double),
        ("dt_max", C.c_double),
        ("alpha0", C.c_double),
        ("f_inc", C.c_double),
        ("f_dec", C.c_double),
        ("N_min", C.c_int32),
    ]


class OrFireResult(C.Structure):
    _fields_ = [
        ("steps", C.c_int32),
        ("converged", C.c_int32),
        ("max_force", C.c_double),
        ("potential_energy", C.c_double),
        ("n_energy_samples", C.c_int64),
    ]


def build(force: bool = False) -> str:
    """Compile libmdoracle.so with the committed Makefile (no-op when fresh)."""
    src = os.path.join(_HERE, "mdoracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-C", _HERE, "libmdoracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return _LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            build()
            L = C.CDLL(_LIB_PATH)
            dp = C.POINTER(C.c_double)
            ip = C.POINTER(C.c_int32)
            L.or_forces_allpairs.argtypes = [C.POINTER(OrLJ), C.c_int64, dp, ip, C.c_double,
                                             C.c_double, C.c_int32, C.c_int32, C.c_int32, dp, dp,
                                             dp, C.c_int32]
            L.or_forces_cells.argtypes = [C.POINTER(OrLJ), C.c_int64, dp, ip, C.c_double,
                                          C.c_double, C.c_int32, C.c_int32, dp, dp, dp, C.c_int32]
            L.or_count_pairs.argtypes = [C.POINTER(OrLJ), C.c_int64, dp, ip, C.c_double,
                                         C.c_double, C.c_int32, C.c_int32]
            L.or_count_pairs.restype = C.c_int64
            L.or_n_profile.argtypes = [C.c_int64, dp, ip, C.c_double, C.c_int32, ip]
            L.or_pressure_profile.argtypes = [C.POINTER(OrLJ), C.c_int64, dp, dp, ip, C.c_double,
                                              C.c_double, C.c_int32, C.c_int32, C.c_int32, dp]
            L.or_partial_U_lambda.argtypes = [C.POINTER(OrLJ), C.c_int64, dp, ip, C.c_double,
                                              C.c_double, C.c_int32, C.c_int32, C.c_double, dp,
                                              dp, C.c_int32]
            L.or_count_pairs_cells.argtypes = [C.POINTER(OrLJ), C.c_int64, dp, ip, C.c_double,
                                               C.c_double, C.c_int32]
            L.or_count_pairs_cells.restype = C.c_int64
            L.or_forces_rows.argtypes = [C.POINTER(OrLJ), C.c_int64, dp, ip, C.c_double,
                                         C.c_double, C.c_int32, C.c_int32, C.c_int64, C.c_int64,
                                         dp, C.c_int32]
            L.or_ref_thread_values.argtypes = [C.POINTER(OrLJ), C.c_int64, dp, dp, ip,
                                               C.c_double, C.c_double, C.c_int32, C.c_int32,
                                               C.c_int32, C.c_int32, C.c_double, dp, C.c_int32]
            L.or_ref_block_partials.argtypes = [C.c_int64, dp, C.c_int32, dp]
            L.or_ref_integrator.argtypes = [C.c_int32, C.c_int64, dp, dp, dp, C.c_double,
                                            C.c_double, C.c_double, C.c_double, C.c_double,
                                            C.c_double]
            L.or_ref_block_partials.restype = C.c_double
            L.or_cell_grid.argtypes = [C.c_double, C.c_double, C.c_double, ip, ip]
            L.or_cell_bin.argtypes = [C.c_int64, dp, C.c_double, C.c_double, C.c_int32,
                                      C.c_int32, ip]
            L.or_cell_sort.argtypes = [C.c_int64, ip, C.c_int32, ip, ip]
            L.or_pbc_wrap.argtypes = [C.c_double, C.c_double]
            L.or_pbc_wrap.restype = C.c_double
            sp = C.POINTER(OrSim)
            for name in ("or_sim_setup", "or_step_nve", "or_step_nose_hoover"):
                getattr(L, name).argtypes = [sp]
            L.or_sim_cal_forces.argtypes = [sp, C.c_int32]
            L.or_sim_piston_walls.argtypes = [sp, C.c_int32, dp, dp]
            L.or_sim_piston_walls.restype = None
            L.or_step_nph.argtypes = [sp, C.c_double]
            L.or_step_nph_piston.argtypes = [sp, C.c_double]
            for name in ("or_total_K", "or_total_U", "or_instant_pressure"):
                getattr(L, name).argtypes = [sp]
                getattr(L, name).restype = C.c_double
            L.or_scalar_pressure.argtypes = [sp, C.c_int32]
            L.or_scalar_pressure.restype = C.c_double
            L.or_fire_minimize.argtypes = [C.POINTER(OrLJ), C.c_int64, dp, dp, dp, ip,
                                           C.c_double, C.c_double, C.c_double, C.c_int32,
                                           C.POINTER(OrFireParams), C.c_int32, C.c_int32,
                                           C.c_int32, C.c_int32, C.POINTER(OrFireResult), ip, dp,
                                           C.c_int64]
            _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def make_lj(cfg) -> OrLJ:
    """LJ parameters from a config mapping with the MDConfig key names."""
    lj = OrLJ()
    lj.sigma[:] = [cfg["SIGMA_AA"], cfg["SIGMA_BB"], cfg["SIGMA_AB"]]
    lj.epsilon[:] = [cfg["EPSILON_AA"], cfg["EPSILON_BB"], cfg["EPSILON_AB"]]
    lj.mass_a = cfg["MASS_A"]
    lj.mass_b = cfg["MASS_B"]
    lj.cutoff = cfg["cutoff"]
    return lj


def _pos2(pos):
    p = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 2)
    return p


def forces(cfg, pos, types, Lx, Ly, periodic_y=1, mode=OR_FP64, ws1_halo=0, cells=False,
           nthreads=0):
    """Return (acc[n,2], U, W) for one frame."""
    p = _pos2(pos)
    t = np.ascontiguousarray(types, dtype=np.int32)
    n = p.shape[0]
    acc = np.zeros((n, 2), dtype=np.float64)
    U = C.c_double(0.0)
    W = C.c_double(0.0)
    lj = make_lj(cfg)
    if cells:
        rc = lib().or_forces_cells(C.byref(lj), n, _dp(p), _ip(t), Lx, Ly, periodic_y, mode,
                                   _dp(acc), C.byref(U), C.byref(W), nthreads)
    else:
        rc = lib().or_forces_allpairs(C.byref(lj), n, _dp(p), _ip(t), Lx, Ly, periodic_y, mode,
                                      ws1_halo, _dp(acc), C.byref(U), C.byref(W), nthreads)
    if rc != 0:
        raise RuntimeError(f"oracle forces failed ({rc})")
    return acc, U.value, W.value


def count_pairs(cfg, pos, types, Lx, Ly, periodic_y=1, nthreads=0):
    p = _pos2(pos)
    t = np.ascontiguousarray(types, dtype=np.int32)
    lj = make_lj(cfg)
    return int(lib().or_count_pairs(C.byref(lj), p.shape[0], _dp(p), _ip(t), Lx, Ly, periodic_y,
                                    nthreads))


def partial_U_lambda(cfg, pos, types, Lx, Ly, eps_lambda, periodic_y=1, mode=0, nthreads=0):
    """(dU/dlambda, magnitude scale) of or_partial_U_lambda (all pairs)."""
    p = _pos2(pos)
    t = np.ascontiguousarray(types, dtype=np.int32)
    lj = make_lj(cfg)
    out = C.c_double()
    scale = C.c_double()
    rc = lib().or_partial_U_lambda(C.byref(lj), p.shape[0], _dp(p), _ip(t), Lx, Ly, periodic_y,
                                   mode, float(eps_lambda), C.byref(out), C.byref(scale),
                                   nthreads)
    assert rc == 0
    return out.value, scale.value


def n_profile(pos, types, Lx, nb):
    """get_N_profile: (counts of type 0, counts of other types) in x bins."""
    p = _pos2(pos)
    t = np.ascontiguousarray(types, dtype=np.int32)
    out = np.zeros(2 * nb, dtype=np.int32)
    assert lib().or_n_profile(p.shape[0], _dp(p), _ip(t), Lx, nb, _ip(out)) == 0
    return out[:nb], out[nb:]


def pressure_profile(cfg, pos, vel, types, Lx, Ly, nb, periodic_y=1, mode=0):
    """get_pressure_profile: (Pxx, Pyy, Pxy) in y bins."""
    p = _pos2(pos)
    v = _pos2(vel)
    t = np.ascontiguousarray(types, dtype=np.int32)
    lj = make_lj(cfg)
    out = np.zeros(3 * nb)
    assert lib().or_pressure_profile(C.byref(lj), p.shape[0], _dp(p), _dp(v), _ip(t), Lx, Ly,
                                     periodic_y, mode, nb, _dp(out)) == 0
    return out[:nb], out[nb:2 * nb], out[2 * nb:]


def count_pairs_cells(cfg, pos, types, Lx, Ly, nthreads=0):
    p = _pos2(pos)
    t = np.ascontiguousarray(types, dtype=np.int32)
    lj = make_lj(cfg)
    return int(lib().or_count_pairs_cells(C.byref(lj), p.shape[0], _dp(p), _ip(t), Lx, Ly,
                                          nthreads))


def forces_rows(cfg, pos, types, Lx, Ly, row0, nrows, periodic_y=1, mode=OR_REF_MIXED,
                nthreads=0):
    """acc of rows [row0, row0+nrows) through the all-pairs loop."""
    p = _pos2(pos)
    t = np.ascontiguousarray(types, dtype=np.int32)
    acc = np.zeros((nrows, 2))
    lj = make_lj(cfg)
    rc = lib().or_forces_rows(C.byref(lj), p.shape[0], _dp(p), _ip(t), Lx, Ly, periodic_y, mode,
                              row0, nrows, _dp(acc), nthreads)
    if rc != 0:
        raise RuntimeError("oracle forces_rows failed")
    return acc


OR_SUM_U, OR_SUM_P, OR_SUM_K, OR_SUM_DUDL = 0, 1, 2, 3


def ref_thread_values(cfg, pos, vel, types, Lx, Ly, what, periodic_y=1, mode=OR_REF_MIXED,
                      ws1_halo=0, eps_lambda=0.0, nthreads=0):
    """Per-thread values of the reference's block-reduced kernels (OR_SUM_*)."""
    p = _pos2(pos)
    v = np.ascontiguousarray(vel, dtype=np.float64).reshape(-1, 2)
    t = np.ascontiguousarray(types, dtype=np.int32)
    out = np.zeros(p.shape[0])
    lj = make_lj(cfg)
    rc = lib().or_ref_thread_values(C.byref(lj), p.shape[0], _dp(p), _dp(v), _ip(t), Lx, Ly,
                                    periodic_y, mode, ws1_halo, what, float(eps_lambda),
                                    _dp(out), nthreads)
    if rc != 0:
        raise RuntimeError(f"oracle ref_thread_values failed ({rc})")
    return out


def ref_block_partials(values, threads=256):
    """(block-order total, per-block partials) of the reference's block tree."""
    v = np.ascontiguousarray(values, dtype=np.float64)
    nb = (len(v) + threads - 1) // threads
    part = np.zeros(max(nb, 1))
    tot = lib().or_ref_block_partials(len(v), _dp(v), threads, _dp(part))
    return tot, part[:nb]


def ref_integrator(which, pos, vel, acc, dt, xi=0.0, lin=1.0, vsc=1.0, Lx=0.0, Ly=0.0):
    """One of the reference's integrator kernels (or_ref_integrator): new (pos, vel)."""
    p = np.array(_pos2(pos), dtype=np.float64, copy=True)
    v = np.array(_pos2(vel), dtype=np.float64, copy=True)
    a = np.ascontiguousarray(_pos2(acc), dtype=np.float64)
    assert lib().or_ref_integrator(which, p.shape[0], _dp(p), _dp(v), _dp(a), dt, xi, lin, vsc,
                                   Lx, Ly) == 0
    return p, v


def cell_build(pos, Lx, Ly, cell_min):
    """Project binning: (cell ids, stable permutation, ncx, ncy)."""
    p = _pos2(pos)
    n = p.shape[0]
    ncx = C.c_int32()
    ncy = C.c_int32()
    lib().or_cell_grid(Lx, Ly, cell_min, C.byref(ncx), C.byref(ncy))
    cell = np.zeros(n, dtype=np.int32)
    lib().or_cell_bin(n, _dp(p), Lx, Ly, ncx.value, ncy.value, _ip(cell))
    perm = np.zeros(n, dtype=np.int32)
    start = np.zeros(ncx.value * ncy.value + 1, dtype=np.int32)
    lib().or_cell_sort(n, _ip(cell), ncx.value * ncy.value, _ip(perm), _ip(start))
    return cell, perm, ncx.value, ncy.value


def pbc_wrap(x, L):
    return lib().or_pbc_wrap(float(x), float(L))


class Sim:
    """Stateful oracle engine mirroring MDSimulation's hot path."""

    def __init__(self, cfg, pos, vel, types, mode=OR_FP64, ws1_halo=0, use_cells=True,
                 nthreads=0, ref_threads=0):
        self.pos = np.array(_pos2(pos), dtype=np.float64, copy=True)
        n = self.pos.shape[0]
        self.vel = np.array(np.asarray(vel, dtype=np.float64).reshape(n, 2), copy=True)
        self.acc = np.zeros((n, 2), dtype=np.float64)
        self.type = np.array(np.asarray(types, dtype=np.int32).reshape(n), copy=True)
        s = OrSim()
        s.n = n
        s.pos = _dp(self.pos)
        s.vel = _dp(self.vel)
        s.acc = _dp(self.acc)
        s.type = _ip(self.type)
        s.lj = make_lj(cfg)
        s.dt = cfg["dt"]
        s.Q = cfg["Q"]
        s.T_target = cfg["T_target"]
        s.n_global = int(cfg.get("n_particles_global", n) or n)
        s.barostat_mass = cfg.get("barostat_mass", 1.0e4)
        s.k_piston = cfg.get("k_piston", 100.0)
        s.area_rate_init = cfg.get("barostat_area_rate_init", 0.0)
        s.hmin_ratio = cfg.get("barostat_height_min_ratio", 0.6)
        s.hmax_ratio = cfg.get("barostat_height_max_ratio", 1.4)
        s.Lx = cfg["box_w_global"]
        s.Ly = cfg["box_h_global"]
        s.mode = mode
        s.ws1_halo = ws1_halo
        s.use_cells = 1 if use_cells else 0
        s.nthreads = nthreads
        s.ref_threads = ref_threads
        self.s = s
        lib().or_sim_setup(C.byref(s))

    def step_nve(self, n=1):
        for _ in range(n):
            lib().or_step_nve(C.byref(self.s))

    def step_nose_hoover(self, n=1):
        for _ in range(n):
            lib().or_step_nose_hoover(C.byref(self.s))

    def step_nph(self, p_ext, n=1):
        for _ in range(n):
            lib().or_step_nph(C.byref(self.s), p_ext)

    def step_nph_piston(self, p_ext, n=1):
        for _ in range(n):
            lib().or_step_nph_piston(C.byref(self.s), p_ext)

    def cal_forces(self, periodic_y=1):
        lib().or_sim_cal_forces(C.byref(self.s), periodic_y)

    def piston_walls(self, update_acc=False):
        """(upper-wall force, wall energy); update_acc adds the walls to acc."""
        up, en = C.c_double(), C.c_double()
        lib().or_sim_piston_walls(C.byref(self.s), 1 if update_acc else 0, C.byref(up),
                                  C.byref(en))
        return up.value, en.value

    def total_K(self):
        return lib().or_total_K(C.byref(self.s))

    def total_U(self):
        return lib().or_total_U(C.byref(self.s))

    def instant_pressure(self):
        return lib().or_instant_pressure(C.byref(self.s))

    def __getattr__(self, name):
        s = self.__dict__.get("s")
        if s is not None and name in dict(OrSim._fields_):
            return getattr(s, name)
        raise AttributeError(name)


def fire_minimize(cfg, pos, types, Lx, Ly, force_tol, max_steps, params, mode=OR_FP64,
                  ws1_halo=0, use_cells=True, nthreads=0, trace_cap=64):
    """EnergyMinimizer::minimize_frame on the CPU. Returns a dict."""
    p = np.array(_pos2(pos), dtype=np.float64, copy=True)
    n = p.shape[0]
    vel = np.zeros((n, 2))
    acc = np.zeros((n, 2))
    t = np.ascontiguousarray(types, dtype=np.int32)
    fp = OrFireParams(params["dt_init"], params["dt_max"], params["alpha0"], params["f_inc"],
                      params["f_dec"], params["N_min"])
    res = OrFireResult()
    es = np.zeros(trace_cap, dtype=np.int32)
    et = np.zeros(trace_cap, dtype=np.float64)
    lj = make_lj(cfg)
    rc = lib().or_fire_minimize(C.byref(lj), n, _dp(p), _dp(vel), _dp(acc), _ip(t), Lx, Ly,
                                force_tol, max_steps, C.byref(fp), mode, ws1_halo,
                                1 if use_cells else 0, nthreads, C.byref(res), _ip(es), _dp(et),
                                trace_cap)
    if rc != 0:
        raise RuntimeError(f"oracle FIRE failed ({rc})")
    k = min(res.n_energy_samples, trace_cap)
    return dict(pos=p, vel=vel, acc=acc, steps=res.steps, converged=bool(res.converged),
                max_force=res.max_force, potential_energy=res.potential_energy,
                energy_steps=es[:k].tolist(), energy_trace=et[:k].tolist())
