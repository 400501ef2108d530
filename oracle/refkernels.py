"""ctypes binding of the reference's own CUDA kernels (oracle/_ref/libref_kernels.so).

The library is the reference's unmodified src/md_cuda_common.cu compiled for
sm_100a, plus oracle/ref_kernels.cu, a restatement of the reference's host
step logic at MPI world size 1 (src/md_env.cu:1511-2360). oracle/build_ref.py
builds it where the reference tree is present; the built file travels with the
repository to the GPU machine.

TEST INFRASTRUCTURE ONLY: the parity tests use it to pin the oracle and the
product against the reference's own kernels, the golden-fixture script
records its outputs, and bench.py times the reference's single-GPU step with
it. The product package never imports it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libref_kernels.so")
_lib = None

KIND_NVE, KIND_NH, KIND_NPH, KIND_PISTON = 0, 1, 2, 3
(HALF_VV, SECOND_HALF_VV, HALF_VV_NH, SECOND_HALF_VV_NH, HALF_NPH_VEL, NPH_SCALE_DRIFT,
 HALF_VV_PISTON) = range(7)


class RefLJ(C.Structure):
    _fields_ = [("sigma", C.c_double * 3), ("epsilon", C.c_double * 3), ("mass_a", C.c_double),
                ("mass_b", C.c_double), ("cutoff", C.c_double)]


class RefParams(C.Structure):
    _fields_ = [("dt", C.c_double), ("Q", C.c_double), ("T_target", C.c_double),
                ("barostat_mass", C.c_double), ("k_piston", C.c_double),
                ("area_rate_init", C.c_double), ("hmin_ratio", C.c_double),
                ("hmax_ratio", C.c_double), ("n_global", C.c_int64), ("threads", C.c_int32),
                ("ws1_halo", C.c_int32)]


class RefState(C.Structure):
    _fields_ = [("Lx", C.c_double), ("Ly", C.c_double), ("Lx0", C.c_double),
                ("Ly0", C.c_double), ("t", C.c_double), ("xi", C.c_double),
                ("nph_area_momentum", C.c_double), ("nph_aspect_ratio", C.c_double),
                ("piston_velocity", C.c_double), ("piston_force", C.c_double),
                ("last_P", C.c_double), ("nph_init", C.c_int32), ("piston_vel_init", C.c_int32),
                ("piston_active", C.c_int32), ("n_halo_left", C.c_int32),
                ("n_halo_right", C.c_int32), ("pad", C.c_int32)]


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"{LIB_PATH} is not built (oracle/build_ref.py)")
        L = C.CDLL(LIB_PATH)
        vp, dp = C.c_void_p, C.POINTER(C.c_double)
        L.refk_device_count.restype = C.c_int
        L.refk_create.argtypes = [C.POINTER(RefLJ), C.POINTER(RefParams), C.c_int32, vp,
                                  C.c_double, C.c_double, C.POINTER(vp)]
        L.refk_destroy.argtypes = [vp]
        L.refk_destroy.restype = None
        L.refk_get_frame.argtypes = [vp, vp]
        L.refk_set_frame.argtypes = [vp, vp]
        L.refk_get_state.argtypes = [vp, C.POINTER(RefState)]
        L.refk_set_state.argtypes = [vp, C.POINTER(RefState)]
        L.refk_cal_forces.argtypes = [vp, C.c_int32]
        L.refk_total_K.argtypes = [vp, dp, dp]
        L.refk_total_U.argtypes = [vp, dp, dp]
        L.refk_pressure_sum.argtypes = [vp, C.c_int32, dp, dp]
        L.refk_piston_wall.argtypes = [vp, C.c_int32, dp, dp]
        L.refk_partial_U_lambda.argtypes = [vp, C.c_double, C.c_int32, dp, dp]
        L.refk_integrator.argtypes = [vp, C.c_int32, C.c_double, C.c_double, C.c_double,
                                      C.c_double, C.c_double, C.c_double]
        L.refk_step.argtypes = [vp, C.c_int32, C.c_double, C.c_int32, dp, dp]
        L.refk_time_steps.argtypes = [vp, C.c_int32, C.c_double, C.c_int32, dp]
        _lib = L
    return _lib


def _ok(rc, what):
    if rc != 0:
        raise RuntimeError(f"reference kernel call {what} failed ({rc})")


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class RefSim:
    """The reference's MDSimulation step path at world size 1 on one GPU.

    cfg: a mapping with the MDConfig key names; frame: a 64-byte Particle
    record array (md_simulation_cuda_b200.PARTICLE_DTYPE layout)."""

    def __init__(self, cfg, frame, ws1_halo=False, threads=256, init_forces=True):
        lj = RefLJ()
        lj.sigma[:] = [cfg["SIGMA_AA"], cfg["SIGMA_BB"], cfg["SIGMA_AB"]]
        lj.epsilon[:] = [cfg["EPSILON_AA"], cfg["EPSILON_BB"], cfg["EPSILON_AB"]]
        lj.mass_a, lj.mass_b, lj.cutoff = cfg["MASS_A"], cfg["MASS_B"], cfg["cutoff"]
        p = RefParams()
        p.dt = cfg["dt"]
        p.Q = cfg.get("Q", 1.0)
        p.T_target = cfg.get("T_target", 1.0)
        p.barostat_mass = cfg.get("barostat_mass", 1.0e4)
        p.k_piston = cfg.get("k_piston", 100.0)
        p.area_rate_init = cfg.get("barostat_area_rate_init", 0.0)
        p.hmin_ratio = cfg.get("barostat_height_min_ratio", 0.6)
        p.hmax_ratio = cfg.get("barostat_height_max_ratio", 1.4)
        p.n_global = int(cfg.get("n_particles_global", len(frame)) or len(frame))
        p.threads = threads
        p.ws1_halo = 1 if ws1_halo else 0
        self.n = len(frame)
        self.threads = threads
        self._frame_dtype = frame.dtype
        fr = np.ascontiguousarray(frame)
        h = C.c_void_p()
        _ok(lib().refk_create(C.byref(lj), C.byref(p), self.n, fr.ctypes.data_as(C.c_void_p),
                              float(cfg["box_w_global"]), float(cfg["box_h_global"]),
                              C.byref(h)), "create")
        self.h = h
        if init_forces:
            self.cal_forces(1)

    def close(self):
        if getattr(self, "h", None):
            lib().refk_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def blocks(self):
        return (self.n + self.threads - 1) // self.threads

    def frame(self):
        out = np.zeros(self.n, dtype=self._frame_dtype)
        _ok(lib().refk_get_frame(self.h, out.ctypes.data_as(C.c_void_p)), "get_frame")
        return out

    def set_frame(self, fr):
        fr = np.ascontiguousarray(fr)
        _ok(lib().refk_set_frame(self.h, fr.ctypes.data_as(C.c_void_p)), "set_frame")

    def state(self):
        s = RefState()
        _ok(lib().refk_get_state(self.h, C.byref(s)), "state")
        return {k: getattr(s, k) for k, _ in RefState._fields_}

    def set_state(self, **kw):
        s = RefState()
        _ok(lib().refk_get_state(self.h, C.byref(s)), "state")
        for k, v in kw.items():
            setattr(s, k, v)
        _ok(lib().refk_set_state(self.h, C.byref(s)), "set_state")

    def cal_forces(self, periodic_y=1):
        _ok(lib().refk_cal_forces(self.h, periodic_y), "cal_forces")

    def _partials(self, name, *args):
        part = np.zeros(max(self.blocks, 1))
        tot = C.c_double()
        _ok(getattr(lib(), name)(self.h, *args, C.byref(tot), _dp(part)), name)
        return tot.value, part[:self.blocks]

    def total_K(self):
        return self._partials("refk_total_K")

    def total_U(self):
        return self._partials("refk_total_U")

    def pressure_sum(self, periodic_y=1):
        return self._partials("refk_pressure_sum", periodic_y)

    def partial_U_lambda(self, eps_lambda, periodic_y=1):
        return self._partials("refk_partial_U_lambda", float(eps_lambda), periodic_y)

    def piston_wall(self, update_acc=False):
        up, en = C.c_double(), C.c_double()
        _ok(lib().refk_piston_wall(self.h, 1 if update_acc else 0, C.byref(up), C.byref(en)),
            "piston_wall")
        return up.value, en.value

    def integrator(self, which, dt, xi=0.0, lin=1.0, vsc=1.0, Lx_new=0.0, Ly_new=0.0):
        _ok(lib().refk_integrator(self.h, which, dt, xi, lin, vsc, Lx_new, Ly_new), "integrator")

    def step(self, kind, nsteps=1, p_ext=0.0, trace=False):
        if not trace:
            _ok(lib().refk_step(self.h, kind, p_ext, nsteps, None, None), "step")
            return None
        K = np.zeros(nsteps)
        U = np.zeros(nsteps)
        _ok(lib().refk_step(self.h, kind, p_ext, nsteps, _dp(K), _dp(U)), "step")
        return K, U

    def time_steps(self, kind, nsteps, p_ext=0.0):
        ms = C.c_double()
        _ok(lib().refk_time_steps(self.h, kind, p_ext, nsteps, C.byref(ms)), "time_steps")
        return ms.value


def device_count() -> int:
    return int(lib().refk_device_count()) if available() else 0
