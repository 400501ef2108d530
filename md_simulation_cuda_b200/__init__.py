"""md_simulation_cuda_b200 — B200-native MD stepping path of MD_Simulation_CUDA.

Python mirror of the reference's C++ surface for the hot path, over the C ABI of
``libmdb200.so`` (include/mdb200.h):

* ``MDConfig`` / ``MDConfigManager``  — include/md_config.hpp:14-111
* ``MDSimulation``                    — include/md_env.hpp:51-263 (hot path)
* ``EnergyMinimizer``, ``FireParams``, ``MinimizeResult``
                                      — include/md_energy_minimizer.hpp:11-97
* ``FileWriter`` / ``FileReader``     — include/md_common.hpp:88-122 (PFRAME v2)
* ``Batch``                           — many independent systems in one launch
* ``Server``                          — continuous batching of MD / FIRE requests
* ``TrajectoryWriter``                — asynchronous PFRAME writer

Frames are numpy arrays of ``PARTICLE_DTYPE`` (the 64-byte Particle of
include/md_particle.hpp:31-38). The MPI communicator arguments of the reference
are accepted and ignored: one process drives one GPU and resolves every
periodic image itself.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from ._lib import (FIRE_AUTO, FIRE_FP32, FIRE_FP64, LANES_AUTO, LANES_ONE, LANES_SPLIT,
                   STEPS_AUTO, STEPS_MULTI, STEPS_PER_PHASE,
                   MDB_ERR_ARG, MDBConfigC, MDBError,
                   MDBFireParams, MDBMinimizeResult,
                   MDBNphProtocol, MDBNphRecord, MDBNphResult, MDBObservables, MDBRequest,
                   MDBRequestResult, MDBServerOptions, MDBServerStats, PARTICLE_DTYPE, check,
                   frame_ptr, lib, options)

# job kinds (mdb200.h MDB_JOB_*) and request states (MDB_REQ_*)
JOB_FIRE, JOB_NVE, JOB_NVT = 0, 1, 2
REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED = 0, 1, 2, 3
# server admission orders (MDB_ORDER_*)
ORDER_FIFO, ORDER_SHORTEST = 0, 1

__all__ = [
    "PARTICLE_DTYPE", "MDBError", "MDConfig", "MDConfigManager", "MDSimulation",
    "EnergyMinimizer", "FireParams", "MinimizeResult", "FileWriter", "FileReader",
    "TrajectoryWriter", "Batch", "Server", "RequestResult", "make_frame", "compute_forces",
    "cell_build", "kernel_launches", "JOB_FIRE", "JOB_NVE", "JOB_NVT", "REQ_QUEUED",
    "REQ_RUNNING", "REQ_DONE", "REQ_FAILED", "ORDER_FIFO", "ORDER_SHORTEST",
]

MDConfig = MDBConfigC  # field-for-field MDConfig


def make_frame(n: int) -> np.ndarray:
    """A zeroed frame of n particles."""
    return np.zeros(n, dtype=PARTICLE_DTYPE)


def _as_frame(frame) -> np.ndarray:
    f = np.ascontiguousarray(frame)
    if f.dtype != PARTICLE_DTYPE:
        raise TypeError("frame must have PARTICLE_DTYPE")
    return f


class MDConfigManager:
    """MDConfigManager (include/md_config.hpp:82-111, src/md_config.cpp)."""

    def __init__(self, config: Optional[MDBConfigC] = None):
        if config is None:
            config = MDBConfigC()
            check(lib().mdb_config_default(C.byref(config)))
        self.config = config

    @staticmethod
    def config_from_json(filepath: str) -> "MDConfigManager":
        cfg = MDBConfigC()
        if not os.path.exists(filepath):
            raise RuntimeError("Failed to open config file: " + str(filepath))
        check(lib().mdb_config_from_json_file(os.fsencode(filepath), C.byref(cfg)))
        return MDConfigManager(cfg)

    def _dump(self, indent: int) -> str:
        need = C.c_size_t(0)
        check(lib().mdb_config_to_json(C.byref(self.config), indent, None, 0, C.byref(need)))
        buf = C.create_string_buffer(need.value + 1)
        check(lib().mdb_config_to_json(C.byref(self.config), indent, buf, len(buf), None))
        return buf.value.decode()

    def config_to_json(self, filepath: str) -> None:
        try:
            with open(filepath, "w") as f:
                f.write(self._dump(4) + "\n")
        except OSError as e:
            raise RuntimeError("Failed to open config file for writing: " + str(filepath)) from e

    def serialize(self) -> str:
        return self._dump(-1)

    def deserialize(self, data: str) -> None:
        # load_from_json_object starts from struct defaults, like the reference
        cfg = MDBConfigC()
        check(lib().mdb_config_from_json(data.encode(), C.byref(cfg)))
        self.config = cfg

    def apply_override(self, key: str, value: str) -> bool:
        rc = lib().mdb_config_apply_override(C.byref(self.config), key.encode(), value.encode())
        return rc == 0

    def apply_overrides(self, overrides: Sequence) -> None:
        for item in overrides:
            key, value = (item.key, item.value) if hasattr(item, "key") else item
            if not self.apply_override(key, value):
                raise RuntimeError(f"Invalid override '{key}={value}'")

    @staticmethod
    def parse_override_argument(argument: str):
        """(key, value) or None, like the reference's bool + out parameters."""
        k = C.create_string_buffer(1024)
        v = C.create_string_buffer(4096)
        rc = lib().mdb_parse_override_argument(argument.encode(), k, len(k), v, len(v))
        if rc != 0:
            return None
        return k.value.decode(), v.value.decode()

    def copy(self) -> "MDConfigManager":
        c = MDBConfigC()
        C.memmove(C.byref(c), C.byref(self.config), C.sizeof(MDBConfigC))
        return MDConfigManager(c)


def _config_of(cfg) -> MDBConfigC:
    if isinstance(cfg, MDConfigManager):
        return cfg.config
    if isinstance(cfg, MDBConfigC):
        return cfg
    if isinstance(cfg, dict):
        m = MDConfigManager()
        for k, v in cfg.items():
            if isinstance(v, str):
                setattr(m.config, k, v.encode())
            else:
                setattr(m.config, k, v)
        return m.config
    raise TypeError("expected MDConfigManager, MDConfig or dict")


class MDSimulation:
    """The stepping part of class MDSimulation (include/md_env.hpp:51-263).

    MDSimulation(cfg, comm)                -> lattice initialisation
    MDSimulation(cfg, comm, filename, step) -> frame `step` of a PFRAME file
    MDSimulation(cfg, frame=array)          -> an in-memory frame
    """

    def __init__(self, config_manager, comm=None, filename: Optional[str] = None,
                 step: Optional[int] = None, *, frame=None, device: int = 0,
                 skin: Optional[float] = None, use_graphs: bool = True,
                 state_file: Optional[str] = None, max_neighbors: Optional[int] = None,
                 autotune: bool = False, step_kernel: Optional[int] = None,
                 lanes: Optional[int] = None):
        self.cfg_manager = config_manager if isinstance(config_manager, MDConfigManager) \
            else MDConfigManager(_config_of(config_manager))
        self._h = C.c_void_p()
        opt = options(device, skin, use_graphs, max_neighbors, autotune=autotune,
                      step_kernel=step_kernel, lanes=lanes)
        cfg = self.cfg_manager.config
        if state_file is not None:
            # a checkpoint: frame `step` of `filename` plus the integrator state
            check(lib().mdb_sim_create_from_checkpoint(
                C.byref(cfg), os.fsencode(filename), int(step or 0), os.fsencode(state_file),
                C.byref(opt), C.byref(self._h)))
        elif filename is not None:
            check(lib().mdb_sim_create_from_pframe(C.byref(cfg), os.fsencode(filename),
                                                   int(step or 0), C.byref(opt),
                                                   C.byref(self._h)))
        elif frame is not None:
            f = _as_frame(frame)
            check(lib().mdb_sim_create(C.byref(cfg), frame_ptr(f), len(f), C.byref(opt),
                                       C.byref(self._h)))
        else:
            check(lib().mdb_sim_create(C.byref(cfg), None, 0, C.byref(opt), C.byref(self._h)))
        self._h_particles = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            # (no ctypes constructor here: at interpreter exit the module
            # globals may already be gone)
            self._h = None
            try:
                lib().mdb_sim_destroy(h)
            except Exception:
                pass

    def close(self):
        self.__del__()

    # ---- steps --------------------------------------------------------
    def step_single_NVE(self, nsteps: int = 1) -> None:
        check(lib().mdb_sim_step_nve(self._h, nsteps))

    step_single = step_single_NVE  # README.md:27 name

    def step_single_nose_hoover(self, do_middle_wrap: bool = False, nsteps: int = 1) -> None:
        check(lib().mdb_sim_step_nose_hoover(self._h, nsteps, 1 if do_middle_wrap else 0))

    def step_single_NPH(self, pressure_ext: float, nsteps: int = 1) -> None:
        check(lib().mdb_sim_step_nph(self._h, float(pressure_ext), nsteps))

    def step_single_NPH_piston(self, pressure_ext: float, nsteps: int = 1) -> None:
        check(lib().mdb_sim_step_nph_piston(self._h, float(pressure_ext), nsteps))

    # ---- observables --------------------------------------------------
    def _scalar(self, fn) -> float:
        out = C.c_double()
        check(fn(self._h, C.byref(out)))
        return out.value

    def cal_total_K(self) -> float:
        return self._scalar(lib().mdb_sim_total_K)

    def cal_total_U(self) -> float:
        return self._scalar(lib().mdb_sim_total_U)

    def cal_partial_U_lambda(self, epsilon_lambda: float) -> float:
        """dU/dlambda of the area-preserving deformation (MDSimulation::
        cal_partial_U_lambda, src/md_env.cu:2362-2406)."""
        v = C.c_double()
        check(lib().mdb_sim_partial_U_lambda(self._h, float(epsilon_lambda), C.byref(v)))
        return v.value

    def get_N_profile(self, n_bins: int) -> np.ndarray:
        """get_N_profile: [count of type 0 per x bin..., count of others...]."""
        out = np.zeros(2 * n_bins, dtype=np.int32)
        check(lib().mdb_sim_n_profile(self._h, int(n_bins),
                                      out.ctypes.data_as(C.POINTER(C.c_int32))))
        return out

    def get_density_profile(self, n_bins: int) -> np.ndarray:
        """get_density_profile: (n_A - n_B) / (n_A + n_B) per x bin."""
        out = np.zeros(n_bins)
        check(lib().mdb_sim_density_profile(self._h, int(n_bins),
                                            out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def get_pressure_profile(self, n_bins: int) -> np.ndarray:
        """get_pressure_profile: [Pxx..., Pyy..., Pxy...] per y bin."""
        out = np.zeros(3 * n_bins)
        check(lib().mdb_sim_pressure_profile(self._h, int(n_bins),
                                             out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def run_nph_protocol(self, protocol: Optional[MDBNphProtocol] = None,
                         record_cap: int = 100000, host_driven: Optional[bool] = None):
        """The NPH driver protocol (AUTO_TARGET -> NPH_WARMUP -> NPH_PRODUCTION of
        tests/run_NPH_test/run_test_NPH.cpp); parameters from the config unless
        given. By default one graph launch with the decisions on the device;
        host_driven=True takes them on the host between step chunks.
        Returns (result, records)."""
        if protocol is None:
            protocol = nph_protocol_from_config(self.cfg_manager)
        if host_driven is not None:
            protocol = MDBNphProtocol.from_buffer_copy(protocol)
            protocol.host_driven = 1 if host_driven else 0
        recs = (MDBNphRecord * max(1, record_cap))()
        res = MDBNphResult()
        check(lib().mdb_sim_run_nph_protocol(self._h, C.byref(protocol), recs, record_cap,
                                             C.byref(res)))
        return res, list(recs[:min(res.n_records, record_cap)])

    def cal_instant_pressure(self) -> float:
        return self._scalar(lib().mdb_sim_instant_pressure)

    def observables_async(self, out_ptr: int) -> None:
        """Queue the observables record into host memory at out_ptr (an
        MDBObservables-sized buffer, ideally pinned); valid after synchronize()."""
        check(lib().mdb_sim_observables_async(self._h, C.c_void_p(out_ptr)))

    def observables(self) -> MDBObservables:
        o = MDBObservables()
        check(lib().mdb_sim_observables(self._h, C.byref(o)))
        return o

    @property
    def t(self) -> float:
        return self.observables().t

    def get_Lx(self) -> float:
        return self.observables().Lx

    def get_Ly(self) -> float:
        return self.observables().Ly

    def get_last_instant_pressure(self) -> float:
        return self.observables().last_instant_pressure

    def get_nph_area_rate(self) -> float:
        return self.observables().nph_area_rate

    def get_nph_piston_velocity(self) -> float:
        return self.observables().nph_piston_velocity

    def get_nph_piston_force(self) -> float:
        return self.observables().nph_piston_force

    @property
    def xi(self) -> float:
        return self.observables().xi

    # ---- frames -------------------------------------------------------
    def n_particles(self) -> int:
        return int(self.observables().n)

    def sample_collect(self) -> None:
        n = self.n_particles()
        f = make_frame(n)
        check(lib().mdb_sim_get_frame(self._h, frame_ptr(f), n))
        self._h_particles = f

    def get_host_particles(self) -> np.ndarray:
        if self._h_particles is None:
            self.sample_collect()
        return self._h_particles.copy()

    def set_frame(self, frame) -> None:
        f = _as_frame(frame)
        check(lib().mdb_sim_set_frame(self._h, frame_ptr(f), len(f)))

    def save_checkpoint(self, filename: str, step: int, state_file: str) -> None:
        """save_env plus the integrator state (restore with
        MDSimulation(cfg, filename=..., step=..., state_file=...))."""
        check(lib().mdb_sim_save_checkpoint(self._h, os.fsencode(filename), int(step),
                                            os.fsencode(state_file)))

    def save_env(self, filename: str, step: int) -> None:
        check(lib().mdb_sim_save_pframe(self._h, os.fsencode(filename), int(step)))

    def synchronize(self) -> None:
        check(lib().mdb_sim_synchronize(self._h))

    def phase_times(self, nsteps: int, nose_hoover: bool = True, nph: bool = False):
        """Summed (drift, rebuild, force) milliseconds of nsteps eager steps,
        from CUDA events on this handle's stream (NPH steps at the pressure of
        the last step_single_NPH call when nph is set)."""
        out = (C.c_double * 3)()
        kind = 3 if nph else (2 if nose_hoover else 1)
        check(lib().mdb_sim_phase_times(self._h, kind, int(nsteps), out))
        return tuple(out)

    def cuda_stream(self) -> int:
        p = C.c_void_p()
        check(lib().mdb_sim_cuda_stream(self._h, C.byref(p)))
        return p.value or 0

    def schedule(self) -> dict:
        """The engine schedule in use (built in, or chosen by the autotuner)."""
        s = _lib.MDBSchedule()
        check(lib().mdb_sim_schedule(self._h, C.byref(s)))
        return s.as_dict()


@dataclass
class FireParams:
    """FireParams (include/md_energy_minimizer.hpp:11-25)."""
    dt_init: float = 0.0
    dt_max: float = 0.0
    alpha0: float = 0.1
    f_inc: float = 1.1
    f_dec: float = 0.5
    N_min: int = 5

    @staticmethod
    def from_config(cfg) -> "FireParams":
        c = _config_of(cfg)
        return FireParams(dt_init=c.dt, dt_max=5.0 * c.dt)

    def _c(self) -> MDBFireParams:
        return MDBFireParams(self.dt_init, self.dt_max, self.alpha0, self.f_inc, self.f_dec,
                             int(self.N_min), 0)


@dataclass
class MinimizeResult:
    """MinimizeResult (include/md_energy_minimizer.hpp:27-35)."""
    frame: np.ndarray = field(default_factory=lambda: make_frame(0))
    energy_steps: List[int] = field(default_factory=list)
    energy_trace: List[float] = field(default_factory=list)
    steps: int = 0
    converged: bool = False
    max_force: float = 0.0
    potential_energy: float = 0.0
    nonfinite: bool = False


class EnergyMinimizer:
    """EnergyMinimizer (include/md_energy_minimizer.hpp:37-97)."""

    def __init__(self, config_manager, comm=None, *, device: int = 0,
                 skin: Optional[float] = None, use_graphs: bool = True,
                 fire_precision: Optional[int] = None):
        self.cfg_manager = config_manager if isinstance(config_manager, MDConfigManager) \
            else MDConfigManager(_config_of(config_manager))
        # allocate_buffers (src/md_energy_minimizer.cu:92-100)
        if self.cfg_manager.config.n_cap <= 0:
            raise RuntimeError("EnergyMinimizer: n_cap must be positive.")
        self._opt = options(device, skin, use_graphs, fire_precision=fire_precision)

    def minimize_frame(self, frame, force_tol: float, max_steps: int,
                       params: FireParams) -> MinimizeResult:
        f = _as_frame(frame)
        if max_steps <= 0:
            raise RuntimeError("EnergyMinimizer: max_steps must be positive.")
        if len(f) > self.cfg_manager.config.n_cap:
            raise RuntimeError("EnergyMinimizer: input frame exceeds buffer capacity.")
        out = make_frame(len(f))
        res = MDBMinimizeResult()
        cap = max_steps // 1000 + 4
        es = np.zeros(cap, dtype=np.int32)
        et = np.zeros(cap, dtype=np.float64)
        p = params._c()
        check(lib().mdb_fire_minimize(
            C.byref(self.cfg_manager.config), frame_ptr(f), len(f), float(force_tol),
            int(max_steps), C.byref(p), C.byref(self._opt), frame_ptr(out), C.byref(res),
            es.ctypes.data_as(C.POINTER(C.c_int32)), et.ctypes.data_as(C.POINTER(C.c_double)),
            cap))
        k = min(res.n_energy_samples, cap)
        return MinimizeResult(frame=out, energy_steps=es[:k].tolist(),
                              energy_trace=et[:k].tolist(), steps=res.steps,
                              converged=bool(res.converged), max_force=res.max_force,
                              potential_energy=res.potential_energy,
                              nonfinite=bool(res.nonfinite))


class FileWriter:
    """FileWriter (include/md_common.hpp:88-99): PFRAME v2 frames."""

    def __init__(self, path: str, append: bool):
        self.path = path
        if append:
            n = C.c_int64()
            last = C.c_uint64()
            rc = lib().mdb_pframe_count(os.fsencode(path), C.byref(n), C.byref(last))
            if rc != 0 and not os.path.exists(path):
                raise RuntimeError("Failed to open file for append: " + path)
            self._fresh = False
        else:
            self._fresh = True

    def write_frame(self, data, frame_index: int) -> None:
        f = _as_frame(data)
        check(lib().mdb_pframe_write(os.fsencode(self.path), 0 if self._fresh else 1,
                                     frame_ptr(f), len(f), int(frame_index)))
        self._fresh = False


def nph_protocol_from_config(config) -> MDBNphProtocol:
    """NPH protocol parameters as the reference's driver derives them."""
    p = MDBNphProtocol()
    check(lib().mdb_nph_protocol_from_config(C.byref(_config_of(config)), C.byref(p)))
    return p


def nph_protocol_dry_run(protocol: MDBNphProtocol, pressures, record_cap: int = 100000):
    """The protocol's decisions for given pressures per step (no GPU):
    (result, records, chunks)."""
    p = np.ascontiguousarray(pressures, dtype=np.float64)
    recs = (MDBNphRecord * max(1, record_cap))()
    res = MDBNphResult()
    chunks = C.c_int64()
    check(lib().mdb_nph_protocol_dry_run(C.byref(protocol),
                                         p.ctypes.data_as(C.POINTER(C.c_double)), len(p),
                                         recs, record_cap, C.byref(res), C.byref(chunks)))
    return res, list(recs[:min(res.n_records, record_cap)]), chunks.value


class TrajectoryWriter:
    """Asynchronous PFRAME writer (mdb_traj_writer_*): write() queues the
    simulation's current frame and returns; a thread compresses and appends."""

    def __init__(self, path: str, append: bool = False, depth: int = 4):
        self._h = C.c_void_p()
        check(lib().mdb_traj_writer_open(os.fsencode(path), 1 if append else 0, int(depth),
                                         C.byref(self._h)))

    def write(self, sim: "MDSimulation", frame_index: int) -> None:
        check(lib().mdb_traj_writer_write(self._h, sim._h, int(frame_index)))

    def flush(self) -> None:
        check(lib().mdb_traj_writer_flush(self._h))

    def close(self) -> None:
        if self._h is not None and self._h.value:
            h, self._h = self._h, C.c_void_p()
            check(lib().mdb_traj_writer_close(h))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class FileReader:
    """FileReader (include/md_common.hpp:101-122)."""

    def __init__(self, path: str):
        self.path = path
        n = C.c_int64()
        last = C.c_uint64()
        check(lib().mdb_pframe_count(os.fsencode(path), C.byref(n), C.byref(last)))
        self.n_frames = n.value

    def read(self, frame_index: int) -> np.ndarray:
        n = C.c_int64()
        rc = lib().mdb_pframe_read(os.fsencode(self.path), int(frame_index), None, 0, C.byref(n))
        if rc not in (0, 3):
            check(rc)
        f = make_frame(n.value)
        check(lib().mdb_pframe_read(os.fsencode(self.path), int(frame_index), frame_ptr(f),
                                    n.value, C.byref(n)))
        return f


class Batch:
    """Many independent systems advanced together on one GPU: FIRE quenches
    (add_fire) or MD segments of one kind (add_md)."""

    def __init__(self, device: int = 0, skin: Optional[float] = None, use_graphs: bool = True,
                 fire_precision: Optional[int] = None, autotune: bool = False,
                 max_neighbors: Optional[int] = None, lanes: Optional[int] = None):
        self._h = C.c_void_p()
        self._opt = options(device, skin, use_graphs, max_neighbors,
                            fire_precision=fire_precision, autotune=autotune, lanes=lanes)
        check(lib().mdb_batch_create(C.byref(self._opt), C.byref(self._h)))
        self._sizes = []
        self._caps = []

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            # (no ctypes constructor here: at interpreter exit the module
            # globals may already be gone)
            self._h = None
            try:
                lib().mdb_batch_destroy(h)
            except Exception:
                pass

    def add_fire(self, config, frame, force_tol: float, max_steps: int,
                 params: FireParams) -> int:
        f = _as_frame(frame)
        sid = C.c_int32()
        p = params._c()
        check(lib().mdb_batch_add_fire(self._h, C.byref(_config_of(config)), frame_ptr(f), len(f),
                                       float(force_tol), int(max_steps), C.byref(p),
                                       C.byref(sid)))
        self._sizes.append(len(f))
        self._caps.append(max_steps // 1000 + 4)
        return sid.value

    def add_md(self, config, frame, kind: int, nsteps: int) -> int:
        """An MD segment of nsteps NVE (JOB_NVE) or Nose-Hoover (JOB_NVT) steps."""
        f = _as_frame(frame)
        sid = C.c_int32()
        check(lib().mdb_batch_add_md(self._h, C.byref(_config_of(config)), frame_ptr(f), len(f),
                                     int(kind), int(nsteps), C.byref(sid)))
        self._sizes.append(len(f))
        self._caps.append(4)
        return sid.value

    def run(self, iterations: int = -1) -> None:
        check(lib().mdb_batch_run(self._h, int(iterations)))

    def schedule(self) -> dict:
        """The engine schedule of the batch (zeros before its first run)."""
        s = _lib.MDBSchedule()
        check(lib().mdb_batch_schedule(self._h, C.byref(s)))
        return s.as_dict()

    def issue(self, iterations: int = -1) -> int:
        """Issue one chunk without waiting; returns its length."""
        k = C.c_int64()
        check(lib().mdb_batch_issue(self._h, int(iterations), C.byref(k)))
        return k.value

    def idle(self) -> bool:
        v = C.c_int32()
        check(lib().mdb_batch_query(self._h, C.byref(v)))
        return bool(v.value)

    def collect(self) -> None:
        check(lib().mdb_batch_collect(self._h))

    def done_flags(self) -> np.ndarray:
        d = np.zeros(len(self._sizes), dtype=np.int32)
        check(lib().mdb_batch_done_flags(self._h, d.ctypes.data_as(C.POINTER(C.c_int32)), len(d)))
        return d.astype(bool)

    def partial_U_lambda(self, epsilon_lambda: float) -> np.ndarray:
        """cal_partial_U_lambda of every system."""
        out = np.zeros(len(self._sizes))
        check(lib().mdb_batch_partial_U_lambda_all(self._h, float(epsilon_lambda),
                                                   out.ctypes.data_as(C.POINTER(C.c_double)),
                                                   len(out)))
        return out

    def energies(self, sys_id: int):
        """(K, U, xi) of one system."""
        K, U, xi = C.c_double(), C.c_double(), C.c_double()
        check(lib().mdb_batch_energies(self._h, sys_id, C.byref(K), C.byref(U), C.byref(xi)))
        return K.value, U.value, xi.value

    def system_info(self, sys_id: int):
        """(n, done, steps) of one system."""
        n, d, st = C.c_int64(), C.c_int32(), C.c_int64()
        check(lib().mdb_batch_system_info(self._h, sys_id, C.byref(n), C.byref(d), C.byref(st)))
        return n.value, bool(d.value), st.value

    def system_stats(self, sys_id: int):
        """(cell-list rebuilds so far, particles whose list overflowed at the
        last rebuild) of one system."""
        r, o = C.c_int64(), C.c_int32()
        check(lib().mdb_batch_system_stats(self._h, sys_id, C.byref(r), C.byref(o)))
        return r.value, o.value

    def device_bytes(self) -> int:
        b = C.c_int64()
        check(lib().mdb_batch_device_bytes(self._h, C.byref(b)))
        return b.value

    def progress(self):
        a = C.c_int32()
        b = C.c_int32()
        check(lib().mdb_batch_progress(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def frame(self, sys_id: int) -> np.ndarray:
        f = make_frame(self._sizes[sys_id])
        check(lib().mdb_batch_get_frame(self._h, sys_id, frame_ptr(f), len(f)))
        return f

    def fire_result(self, sys_id: int, with_frame: bool = True) -> MinimizeResult:
        res = MDBMinimizeResult()
        cap = self._caps[sys_id]
        es = np.zeros(cap, dtype=np.int32)
        et = np.zeros(cap, dtype=np.float64)
        check(lib().mdb_batch_get_fire_result(self._h, sys_id, C.byref(res),
                                              es.ctypes.data_as(C.POINTER(C.c_int32)),
                                              et.ctypes.data_as(C.POINTER(C.c_double)), cap))
        k = min(res.n_energy_samples, cap)
        return MinimizeResult(frame=self.frame(sys_id) if with_frame else make_frame(0),
                              energy_steps=es[:k].tolist(), energy_trace=et[:k].tolist(),
                              steps=res.steps, converged=bool(res.converged),
                              max_force=res.max_force, potential_energy=res.potential_energy,
                              nonfinite=bool(res.nonfinite))

    def cuda_stream(self) -> int:
        p = C.c_void_p()
        check(lib().mdb_batch_cuda_stream(self._h, C.byref(p)))
        return p.value or 0


def place_lpt(costs, nbins: int):
    """Greedy longest-processing-time placement (mdb_place_lpt): the bin of
    every item and the load of every bin."""
    c = np.ascontiguousarray(costs, dtype=np.float64)
    out = np.zeros(len(c), dtype=np.int32)
    load = np.zeros(nbins, dtype=np.float64)
    check(lib().mdb_place_lpt(c.ctypes.data_as(C.POINTER(C.c_double)), len(c), int(nbins),
                              out.ctypes.data_as(C.POINTER(C.c_int32)),
                              load.ctypes.data_as(C.POINTER(C.c_double))))
    return out, load


class MultiBatch:
    """Independent systems over several GPUs (mdb_multibatch_*): placed at the
    first run by longest-processing-time on particles x steps, one batch per
    device, run concurrently; a device may be listed more than once."""

    def __init__(self, devices=(0,), skin: Optional[float] = None, use_graphs: bool = True,
                 fire_precision: Optional[int] = None, autotune: bool = False):
        self._h = C.c_void_p()
        self._opt = options(0, skin, use_graphs, fire_precision=fire_precision,
                            autotune=autotune)
        dv = np.ascontiguousarray(list(devices), dtype=np.int32)
        check(lib().mdb_multibatch_create(C.byref(self._opt),
                                          dv.ctypes.data_as(C.POINTER(C.c_int32)), len(dv),
                                          C.byref(self._h)))
        self._sizes = []
        self._caps = []

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._h = None
            try:
                lib().mdb_multibatch_destroy(h)
            except Exception:
                pass

    def add_fire(self, config, frame, force_tol: float, max_steps: int,
                 params: FireParams) -> int:
        f = _as_frame(frame)
        sid = C.c_int32()
        p = params._c()
        check(lib().mdb_multibatch_add_fire(self._h, C.byref(_config_of(config)), frame_ptr(f),
                                            len(f), float(force_tol), int(max_steps),
                                            C.byref(p), C.byref(sid)))
        self._sizes.append(len(f))
        self._caps.append(max_steps // 1000 + 4)
        return sid.value

    def add_md(self, config, frame, kind: int, nsteps: int) -> int:
        f = _as_frame(frame)
        sid = C.c_int32()
        check(lib().mdb_multibatch_add_md(self._h, C.byref(_config_of(config)), frame_ptr(f),
                                          len(f), int(kind), int(nsteps), C.byref(sid)))
        self._sizes.append(len(f))
        self._caps.append(4)
        return sid.value

    def run(self, iterations: int = -1) -> None:
        check(lib().mdb_multibatch_run(self._h, int(iterations)))

    def placement(self) -> np.ndarray:
        out = np.zeros(len(self._sizes), dtype=np.int32)
        check(lib().mdb_multibatch_placement(self._h, out.ctypes.data_as(C.POINTER(C.c_int32)),
                                             len(out)))
        return out

    def progress(self):
        a, b = C.c_int32(), C.c_int32()
        check(lib().mdb_multibatch_progress(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def system_info(self, sys_id: int):
        n, d, st = C.c_int64(), C.c_int32(), C.c_int64()
        check(lib().mdb_multibatch_system_info(self._h, sys_id, C.byref(n), C.byref(d),
                                               C.byref(st)))
        return n.value, bool(d.value), st.value

    def energies(self, sys_id: int):
        K, U, xi = C.c_double(), C.c_double(), C.c_double()
        check(lib().mdb_multibatch_energies(self._h, sys_id, C.byref(K), C.byref(U),
                                            C.byref(xi)))
        return K.value, U.value, xi.value

    def frame(self, sys_id: int) -> np.ndarray:
        f = make_frame(self._sizes[sys_id])
        check(lib().mdb_multibatch_get_frame(self._h, sys_id, frame_ptr(f), len(f)))
        return f

    def fire_result(self, sys_id: int, with_frame: bool = True) -> MinimizeResult:
        res = MDBMinimizeResult()
        cap = self._caps[sys_id]
        es = np.zeros(cap, dtype=np.int32)
        et = np.zeros(cap, dtype=np.float64)
        check(lib().mdb_multibatch_get_fire_result(self._h, sys_id, C.byref(res),
                                                   es.ctypes.data_as(C.POINTER(C.c_int32)),
                                                   et.ctypes.data_as(C.POINTER(C.c_double)),
                                                   cap))
        k = min(res.n_energy_samples, cap)
        return MinimizeResult(frame=self.frame(sys_id) if with_frame else make_frame(0),
                              energy_steps=es[:k].tolist(), energy_trace=et[:k].tolist(),
                              steps=res.steps, converged=bool(res.converged),
                              max_force=res.max_force, potential_energy=res.potential_energy,
                              nonfinite=bool(res.nonfinite))


@dataclass
class RequestResult:
    """A finished request of a Server."""
    status: int
    n: int
    steps: int
    converged: bool
    nonfinite: bool
    K: float
    U: float
    xi: float
    max_force: float
    t_submit: float
    t_start: float
    t_done: float
    frame: np.ndarray = field(repr=False, default=None)

    @property
    def latency(self) -> float:
        """Seconds from submission to the result being available."""
        return self.t_done - self.t_submit


class Server:
    """Continuous batching of MD segments and FIRE quenches on one GPU
    (mdb_server_*): submit_*() queues a request and returns at once; requests
    are admitted into batches by an HBM budget as slots and memory free up,
    and run concurrently with the batches already on the device. `order`:
    ORDER_SHORTEST (default) admits the queued request with the least work
    (particles x steps) first, requests queued longer than `max_wait_ms`
    (default 60 s) ahead of all others; ORDER_FIFO admits oldest first.
    `priorities` (default on): batches holding less work get higher CUDA
    stream priority, so short requests' kernels go first."""

    def __init__(self, device: int = 0, max_active_batches: Optional[int] = None,
                 hbm_budget_bytes: Optional[int] = None, max_batch_particles: Optional[int] = None,
                 max_batch_systems: Optional[int] = None, chunk: Optional[int] = None,
                 skin: Optional[float] = None, use_graphs: bool = True,
                 order: Optional[int] = None, max_wait_ms: Optional[int] = None,
                 priorities: Optional[bool] = None):
        self._h = C.c_void_p()
        o = MDBServerOptions()
        lib().mdb_server_options_default(C.byref(o))
        o.device = device
        for name, v in (("max_active_batches", max_active_batches),
                        ("hbm_budget_bytes", hbm_budget_bytes),
                        ("max_batch_particles", max_batch_particles),
                        ("max_batch_systems", max_batch_systems), ("chunk", chunk),
                        ("skin", skin), ("order", order), ("max_wait_ms", max_wait_ms),
                        ("priorities", None if priorities is None else int(bool(priorities)))):
            if v is not None:
                setattr(o, name, v)
        o.use_graphs = 1 if use_graphs else 0
        check(lib().mdb_server_create(C.byref(o), C.byref(self._h)))
        self._n = {}

    def close(self) -> None:
        if self._h is not None and self._h.value:
            lib().mdb_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _submit(self, config, frame, req: MDBRequest) -> int:
        f = _as_frame(frame)
        rid = C.c_int64()
        check(lib().mdb_server_submit(self._h, C.byref(_config_of(config)), frame_ptr(f), len(f),
                                      C.byref(req), C.byref(rid)))
        self._n[rid.value] = len(f)
        return rid.value

    def submit_md(self, config, frame, nsteps: int, nose_hoover: bool = True) -> int:
        req = MDBRequest()
        req.kind = JOB_NVT if nose_hoover else JOB_NVE
        req.nsteps = int(nsteps)
        return self._submit(config, frame, req)

    def submit_fire(self, config, frame, force_tol: float, max_steps: int,
                    params: "FireParams") -> int:
        req = MDBRequest()
        req.kind = JOB_FIRE
        req.max_steps = int(max_steps)
        req.force_tol = float(force_tol)
        req.fire = params._c()
        return self._submit(config, frame, req)

    def wait(self, rid: int, timeout: float = -1.0) -> int:
        """Waits for a request (timeout < 0: no limit); returns its status."""
        info = MDBRequestResult()
        check(lib().mdb_server_wait(self._h, rid, float(timeout), C.byref(info)))
        return info.status

    def result(self, rid: int) -> RequestResult:
        """The result of a finished request (raises for a failed one); releases it."""
        n = self._n[rid]
        f = make_frame(n)
        info = MDBRequestResult()
        try:
            check(lib().mdb_server_result(self._h, rid, frame_ptr(f), n, C.byref(info)))
        finally:
            if info.status in (REQ_DONE, REQ_FAILED):
                self._n.pop(rid, None)
        return RequestResult(status=info.status, n=info.n, steps=info.steps,
                             converged=bool(info.converged), nonfinite=bool(info.nonfinite),
                             K=info.K, U=info.U, xi=info.xi, max_force=info.max_force,
                             t_submit=info.t_submit, t_start=info.t_start, t_done=info.t_done,
                             frame=f)

    def stats(self) -> MDBServerStats:
        st = MDBServerStats()
        check(lib().mdb_server_stats(self._h, C.byref(st)))
        return st


def compute_forces(config, frame, Lx: float, Ly: float, periodic_y: bool = True,
                   device: int = 0, skin: Optional[float] = None,
                   max_neighbors: Optional[int] = None):
    """One force evaluation: (acc[n,2], U, W)."""
    f = _as_frame(frame)
    n = len(f)
    acc = np.zeros((n, 2))
    U = C.c_double()
    W = C.c_double()
    opt = options(device, skin, True, max_neighbors)
    check(lib().mdb_compute_forces(C.byref(_config_of(config)), frame_ptr(f), n, float(Lx),
                                   float(Ly), 1 if periodic_y else 0, C.byref(opt),
                                   acc.ctypes.data_as(C.POINTER(C.c_double)), C.byref(U),
                                   C.byref(W)))
    return acc, U.value, W.value


def cell_build(pos, Lx: float, Ly: float, cell_min: float, device: int = 0):
    """GPU cell binning: (cell ids, stable permutation, ncx, ncy)."""
    p = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 2)
    n = p.shape[0]
    cell = np.zeros(n, dtype=np.int32)
    perm = np.zeros(n, dtype=np.int32)
    ncx = C.c_int32()
    ncy = C.c_int32()
    check(lib().mdb_cell_build(p.ctypes.data_as(C.POINTER(C.c_double)), n, float(Lx), float(Ly),
                               float(cell_min), device,
                               cell.ctypes.data_as(C.POINTER(C.c_int32)),
                               perm.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(ncx),
                               C.byref(ncy)))
    return cell, perm, ncx.value, ncy.value


def kernel_launches() -> int:
    return int(lib().mdb_kernel_launches())
