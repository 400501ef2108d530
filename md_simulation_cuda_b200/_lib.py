"""ctypes binding of libmdb200.so (the C ABI declared in include/mdb200.h).

The shared library is built in-tree (``md_simulation_cuda_b200/libmdb200.so``)
by ``md_simulation_cuda_b200.build.build()``. Loading fails loudly when it is
missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmdb200.so")

MDB_OK = 0
MDB_ERR_CONFIG = 1
MDB_ERR_ARG = 2
MDB_ERR_CAPACITY = 3
MDB_ERR_NONFINITE = 4
MDB_ERR_BOX = 5
MDB_ERR_CUDA = 6
MDB_ERR_IO = 7
MDB_ERR_STATE = 8
MDB_ERR_NODEVICE = 9

# Particle (include/md_particle.hpp:31-38): 64 bytes.
PARTICLE_DTYPE = np.dtype({
    "names": ["pos", "vel", "acc", "type", "_pad", "theta"],
    "formats": [("<f8", (2,)), ("<f8", (2,)), ("<f8", (2,)), "<i4", "<i4", "<f8"],
    "offsets": [0, 16, 32, 48, 52, 56],
    "itemsize": 64,
})


class MDBError(RuntimeError):
    """A non-zero status from libmdb200; ``code`` is the MDB_ERR_* value."""

    def __init__(self, code, message):
        super().__init__(f"[mdb200 error {code}] {message}")
        self.code = code


class MDBConfigC(C.Structure):
    _fields_ = [
        ("n_particles_global", C.c_int32),
        ("n_particles_type0", C.c_int32),
        ("box_w_global", C.c_double),
        ("box_h_global", C.c_double),
        ("T_init", C.c_double),
        ("T_target", C.c_double),
        ("SIGMA_AA", C.c_double), ("SIGMA_BB", C.c_double), ("SIGMA_AB", C.c_double),
        ("EPSILON_AA", C.c_double), ("EPSILON_BB", C.c_double), ("EPSILON_AB", C.c_double),
        ("MASS_A", C.c_double), ("MASS_B", C.c_double),
        ("devide_p", C.c_double),
        ("dt", C.c_double),
        ("Q", C.c_double),
        ("save_dt_interval", C.c_double),
        ("cutoff", C.c_double),
        ("run_name", C.c_char * 256),
        ("load_name", C.c_char * 256),
        ("THREADS_PER_BLOCK", C.c_int32),
        ("rank_size", C.c_int32),
        ("mu", C.c_double), ("v0", C.c_double), ("D_r", C.c_double), ("D_theta", C.c_double),
        ("barostat_mass", C.c_double),
        ("k_piston", C.c_double),
        ("barostat_area_rate_init", C.c_double),
        ("barostat_height_min_ratio", C.c_double),
        ("barostat_height_max_ratio", C.c_double),
        ("pressure_target_mode", C.c_char * 64),
        ("P_target", C.c_double),
        ("pressure_target_auto_steps", C.c_int32),
        ("pressure_eval_interval_steps", C.c_int32),
        ("pressure_window_samples", C.c_int32),
        ("pressure_tolerance_rel", C.c_double),
        ("pressure_stable_required_windows", C.c_int32),
        ("nph_warmup_min_steps", C.c_int32),
        ("nph_warmup_max_steps", C.c_int32),
        ("nph_steps", C.c_int32),
        ("rank_idx", C.c_int32),
        ("n_local", C.c_int32),
        ("n_halo_left", C.c_int32),
        ("n_halo_right", C.c_int32),
        ("n_cap", C.c_int32),
        ("halo_left_cap", C.c_int32),
        ("halo_right_cap", C.c_int32),
        ("left_rank", C.c_int32),
        ("right_rank", C.c_int32),
        ("x_min", C.c_double),
        ("x_max", C.c_double),
    ]


class MDBOptions(C.Structure):
    _fields_ = [
        ("device", C.c_int32),
        ("skin", C.c_double),
        ("use_graphs", C.c_int32),
        ("max_neighbors", C.c_int32),
        ("stream_priority", C.c_int32),
        ("fire_precision", C.c_int32),
        ("autotune", C.c_int32),
        ("step_kernel", C.c_int32),
        ("lanes", C.c_int32),
        ("reserved", C.c_int32 * 7),
    ]


class MDBSchedule(C.Structure):
    _fields_ = [
        ("list_prefetch_rows", C.c_int32),
        ("nlist_grid", C.c_int32),
        ("rebuild_grid", C.c_int32),
        ("items", C.c_int32),
        ("tuned", C.c_int32),
        ("from_cache", C.c_int32),
        ("skin", C.c_double),
        ("tune_ms", C.c_double),
        ("multi_step", C.c_int32),
        ("multi_step_blocks", C.c_int32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class MDBObservables(C.Structure):
    _fields_ = [
        ("t", C.c_double),
        ("Lx", C.c_double),
        ("Ly", C.c_double),
        ("xi", C.c_double),
        ("last_instant_pressure", C.c_double),
        ("nph_area_momentum", C.c_double),
        ("nph_area_rate", C.c_double),
        ("nph_piston_velocity", C.c_double),
        ("nph_piston_force", C.c_double),
        ("n", C.c_int64),
        ("steps", C.c_int64),
        ("rebuilds", C.c_int64),
        ("piston_mode_active", C.c_int32),
        ("nonfinite", C.c_int32),
    ]


class MDBFireParams(C.Structure):
    _fields_ = [
        ("dt_init", C.c_double),
        ("dt_max", C.c_double),
        ("alpha0", C.c_double),
        ("f_inc", C.c_double),
        ("f_dec", C.c_double),
        ("N_min", C.c_int32),
        ("_pad", C.c_int32),
    ]


class MDBMinimizeResult(C.Structure):
    _fields_ = [
        ("steps", C.c_int32),
        ("converged", C.c_int32),
        ("max_force", C.c_double),
        ("potential_energy", C.c_double),
        ("n_energy_samples", C.c_int64),
        ("nonfinite", C.c_int32),
        ("_pad", C.c_int32),
    ]


class MDBServerOptions(C.Structure):
    _fields_ = [
        ("device", C.c_int32),
        ("max_active_batches", C.c_int32),
        ("hbm_budget_bytes", C.c_int64),
        ("max_batch_particles", C.c_int64),
        ("max_batch_systems", C.c_int32),
        ("chunk", C.c_int32),
        ("skin", C.c_double),
        ("use_graphs", C.c_int32),
        ("max_neighbors", C.c_int32),
        ("order", C.c_int32),
        ("max_wait_ms", C.c_int32),
        ("priorities", C.c_int32),
        ("reserved", C.c_int32 * 5),
    ]


class MDBRequest(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("max_steps", C.c_int32),
        ("nsteps", C.c_int64),
        ("force_tol", C.c_double),
        ("fire", MDBFireParams),
    ]


class MDBRequestResult(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("error", C.c_int32),
        ("n", C.c_int64),
        ("steps", C.c_int64),
        ("converged", C.c_int32),
        ("nonfinite", C.c_int32),
        ("K", C.c_double),
        ("U", C.c_double),
        ("xi", C.c_double),
        ("max_force", C.c_double),
        ("t_submit", C.c_double),
        ("t_start", C.c_double),
        ("t_done", C.c_double),
    ]


class MDBServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_int64), ("queued", C.c_int64), ("running", C.c_int64),
        ("finished", C.c_int64), ("failed", C.c_int64),
        ("batches_admitted", C.c_int64), ("active_batches", C.c_int64),
        ("device_bytes", C.c_int64), ("hbm_budget_bytes", C.c_int64),
        ("particle_steps", C.c_double), ("elapsed_s", C.c_double),
    ]


class MDBNphProtocol(C.Structure):
    _fields_ = [
        ("auto_target", C.c_int32), ("_pad0", C.c_int32), ("P_target", C.c_double),
        ("auto_steps", C.c_int32), ("eval_interval", C.c_int32),
        ("window_samples", C.c_int32), ("stable_required", C.c_int32),
        ("warmup_min_steps", C.c_int32), ("warmup_max_steps", C.c_int32),
        ("production_steps", C.c_int32), ("_pad1", C.c_int32),
        ("tolerance_rel", C.c_double), ("host_driven", C.c_int32),
        ("reserved", C.c_int32 * 7),
    ]


class MDBNphRecord(C.Structure):
    _fields_ = [
        ("step", C.c_int64), ("t", C.c_double), ("phase", C.c_int32), ("_pad", C.c_int32),
        ("P_inst", C.c_double), ("P_target", C.c_double), ("mean", C.c_double),
        ("stddev", C.c_double), ("rel_err", C.c_double), ("Lx", C.c_double),
        ("Ly", C.c_double), ("dA_dt", C.c_double),
    ]


class MDBNphResult(C.Structure):
    _fields_ = [
        ("P_target", C.c_double), ("auto_end_step", C.c_int64),
        ("warmup_end_step", C.c_int64), ("total_steps", C.c_int64),
        ("n_records", C.c_int64), ("forced_switch", C.c_int32), ("finished", C.c_int32),
        ("host_waits", C.c_int64),
    ]


_lib = None
_lock = threading.Lock()

# (name, argtypes, restype) of every exported symbol; restype None means int.
_vp = C.c_void_p
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_cfgp = C.POINTER(MDBConfigC)
_optp = C.POINTER(MDBOptions)
SIGNATURES = {
    "mdb_config_default": ([_cfgp], C.c_int),
    "mdb_config_from_json": ([C.c_char_p, _cfgp], C.c_int),
    "mdb_config_from_json_file": ([C.c_char_p, _cfgp], C.c_int),
    "mdb_config_to_json": ([_cfgp, C.c_int32, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)], C.c_int),
    "mdb_config_apply_override": ([_cfgp, C.c_char_p, C.c_char_p], C.c_int),
    "mdb_parse_override_argument": ([C.c_char_p, C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t], C.c_int),
    "mdb_options_default": ([_optp], None),
    "mdb_pframe_write": ([C.c_char_p, C.c_int32, _vp, C.c_int64, C.c_uint64], C.c_int),
    "mdb_pframe_read": ([C.c_char_p, C.c_uint64, _vp, C.c_int64, C.POINTER(C.c_int64)], C.c_int),
    "mdb_pframe_count": ([C.c_char_p, C.POINTER(C.c_int64), C.POINTER(C.c_uint64)], C.c_int),
    "mdb_sim_create": ([_cfgp, _vp, C.c_int64, _optp, C.POINTER(_vp)], C.c_int),
    "mdb_sim_create_from_pframe": ([_cfgp, C.c_char_p, C.c_uint64, _optp, C.POINTER(_vp)], C.c_int),
    "mdb_sim_destroy": ([_vp], C.c_int),
    "mdb_sim_step_nve": ([_vp, C.c_int64], C.c_int),
    "mdb_sim_step_nose_hoover": ([_vp, C.c_int64, C.c_int32], C.c_int),
    "mdb_sim_step_nph": ([_vp, C.c_double, C.c_int64], C.c_int),
    "mdb_sim_step_nph_piston": ([_vp, C.c_double, C.c_int64], C.c_int),
    "mdb_sim_total_K": ([_vp, _dp], C.c_int),
    "mdb_sim_total_U": ([_vp, _dp], C.c_int),
    "mdb_sim_instant_pressure": ([_vp, _dp], C.c_int),
    "mdb_sim_partial_U_lambda": ([_vp, C.c_double, _dp], C.c_int),
    "mdb_sim_n_profile": ([_vp, C.c_int32, _ip], C.c_int),
    "mdb_sim_density_profile": ([_vp, C.c_int32, _dp], C.c_int),
    "mdb_sim_pressure_profile": ([_vp, C.c_int32, _dp], C.c_int),
    "mdb_sim_observables": ([_vp, C.POINTER(MDBObservables)], C.c_int),
    "mdb_sim_observables_async": ([_vp, _vp], C.c_int),
    "mdb_sim_get_frame": ([_vp, _vp, C.c_int64], C.c_int),
    "mdb_sim_set_frame": ([_vp, _vp, C.c_int64], C.c_int),
    "mdb_sim_save_pframe": ([_vp, C.c_char_p, C.c_uint64], C.c_int),
    "mdb_sim_get_config": ([_vp, _cfgp], C.c_int),
    "mdb_sim_save_checkpoint": ([_vp, C.c_char_p, C.c_uint64, C.c_char_p], C.c_int),
    "mdb_sim_create_from_checkpoint": ([_cfgp, C.c_char_p, C.c_uint64, C.c_char_p, _optp,
                                        C.POINTER(_vp)], C.c_int),
    "mdb_traj_writer_open": ([C.c_char_p, C.c_int32, C.c_int32, C.POINTER(_vp)], C.c_int),
    "mdb_traj_writer_write": ([_vp, _vp, C.c_uint64], C.c_int),
    "mdb_traj_writer_flush": ([_vp], C.c_int),
    "mdb_traj_writer_close": ([_vp], C.c_int),
    "mdb_sim_cuda_stream": ([_vp, C.POINTER(_vp)], C.c_int),
    "mdb_sim_synchronize": ([_vp], C.c_int),
    "mdb_sim_phase_times": ([_vp, C.c_int32, C.c_int64, _dp], C.c_int),
    "mdb_sim_schedule": ([_vp, C.POINTER(MDBSchedule)], C.c_int),
    "mdb_fire_params_from_config": ([_cfgp, C.POINTER(MDBFireParams)], C.c_int),
    "mdb_fire_minimize": ([_cfgp, _vp, C.c_int64, C.c_double, C.c_int32, C.POINTER(MDBFireParams),
                           _optp, _vp, C.POINTER(MDBMinimizeResult), _ip, _dp, C.c_int64], C.c_int),
    "mdb_batch_create": ([_optp, C.POINTER(_vp)], C.c_int),
    "mdb_batch_destroy": ([_vp], C.c_int),
    "mdb_batch_add_fire": ([_vp, _cfgp, _vp, C.c_int64, C.c_double, C.c_int32,
                            C.POINTER(MDBFireParams), _ip], C.c_int),
    "mdb_batch_add_md": ([_vp, _cfgp, _vp, C.c_int64, C.c_int32, C.c_int64, _ip], C.c_int),
    "mdb_batch_run": ([_vp, C.c_int64], C.c_int),
    "mdb_batch_progress": ([_vp, _ip, _ip], C.c_int),
    "mdb_batch_system_info": ([_vp, C.c_int32, C.POINTER(C.c_int64), _ip, C.POINTER(C.c_int64)], C.c_int),
    "mdb_batch_system_stats": ([_vp, C.c_int32, C.POINTER(C.c_int64), _ip], C.c_int),
    "mdb_batch_get_frame": ([_vp, C.c_int32, _vp, C.c_int64], C.c_int),
    "mdb_batch_get_fire_result": ([_vp, C.c_int32, C.POINTER(MDBMinimizeResult), _ip, _dp, C.c_int64], C.c_int),
    "mdb_batch_energies": ([_vp, C.c_int32, _dp, _dp, _dp], C.c_int),
    "mdb_batch_energies_all": ([_vp, _dp, _dp, _dp, C.c_int32], C.c_int),
    "mdb_batch_issue": ([_vp, C.c_int64, C.POINTER(C.c_int64)], C.c_int),
    "mdb_batch_query": ([_vp, _ip], C.c_int),
    "mdb_batch_collect": ([_vp], C.c_int),
    "mdb_batch_done_flags": ([_vp, _ip, C.c_int32], C.c_int),
    "mdb_batch_partial_U_lambda_all": ([_vp, C.c_double, _dp, C.c_int32], C.c_int),
    "mdb_batch_device_bytes": ([_vp, C.POINTER(C.c_int64)], C.c_int),
    "mdb_batch_schedule": ([_vp, C.POINTER(MDBSchedule)], C.c_int),
    "mdb_place_lpt": ([_dp, C.c_int32, C.c_int32, _ip, _dp], C.c_int),
    "mdb_multibatch_create": ([_optp, _ip, C.c_int32, C.POINTER(_vp)], C.c_int),
    "mdb_multibatch_destroy": ([_vp], C.c_int),
    "mdb_multibatch_add_fire": ([_vp, _cfgp, _vp, C.c_int64, C.c_double, C.c_int32,
                                 C.POINTER(MDBFireParams), _ip], C.c_int),
    "mdb_multibatch_add_md": ([_vp, _cfgp, _vp, C.c_int64, C.c_int32, C.c_int64, _ip], C.c_int),
    "mdb_multibatch_run": ([_vp, C.c_int64], C.c_int),
    "mdb_multibatch_placement": ([_vp, _ip, C.c_int32], C.c_int),
    "mdb_multibatch_progress": ([_vp, _ip, _ip], C.c_int),
    "mdb_multibatch_system_info": ([_vp, C.c_int32, C.POINTER(C.c_int64), _ip,
                                    C.POINTER(C.c_int64)], C.c_int),
    "mdb_multibatch_get_frame": ([_vp, C.c_int32, _vp, C.c_int64], C.c_int),
    "mdb_multibatch_get_fire_result": ([_vp, C.c_int32, C.POINTER(MDBMinimizeResult), _ip, _dp,
                                        C.c_int64], C.c_int),
    "mdb_multibatch_energies": ([_vp, C.c_int32, _dp, _dp, _dp], C.c_int),
    "mdb_batch_cuda_stream": ([_vp, C.POINTER(_vp)], C.c_int),
    "mdb_server_options_default": ([C.POINTER(MDBServerOptions)], None),
    "mdb_server_create": ([C.POINTER(MDBServerOptions), C.POINTER(_vp)], C.c_int),
    "mdb_server_destroy": ([_vp], C.c_int),
    "mdb_server_submit": ([_vp, _cfgp, _vp, C.c_int64, C.POINTER(MDBRequest),
                           C.POINTER(C.c_int64)], C.c_int),
    "mdb_server_wait": ([_vp, C.c_int64, C.c_double, C.POINTER(MDBRequestResult)], C.c_int),
    "mdb_server_result": ([_vp, C.c_int64, _vp, C.c_int64, C.POINTER(MDBRequestResult)],
                          C.c_int),
    "mdb_server_stats": ([_vp, C.POINTER(MDBServerStats)], C.c_int),
    "mdb_compute_forces": ([_cfgp, _vp, C.c_int64, C.c_double, C.c_double, C.c_int32, _optp, _dp,
                            _dp, _dp], C.c_int),
    "mdb_cell_build": ([_dp, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_int32, _ip, _ip,
                        _ip, _ip], C.c_int),
    "mdb_compute_forces_noalloc": ([_cfgp, _vp, _vp, C.c_int64, C.c_double, C.c_double, C.c_int32,
                                    _vp, _vp, _vp], C.c_int),
    "mdb_nph_protocol_from_config": ([_cfgp, C.POINTER(MDBNphProtocol)], C.c_int),
    "mdb_sim_run_nph_protocol": ([_vp, C.POINTER(MDBNphProtocol), C.POINTER(MDBNphRecord),
                                  C.c_int64, C.POINTER(MDBNphResult)], C.c_int),
    "mdb_nph_protocol_dry_run": ([C.POINTER(MDBNphProtocol), _dp, C.c_int64,
                                  C.POINTER(MDBNphRecord), C.c_int64, C.POINTER(MDBNphResult),
                                  C.POINTER(C.c_int64)], C.c_int),
    "mdb_last_error": ([C.c_char_p, C.c_size_t], C.c_int),
    "mdb_version": ([], C.c_char_p),
    "mdb_kernel_launches": ([], C.c_int64),
}


def lib():
    """Load libmdb200.so (raises if it has not been built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"libmdb200.so not found at {LIB_PATH}; build it with "
                    "`python -c 'import md_simulation_cuda_b200.build as b; b.build()'`")
            L = C.CDLL(LIB_PATH)
            for name, (argt, rest) in SIGNATURES.items():
                fn = getattr(L, name)
                fn.argtypes = argt
                fn.restype = rest
            _lib = L
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(4096)
    lib().mdb_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int):
    if rc != MDB_OK:
        raise MDBError(rc, last_error())
    return rc


FIRE_AUTO, FIRE_FP32, FIRE_FP64 = 0, 1, 2
STEPS_AUTO, STEPS_PER_PHASE, STEPS_MULTI = 0, 1, 2
LANES_AUTO, LANES_ONE, LANES_SPLIT = 0, 1, 4


def options(device=0, skin=None, use_graphs=True, max_neighbors=None,
            fire_precision=None, autotune=None, step_kernel=None, lanes=None) -> MDBOptions:
    o = MDBOptions()
    lib().mdb_options_default(C.byref(o))
    o.device = device
    if lanes is not None:
        o.lanes = int(lanes)
    if step_kernel is not None:
        o.step_kernel = int(step_kernel)
    if autotune is not None:
        o.autotune = 1 if autotune else 0
    if fire_precision is not None:
        o.fire_precision = int(fire_precision)
    if skin is not None:
        o.skin = float(skin)
    o.use_graphs = 1 if use_graphs else 0
    if max_neighbors is not None:
        o.max_neighbors = int(max_neighbors)
    return o


def frame_ptr(frame: np.ndarray):
    if frame.dtype != PARTICLE_DTYPE or not frame.flags["C_CONTIGUOUS"]:
        raise TypeError("frame must be a C-contiguous array of PARTICLE_DTYPE")
    return C.c_void_p(frame.ctypes.data)
