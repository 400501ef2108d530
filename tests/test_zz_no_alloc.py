"""mdb_compute_forces_noalloc (device buffers in, device buffers out, scratch in
a fixed device array) against mdb_compute_forces on the same frames.

Tolerances are those of the force parity tests: relative L2 1e-5 on the
accelerations, relative 1e-6 on U and W. Several calls run back to back on one
stream, so each call must start from a cleared scratch array.
"""
import ctypes as C

import numpy as np
import pytest

import md_simulation_cuda_b200 as mdb
from md_simulation_cuda_b200 import _lib
from md_simulation_cuda_b200 import workloads as wl
from tests.helpers import rel_err, rel_l2

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5


def _noalloc(cfg, frame, Lx, Ly, periodic_y=True):
    import torch

    dev = torch.device("cuda", 0)
    pos = torch.from_numpy(np.ascontiguousarray(frame["pos"], dtype=np.float64)).to(dev)
    typ = torch.from_numpy(np.ascontiguousarray(frame["type"], dtype=np.int32)).to(dev)
    n = len(frame)
    acc = torch.full((n, 2), float("nan"), dtype=torch.float64, device=dev)
    uw = torch.full((2,), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    rc = _lib.lib().mdb_compute_forces_noalloc(
        C.byref(mdb._config_of(cfg)), C.c_void_p(pos.data_ptr()), C.c_void_p(typ.data_ptr()), n,
        float(Lx), float(Ly), 1 if periodic_y else 0, C.c_void_p(stream.cuda_stream),
        C.c_void_p(acc.data_ptr()), C.c_void_p(uw.data_ptr()))
    assert rc == _lib.MDB_OK, _lib.last_error()
    stream.synchronize()
    a = acc.cpu().numpy()
    u, w = uw.cpu().numpy().tolist()
    return a, u, w


def _check(cfg, frame, Lx, Ly, periodic_y=True):
    a, u, w = _noalloc(cfg, frame, Lx, Ly, periodic_y)
    ref, U0, W0 = mdb.compute_forces(cfg, frame, Lx, Ly, periodic_y=periodic_y)
    assert np.all(np.isfinite(a))
    assert rel_l2(a, ref) <= FORCE_TOL
    assert rel_err(u, U0) <= 1e-6
    assert rel_err(w, W0) <= 1e-6
    return a, u, w


def test_noalloc_matches_compute_forces_two_calls(built):
    f1, cfg1 = wl.nve_4096()
    L1 = (cfg1["box_w_global"], cfg1["box_h_global"])
    f2, Lx2, Ly2 = wl.lattice_frame(5000, 0.85, 0.5, 0.5, 1.0, seed=2, jitter=0.15)
    cfg2 = wl.config_dict(5000, Lx2, Ly2, dt=0.001)
    first = _check(cfg1, f1, *L1)
    _check(cfg2, f2, Lx2, Ly2)  # a different frame right after
    again = _check(cfg1, f1, *L1)  # and the first one again
    assert np.array_equal(first[0], again[0])  # deterministic
    assert first[1] == again[1] and first[2] == again[2]


def test_noalloc_walls_small_box_and_other_types(built):
    f, Lx, Ly = wl.lattice_frame(3000, 0.8, 2.0, 0.65, 1.0, seed=9)
    cfg = wl.config_dict(3000, Lx, Ly, dt=0.001)
    _check(cfg, f, Lx, Ly, periodic_y=False)
    rng = np.random.default_rng(3)
    L = 6.0
    g = mdb.make_frame(24)
    g["pos"] = rng.uniform(0, L, (24, 2))
    g["type"] = rng.integers(0, 2, 24)
    _check(wl.config_dict(24, L, L, dt=0.001), g, L, L)
    h, Lx, Ly = wl.lattice_frame(1500, 0.8, 1.0, 0.5, 1.0, seed=7)
    h["type"] = rng.integers(0, 4, len(h))
    _check(wl.config_dict(len(h), Lx, Ly, dt=0.001, MASS_B=2.0), h, Lx, Ly)


def test_noalloc_rejects_sizes_beyond_the_maximum(built):
    import torch

    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    cfg = mdb._config_of(wl.config_dict(4, 10.0, 10.0, dt=0.001))
    rc = _lib.lib().mdb_compute_forces_noalloc(C.byref(cfg), p, p, 65537, 10.0, 10.0, 1, None, p,
                                               p)
    assert rc == _lib.MDB_ERR_CAPACITY
    assert "MDB_NOALLOC_MAX_PARTICLES" in _lib.last_error()
