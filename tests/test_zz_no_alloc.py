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


def test_noalloc_against_fp64_oracle(built):
    """The entry point checked on its own: accelerations, U and W against the
    FP64 oracle, periodic and walled in y."""
    from oracle import pyoracle as po

    f, cfg = wl.nve_4096(seed=11)
    Lx, Ly = cfg["box_w_global"], cfg["box_h_global"]
    for periodic_y in (True, False):
        a, u, w = _noalloc(cfg, f, Lx, Ly, periodic_y)
        ref, U0, W0 = po.forces(cfg, f["pos"], f["type"], Lx, Ly, mode=po.OR_FP64,
                                periodic_y=1 if periodic_y else 0)
        assert rel_l2(a, ref) <= FORCE_TOL
        assert rel_err(u, U0) <= 1e-6
        assert rel_err(w, W0) <= 1e-6


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


def test_noalloc_empty_frame_writes_zero_energies(built):
    """n = 0: nothing to evaluate, U and W are written as 0."""
    import torch

    uw = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    cfg = mdb._config_of(wl.config_dict(1, 10.0, 10.0, dt=0.001))
    rc = _lib.lib().mdb_compute_forces_noalloc(C.byref(cfg), None, None, 0, 10.0, 10.0, 1, None,
                                               None, C.c_void_p(uw.data_ptr()))
    assert rc == _lib.MDB_OK, _lib.last_error()
    torch.cuda.synchronize()
    assert uw.cpu().numpy().tolist() == [0.0, 0.0]


def test_noalloc_streams_ordered_by_an_event(built):
    """Two calls on two streams, the second waiting on an event recorded after
    the first: the same results as two calls on one stream."""
    import torch

    f1, cfg1 = wl.nve_4096(seed=4)
    f2, cfg2 = wl.nve_4096(seed=6)
    ref1 = _noalloc(cfg1, f1, cfg1["box_w_global"], cfg1["box_h_global"])
    ref2 = _noalloc(cfg2, f2, cfg2["box_w_global"], cfg2["box_h_global"])
    dev = torch.device("cuda", 0)
    s1, s2 = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    outs = []
    ev = torch.cuda.Event()
    for k, (f, cfg, st) in enumerate(((f1, cfg1, s1), (f2, cfg2, s2))):
        pos = torch.from_numpy(np.ascontiguousarray(f["pos"])).to(dev)
        typ = torch.from_numpy(np.ascontiguousarray(f["type"], dtype=np.int32)).to(dev)
        acc = torch.full((len(f), 2), float("nan"), dtype=torch.float64, device=dev)
        uw = torch.full((2,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        if k == 1:
            st.wait_event(ev)
        rc = _lib.lib().mdb_compute_forces_noalloc(
            C.byref(mdb._config_of(cfg)), C.c_void_p(pos.data_ptr()),
            C.c_void_p(typ.data_ptr()), len(f), cfg["box_w_global"], cfg["box_h_global"], 1,
            C.c_void_p(st.cuda_stream), C.c_void_p(acc.data_ptr()), C.c_void_p(uw.data_ptr()))
        assert rc == _lib.MDB_OK, _lib.last_error()
        if k == 0:
            ev.record(st)
        outs.append((acc, uw, pos, typ))
    torch.cuda.synchronize(dev)
    for (acc, uw, _, _), ref in zip(outs, (ref1, ref2)):
        assert np.array_equal(acc.cpu().numpy(), ref[0])
        assert uw.cpu().numpy().tolist() == [ref[1], ref[2]]


def test_noalloc_allocates_nothing(built):
    """Warm calls leave the device's free memory unchanged."""
    import torch

    f, cfg = wl.nve_4096(seed=2)
    L = cfg["box_w_global"]
    _noalloc(cfg, f, L, L)  # warm: device set-up, torch's own buffers
    dev = torch.device("cuda", 0)
    pos = torch.from_numpy(np.ascontiguousarray(f["pos"])).to(dev)
    typ = torch.from_numpy(np.ascontiguousarray(f["type"], dtype=np.int32)).to(dev)
    acc = torch.empty((len(f), 2), dtype=torch.float64, device=dev)
    uw = torch.empty((2,), dtype=torch.float64, device=dev)
    c = mdb._config_of(cfg)
    torch.cuda.synchronize(dev)
    free0, _ = torch.cuda.mem_get_info(dev)
    for _ in range(5):
        rc = _lib.lib().mdb_compute_forces_noalloc(
            C.byref(c), C.c_void_p(pos.data_ptr()), C.c_void_p(typ.data_ptr()), len(f), L, L, 1,
            None, C.c_void_p(acc.data_ptr()), C.c_void_p(uw.data_ptr()))
        assert rc == _lib.MDB_OK, _lib.last_error()
    torch.cuda.synchronize(dev)
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0
