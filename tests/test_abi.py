"""The C ABI library loads without a GPU and exports every function that
include/mdb200.h declares; the ctypes mirror binds each of them."""
import ctypes as C
import os
import re

import md_simulation_cuda_b200 as mdb
from md_simulation_cuda_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "mdb200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mdb_[A-Za-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported(built):
    names = _declared()
    assert len(names) >= 40
    L = C.CDLL(_lib.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_ctypes_mirror_covers_header(built):
    assert set(_declared()) == set(_lib.SIGNATURES)


def test_struct_layouts(built):
    assert mdb.PARTICLE_DTYPE.itemsize == 64
    assert mdb.PARTICLE_DTYPE.fields["type"][1] == 48
    assert mdb.PARTICLE_DTYPE.fields["theta"][1] == 56
    assert C.sizeof(_lib.MDBConfigC) > 700


def test_errors_are_status_codes_without_gpu(built):
    """Without a CUDA device every GPU entry point returns a status (never
    exits); CPU entry points work."""
    L = _lib.lib()
    cfg = _lib.MDBConfigC()
    assert L.mdb_config_default(C.byref(cfg)) == 0
    h = C.c_void_p()
    f = mdb.make_frame(4)
    rc = L.mdb_sim_create(C.byref(cfg), _lib.frame_ptr(f), 4, None, C.byref(h))
    if not os.environ.get("CUDA_VISIBLE_DEVICES_FOR_TESTS"):
        assert rc != 0 or h.value  # created on a GPU box, a status here
    assert L.mdb_sim_step_nve(None, 1) == _lib.MDB_ERR_ARG
    assert "bad arguments" in _lib.last_error()
    assert L.mdb_version().startswith(b"mdb200")


def test_batch_kinds_cannot_mix_without_gpu(built):
    """Adding systems only stores them (no device work): a batch holds one job
    kind, and MD segments need a positive length."""
    import md_simulation_cuda_b200 as m
    from md_simulation_cuda_b200 import workloads as wl

    f, L = wl.random_frame(50, 0.7, 0.5, 3)
    cfg = wl.config_dict(50, L, L, dt=0.001, T=0.0)
    b = m.Batch()
    b.add_md(cfg, f, m.JOB_NVT, 10)
    try:
        b.add_fire(cfg, f, 1e-4, 100, m.FireParams.from_config(cfg))
        raise AssertionError("mixed kinds accepted")
    except m.MDBError as e:
        assert e.code == _lib.MDB_ERR_STATE
    try:
        b.add_md(cfg, f, m.JOB_NVT, 0)
        raise AssertionError("zero-length segment accepted")
    except m.MDBError as e:
        assert e.code == _lib.MDB_ERR_ARG


def test_server_needs_a_device(built):
    import torch

    import md_simulation_cuda_b200 as m

    if torch.cuda.is_available():
        return  # the GPU server tests cover this case
    try:
        m.Server()
        raise AssertionError("server created without a device")
    except m.MDBError as e:
        assert e.code == _lib.MDB_ERR_NODEVICE


def test_server_option_defaults_and_checks(built):
    """Admission-order and priority options: their defaults, and invalid
    values rejected before any device work (so this runs without a GPU)."""
    import ctypes as C

    import md_simulation_cuda_b200 as m

    o = _lib.MDBServerOptions()
    _lib.lib().mdb_server_options_default(C.byref(o))
    assert o.order == m.ORDER_SHORTEST and o.max_wait_ms == 60000 and o.priorities == 1
    assert o.skin == 0.0  # automatic list skin
    for kw in (dict(order=7), dict(max_wait_ms=-1)):
        try:
            m.Server(**kw)
            raise AssertionError(f"accepted {kw}")
        except m.MDBError as e:
            assert e.code == _lib.MDB_ERR_ARG
    e = _lib.MDBOptions()
    _lib.lib().mdb_options_default(C.byref(e))
    assert e.skin == 0.0 and e.stream_priority == 0 and e.max_neighbors == 48


# ctypes mirror -> C typedef of include/mdb200.h
_MIRRORS = {
    "MDBConfigC": "mdb_config_t", "MDBOptions": "mdb_options_t",
    "MDBSchedule": "mdb_schedule_t", "MDBObservables": "mdb_observables_t",
    "MDBFireParams": "mdb_fire_params_t", "MDBMinimizeResult": "mdb_minimize_result_t",
    "MDBServerOptions": "mdb_server_options_t", "MDBRequest": "mdb_request_t",
    "MDBRequestResult": "mdb_request_result_t", "MDBServerStats": "mdb_server_stats_t",
    "MDBNphProtocol": "mdb_nph_protocol_t", "MDBNphRecord": "mdb_nph_record_t",
    "MDBNphResult": "mdb_nph_result_t",
}


def test_ctypes_structs_match_the_header(tmp_path):
    """Every ctypes mirror has the size and field offsets that a C compiler
    gives the header's struct (a C program compiled against
    include/mdb200.h prints them)."""
    import subprocess

    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "mdb200.h"',
             "int main(void) {"]
    for py, c in _MIRRORS.items():
        lines.append(f'  printf("{py} size %zu\\n", sizeof({c}));')
        for name, _ in getattr(_lib, py)._fields_:
            lines.append(f'  printf("{py} {name} %zu\\n", offsetof({c}, {name}));')
    lines.append("  return 0;\n}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), "-I",
                    "/usr/local/cuda/include", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    got = {}
    for line in out.splitlines():
        py, key, val = line.split()
        got[(py, key)] = int(val)
    for py in _MIRRORS:
        cls = getattr(_lib, py)
        assert got[(py, "size")] == C.sizeof(cls), py
        for name, _ in cls._fields_:
            assert got[(py, name)] == getattr(cls, name).offset, (py, name)


_NULL_CALLS = r"""
import ctypes as C, json, sys
from md_simulation_cuda_b200 import _lib
L = _lib.lib()
out = {}
for name, (argt, res) in sorted(_lib.SIGNATURES.items()):
    args = [0.0 if a is C.c_double else 0 if a in (C.c_int, C.c_int32, C.c_int64, C.c_long,
            C.c_ulong, C.c_size_t) else None for a in argt]
    rc = getattr(L, name)(*args)
    out[name] = rc if isinstance(rc, int) or rc is None else repr(rc)
print(json.dumps(out))
"""


def test_null_arguments_return_a_status(built):
    """Every entry point called with null pointers and zero sizes returns a
    status instead of crashing: MDB_ERR_ARG, except the destroy/close calls
    (no-ops on a null handle, as free(NULL)) and the three getters without a
    status. Runs in a child process so that a crash fails the test."""
    import json
    import subprocess
    import sys

    env = dict(os.environ, PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
    p = subprocess.run([sys.executable, "-c", _NULL_CALLS], capture_output=True, text=True,
                       env=env, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    got = json.loads(p.stdout.strip().splitlines()[-1])
    assert set(got) == set(_lib.SIGNATURES)
    noop = {n for n in got if n.endswith(("_destroy", "_close"))}
    no_status = {"mdb_kernel_launches", "mdb_version", "mdb_options_default",
                 "mdb_server_options_default"}
    for name, rc in got.items():
        if name in noop:
            assert rc == 0, name
        elif name not in no_status:
            assert rc == _lib.MDB_ERR_ARG, (name, rc)
