"""Config JSON, overrides and PFRAME files: CPU functions of libmdb200 against
the reference's own src/md_config.cpp and src/md_common.cpp (compiled from the
reference tree into oracle/_ref/ by oracle/build_ref.py) and against the
committed golden fixtures."""
import ctypes as C
import json
import os

import numpy as np
import pytest

import md_simulation_cuda_b200 as mdb

GOLD = os.path.join(os.path.dirname(__file__), "golden")
REF_LIB = os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle", "_ref",
                       "libref_io.so")


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF_LIB):
        from oracle import build_ref

        build_ref.build()
    if not os.path.exists(REF_LIB):
        pytest.skip("reference format code not built (reference tree absent)")
    return C.CDLL(REF_LIB)


def _configs():
    return sorted(f for f in os.listdir(GOLD) if f.startswith("config_") and f.endswith(".json")
                  and not f.endswith(".dump4.json"))


@pytest.mark.parametrize("name", _configs())
def test_config_roundtrip_matches_golden(built, name):
    """config_from_json + config_to_json reproduce the reference's dump(4)
    output byte for byte (fixtures made by tests/golden/make_golden.py)."""
    src = os.path.join(GOLD, name)
    want = open(src.replace(".json", ".dump4.json")).read()
    m = mdb.MDConfigManager.config_from_json(src)
    got = m._dump(4) + "\n"
    assert got == want


@pytest.mark.parametrize("name", _configs())
def test_config_serialize_matches_reference(built, ref, name):
    txt = open(os.path.join(GOLD, name)).read()
    out = C.create_string_buffer(1 << 16)
    assert ref.ref_config_roundtrip(txt.encode(), out, len(out)) > 0
    m = mdb.MDConfigManager()
    m.deserialize(txt)
    assert m.serialize() == out.value.decode()


def test_config_defaults_for_missing_keys(built):
    m = mdb.MDConfigManager()
    m.deserialize('{"dt": 0.002}')
    c = m.config
    assert c.dt == 0.002 and c.EPSILON_AB == 0.25 and c.Q == 100.0 and c.cutoff == 2.5
    assert c.barostat_mass == 1.0e4 and c.pressure_target_mode == b"auto_initial"
    assert c.n_particles_global == 0 and c.THREADS_PER_BLOCK == 256


@pytest.mark.parametrize("key,value", [
    ("dt", "0.005"), ("dt", " 1e-3 "), ("dt", "abc"), ("dt", "1.5x"), ("dt", "inf"),
    ("n_particles_global", "12"), ("n_particles_global", "12.5"),
    ("n_particles_global", "99999999999"), ("run_name", "my run"), ("nosuchkey", "1"),
    ("barostat_mass", "+7"), ("cutoff", ".5"), ("nph_steps", " -3"),
])
def test_apply_override_matches_reference(built, ref, key, value):
    base = open(os.path.join(GOLD, _configs()[0])).read()
    out = C.create_string_buffer(1 << 16)
    r = ref.ref_config_override(base.encode(), key.encode(), value.encode(), out, len(out))
    m = mdb.MDConfigManager()
    m.deserialize(base)
    ok = m.apply_override(key, value)
    assert ok == (r >= 0)
    if ok:
        assert m.serialize() == out.value.decode()


@pytest.mark.parametrize("arg", ["--dt=0.1", "-Ddt=0.1", "Ddt=3", "dt=4", "--D_r=1", "--dt",
                                 "=5", "--=5", ""])
def test_parse_override_argument_matches_reference(built, ref, arg):
    k = C.create_string_buffer(512)
    v = C.create_string_buffer(512)
    r = ref.ref_parse_override(arg.encode(), k, 512, v, 512)
    mine = mdb.MDConfigManager.parse_override_argument(arg)
    if r == 1:
        assert mine == (k.value.decode(), v.value.decode())
    else:
        assert mine is None


def _frame(n, seed):
    rng = np.random.default_rng(seed)
    f = mdb.make_frame(n)
    f["pos"] = rng.uniform(0, 50, (n, 2))
    f["vel"] = rng.normal(size=(n, 2))
    f["acc"] = rng.normal(size=(n, 2))
    f["type"] = rng.integers(0, 2, n)
    f["theta"] = rng.uniform(0, 6.28, n)
    return f


def test_pframe_bytes_match_reference_writer(built, ref, tmp_path):
    a, b = str(tmp_path / "a.bin"), str(tmp_path / "b.bin")
    f1, f2 = _frame(300, 1), _frame(17, 2)
    assert ref.ref_pframe_write(a.encode(), 0, f1.ctypes.data_as(C.c_void_p), 300, 0) == 0
    assert ref.ref_pframe_write(a.encode(), 1, f2.ctypes.data_as(C.c_void_p), 17, 1000) == 0
    w = mdb.FileWriter(b, False)
    w.write_frame(f1, 0)
    mdb.FileWriter(b, True).write_frame(f2, 1000)
    assert open(a, "rb").read() == open(b, "rb").read()
    # and each reads the other's file
    got = mdb.FileReader(a).read(1000)
    assert got.tobytes() == f2.tobytes()
    out = mdb.make_frame(300)
    assert ref.ref_pframe_read(b.encode(), 0, out.ctypes.data_as(C.c_void_p), 300) == 300
    assert out.tobytes() == f1.tobytes()


def test_pframe_golden_fixture(built):
    """A frame written by the reference's FileWriter (fixture) reads back
    bit-exactly and re-encodes to the same bytes."""
    path = os.path.join(GOLD, "frames_ref.pframe")
    meta = json.load(open(os.path.join(GOLD, "frames_ref.json")))
    r = mdb.FileReader(path)
    assert r.n_frames == len(meta["frames"])
    for fr in meta["frames"]:
        f = r.read(fr["index"])
        assert len(f) == fr["n"]
        assert f.tobytes().hex()[:64] == fr["head_hex"]


def test_pframe_corruption_detected(built, tmp_path):
    p = str(tmp_path / "c.bin")
    w = mdb.FileWriter(p, False)
    w.write_frame(_frame(50, 3), 5)
    data = bytearray(open(p, "rb").read())
    data[-3] ^= 0xFF  # damage the compressed payload
    open(p, "wb").write(bytes(data))
    with pytest.raises(mdb.MDBError):
        mdb.FileReader(p).read(5)
    # a v1 header is rejected
    data = bytearray(open(p, "rb").read())
    data[8:12] = (1).to_bytes(4, "little")
    open(p, "wb").write(bytes(data))
    with pytest.raises(mdb.MDBError):
        mdb.FileReader(p)
