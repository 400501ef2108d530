"""The C++ drop-in header (include/md_b200.hpp) compiles against libmdb200.so
the way a caller of the reference's classes builds, and (on a GPU) its smoke
driver runs the stepping path end to end."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "md_simulation_cuda_b200")


def _compile(out):
    cmd = ["/usr/bin/g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
           os.path.join(ROOT, "tests", "cpp", "shim_smoke.cpp"), "-L", PKG, "-lmdb200",
           f"-Wl,-rpath,{PKG}", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def test_shim_compiles_and_links(built, tmp_path):
    exe = _compile(str(tmp_path / "shim_smoke"))
    assert os.path.getsize(exe) > 0


@pytest.mark.gpu
def test_shim_smoke_runs(built, tmp_path):
    exe = _compile(str(tmp_path / "shim_smoke"))
    cfg = os.path.join(ROOT, "tests", "golden", "config_nve4096.json")
    r = subprocess.run([exe, cfg, str(tmp_path / "s.pframe")], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "shim smoke OK" in r.stdout
