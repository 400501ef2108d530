"""Compiles the reference's own format code for parity tests.

Sources compiled where they lie under the reference tree (never copied):
  src/md_common.cpp  — PFRAME v2 FileWriter/FileReader
  src/md_config.cpp  — MDConfigManager JSON load/save/overrides
together with oracle/ref_shim.cpp into oracle/_ref/libref_io.so.
Dependencies: header-only fmt (bundled with torch), nlohmann/json (bundled
with cudnn_frontend), zlib, CUDA's vector_types.h. The physics sources
(src/md_cuda_common.cu, src/md_env.cu, src/md_energy_minimizer.cu) need MPI,
RAFT/RMM, gDel2D and delaunator and are not buildable here.

TEST INFRASTRUCTURE ONLY.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
OUT = os.path.join(OUT_DIR, "libref_io.so")


def _find(pattern):
    for base in sys.path:
        hits = glob.glob(os.path.join(base, pattern))
        if hits:
            return hits[0]
    return None


def build(reference: str = "/root/reference", force: bool = False) -> str | None:
    src = os.path.join(reference, "src")
    if not os.path.isdir(src):
        return OUT if os.path.exists(OUT) else None
    if os.path.exists(OUT) and not force:
        return OUT
    fmt_core = _find("torch/include/fmt/core.h")
    njson = _find("include/cudnn_frontend/thirdparty/nlohmann/json.hpp")
    if not fmt_core or not njson:
        return None
    fmt_inc = os.path.dirname(os.path.dirname(fmt_core))
    nj_inc = os.path.dirname(os.path.dirname(njson))
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["/usr/bin/g++", "-std=c++17", "-O1", "-shared", "-fPIC", "-DFMT_HEADER_ONLY",
           "-w", f"-I{reference}/include", f"-I{fmt_inc}", f"-I{nj_inc}",
           "-I/usr/local/cuda/include",
           os.path.join(src, "md_common.cpp"), os.path.join(src, "md_config.cpp"),
           os.path.join(HERE, "ref_shim.cpp"), "-lz", "-o", OUT]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force=True))
