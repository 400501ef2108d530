"""Compiles the reference's own code for the parity tests and the bench.

Sources are compiled where they lie under the reference tree (never copied):

  oracle/_ref/libref_io.so       src/md_common.cpp (PFRAME v2 FileWriter /
                                 FileReader) + src/md_config.cpp
                                 (MDConfigManager) + oracle/ref_shim.cpp;
                                 g++ with header-only fmt (bundled with torch),
                                 nlohmann/json (bundled with cudnn_frontend),
                                 zlib and CUDA's vector_types.h.
  oracle/_ref/libref_kernels.so  src/md_cuda_common.cu, unmodified (the force,
                                 energy, pressure, K, integrator and piston
                                 kernels) + oracle/ref_kernels.cu (the
                                 reference's host step logic at world size 1);
                                 nvcc -O3 -DNDEBUG with the default --fmad=true,
                                 the flags of the reference's CMake Release
                                 build, for sm_100a. Its RAFT/RMM includes
                                 resolve to the stand-ins in oracle/ref_stubs/
                                 (only the unused Lanczos solver needs them).

src/md_env.cu and src/md_energy_minimizer.cu are not built: they need MPI,
gDel2D and delaunator (external libraries absent here).

The reference tree comes from the command line (--reference PATH), else from
the MDB_REFERENCE_TREE environment variable, else from the location the
reference is mounted at in the build container. Without a tree the already
built libraries are kept (the GPU machine uses the prebuilt files).

TEST INFRASTRUCTURE ONLY.
"""
from __future__ import annotations

import argparse
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
OUT = os.path.join(OUT_DIR, "libref_io.so")
OUT_KERNELS = os.path.join(OUT_DIR, "libref_kernels.so")
MOUNTED_TREE = "/root/reference"
NVCC = "/usr/local/cuda/bin/nvcc"


def _find(pattern):
    for base in sys.path:
        hits = glob.glob(os.path.join(base, pattern))
        if hits:
            return hits[0]
    return None


def reference_tree(reference: str | None = None) -> str:
    return reference or os.environ.get("MDB_REFERENCE_TREE") or MOUNTED_TREE


def _fmt_include():
    fmt_core = _find("torch/include/fmt/core.h")
    return os.path.dirname(os.path.dirname(fmt_core)) if fmt_core else None


def build_io(reference: str | None = None, force: bool = False) -> str | None:
    ref = reference_tree(reference)
    src = os.path.join(ref, "src")
    if not os.path.isdir(src):
        return OUT if os.path.exists(OUT) else None
    if os.path.exists(OUT) and not force:
        return OUT
    fmt_inc = _fmt_include()
    njson = _find("include/cudnn_frontend/thirdparty/nlohmann/json.hpp")
    if not fmt_inc or not njson:
        return None
    nj_inc = os.path.dirname(os.path.dirname(njson))
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["/usr/bin/g++", "-std=c++17", "-O1", "-shared", "-fPIC", "-DFMT_HEADER_ONLY",
           "-w", f"-I{ref}/include", f"-I{fmt_inc}", f"-I{nj_inc}",
           "-I/usr/local/cuda/include",
           os.path.join(src, "md_common.cpp"), os.path.join(src, "md_config.cpp"),
           os.path.join(HERE, "ref_shim.cpp"), "-lz", "-o", OUT]
    subprocess.run(cmd, check=True)
    return OUT


def build_kernels(reference: str | None = None, force: bool = False) -> str | None:
    ref = reference_tree(reference)
    cu = os.path.join(ref, "src", "md_cuda_common.cu")
    if not os.path.isfile(cu):
        return OUT_KERNELS if os.path.exists(OUT_KERNELS) else None
    driver = os.path.join(HERE, "ref_kernels.cu")
    if (os.path.exists(OUT_KERNELS) and not force
            and os.path.getmtime(OUT_KERNELS) >= os.path.getmtime(driver)):
        return OUT_KERNELS
    fmt_inc = _fmt_include()
    if not fmt_inc or not os.path.exists(NVCC):
        return None
    os.makedirs(OUT_DIR, exist_ok=True)
    flags = ["-O3", "-DNDEBUG", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
             "-Xcompiler", "-fPIC", "-ccbin", "/usr/bin/g++", "-DFMT_HEADER_ONLY", "-w",
             f"-I{ref}/include", f"-I{os.path.join(HERE, 'ref_stubs')}", f"-I{fmt_inc}"]
    jobs, objs = [], []
    for name, path in (("ref_md_cuda_common.o", cu), ("ref_kernels.o", driver)):
        obj = os.path.join(OUT_DIR, name)
        jobs.append(subprocess.Popen([NVCC, *flags, "-c", path, "-o", obj]))
        objs.append(obj)
    if any(j.wait() != 0 for j in jobs):
        raise RuntimeError("nvcc failed on the reference kernels")
    subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-ccbin",
                    "/usr/bin/g++", *objs, "-o", OUT_KERNELS], check=True)
    for obj in objs:
        os.remove(obj)
    return OUT_KERNELS


def build(reference: str | None = None, force: bool = False) -> str | None:
    """Both libraries; returns the path of the format library (or None)."""
    out = build_io(reference, force)
    build_kernels(reference, force)
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--reference", default=None, help="reference source tree")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build_io(a.reference, a.force))
    print(build_kernels(a.reference, a.force))
