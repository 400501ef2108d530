"""Generates the golden fixtures of tests/test_formats.py by running the
reference's own code (src/md_config.cpp, src/md_common.cpp compiled from the
reference tree into oracle/_ref/libref_io.so by oracle/build_ref.py).

Inputs are this project's own seeded configs and frames; outputs are what the
reference writes for them:
  config_<name>.json        input
  config_<name>.dump4.json  MDConfigManager::config_from_json + config_to_json
  frames_ref.pframe         two frames written by the reference FileWriter
  frames_ref.json           their indices, sizes and leading bytes
Run from the repository root: python tests/golden/make_golden.py
"""
import ctypes as C
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import build_ref  # noqa: E402

PDT = np.dtype({"names": ["pos", "vel", "acc", "type", "_pad", "theta"],
                "formats": [("<f8", (2,)), ("<f8", (2,)), ("<f8", (2,)), "<i4", "<i4", "<f8"],
                "offsets": [0, 16, 32, 48, 52, 56], "itemsize": 64})

LJ = dict(SIGMA_AA=1.0, SIGMA_BB=0.88, SIGMA_AB=0.8, EPSILON_AA=1.0, EPSILON_BB=0.5,
          EPSILON_AB=1.5, MASS_A=1.0, MASS_B=1.0, cutoff=2.5)

CONFIGS = {
    "nve4096": dict(LJ, n_particles_global=4096, n_particles_type0=2662,
                    box_w_global=71.55417527999327, box_h_global=71.55417527999327, T_init=1.0,
                    T_target=1.0, dt=0.001, Q=1.0, rank_size=1, run_name="nve_4096"),
    "slab1m": dict(LJ, n_particles_global=1048576, n_particles_type0=524288,
                   box_w_global=1619.0785019260434, box_h_global=809.5392509630217, T_init=0.7,
                   T_target=0.7, dt=0.002, Q=1.0, rank_size=1, save_dt_interval=10.0),
    "nph": dict(LJ, n_particles_global=4194304, box_w_global=2289.733608959784,
                box_h_global=2289.733608959784, dt=0.001, barostat_mass=10.0, P_target=1.0,
                pressure_target_mode="fixed", barostat_height_min_ratio=0.5,
                barostat_height_max_ratio=2.0, nph_steps=5000),
    "sparse": dict(dt=0.0025, load_name="frames/run \"7\"\\a.bin", EPSILON_AB=1e-20,
                   MASS_B=3e21, x_min=-0.0, x_max=123456789012.5, k_piston=0.1, D_theta=1e-5,
                   mu=0.3333333333333333, halo_left_cap=77),
}


def main():
    lib_path = build_ref.build()
    if not lib_path:
        raise SystemExit("reference tree not available")
    R = C.CDLL(lib_path)
    for name, cfg in CONFIGS.items():
        src = os.path.join(HERE, f"config_{name}.json")
        with open(src, "w") as f:
            json.dump(cfg, f, indent=2)
            f.write("\n")
        dst = os.path.join(HERE, f"config_{name}.dump4.json")
        assert R.ref_config_file_roundtrip(src.encode(), dst.encode()) == 0
    rng = np.random.default_rng(2024)
    path = os.path.join(HERE, "frames_ref.pframe")
    meta = []
    for k, (n, idx) in enumerate([(64, 0), (9, 250)]):
        f = np.zeros(n, dtype=PDT)
        f["pos"] = rng.uniform(0, 20, (n, 2))
        f["vel"] = rng.normal(size=(n, 2))
        f["acc"] = rng.normal(size=(n, 2))
        f["type"] = rng.integers(0, 2, n)
        f["theta"] = rng.uniform(0, 2 * np.pi, n)
        assert R.ref_pframe_write(path.encode(), 1 if k else 0, f.ctypes.data_as(C.c_void_p), n,
                                  idx) == 0
        meta.append(dict(index=idx, n=n, head_hex=f.tobytes().hex()[:64]))
    with open(os.path.join(HERE, "frames_ref.json"), "w") as f:
        json.dump(dict(frames=meta), f, indent=1)


if __name__ == "__main__":
    main()
