"""Seeded synthetic inputs for the benchmark configurations.

No public dataset is involved: every frame is generated from a seed with the
shapes, sizes and value distributions of the workload it stands for.

Shared LJ parameters: eps_AA=1.0, eps_BB=0.5, eps_AB=1.5; sigma_AA=1.0,
sigma_BB=0.88, sigma_AB=0.8; cutoff 2.5 (rc_ij = 2.5 sigma_ij); MASS_A =
MASS_B = 1; type 0 = A, type 1 = B.
"""
from __future__ import annotations

import math
from typing import Dict, List, Tuple

import numpy as np

from ._lib import PARTICLE_DTYPE

LJ = dict(SIGMA_AA=1.0, SIGMA_BB=0.88, SIGMA_AB=0.8, EPSILON_AA=1.0, EPSILON_BB=0.5,
          EPSILON_AB=1.5, MASS_A=1.0, MASS_B=1.0, cutoff=2.5)


def config_dict(N: int, Lx: float, Ly: float, dt: float, T: float = 1.0, Q: float = 1.0,
                **extra) -> Dict:
    d = dict(LJ)
    d.update(n_particles_global=int(N), box_w_global=float(Lx), box_h_global=float(Ly),
             T_init=float(T), T_target=float(T), dt=float(dt), Q=float(Q), rank_size=1)
    d.update(extra)
    return d


def _velocities(rng, types, T, mA=1.0, mB=1.0):
    n = len(types)
    m = np.where(types == 0, mA, mB)
    v = rng.normal(0.0, 1.0, (n, 2)) * np.sqrt(T / m)[:, None]
    p = (m[:, None] * v).sum(0) / m.sum()
    return v - p


def lattice_frame(N: int, rho: float, aspect: float, f_A, T: float, seed: int,
                  jitter: float = 0.1) -> Tuple[np.ndarray, float, float]:
    """Jittered square lattice filled row by row; Lx = aspect * Ly.

    f_A is a number (A fraction everywhere) or a callable x/Lx -> A fraction
    (the interface slab)."""
    rng = np.random.default_rng(seed)
    Ly = math.sqrt(N / (rho * aspect))
    Lx = aspect * Ly
    nx = int(math.ceil(math.sqrt(N * aspect)))
    ny = int(math.ceil(N / nx))
    while nx * ny < N:
        ny += 1
    ax, ay = Lx / nx, Ly / ny
    k = np.arange(N)
    ix, iy = k % nx, k // nx
    pos = np.stack([(ix + 0.5) * ax, (iy + 0.5) * ay], axis=1)
    pos += rng.uniform(-jitter, jitter, (N, 2))
    pos[:, 0] %= Lx
    pos[:, 1] %= Ly
    if callable(f_A):
        fa = f_A(pos[:, 0] / Lx)
    else:
        fa = np.full(N, float(f_A))
    types = (rng.random(N) >= fa).astype(np.int32)  # 0 = A with probability f_A
    f = np.zeros(N, dtype=PARTICLE_DTYPE)
    f["pos"] = pos
    f["vel"] = _velocities(rng, types, T)
    f["type"] = types
    return f, Lx, Ly


def random_frame(N: int, rho: float, f_A: float, seed: int) -> Tuple[np.ndarray, float]:
    """Uniform random positions in a square box (FIRE quench starts)."""
    rng = np.random.default_rng(seed)
    L = math.sqrt(N / rho)
    f = np.zeros(N, dtype=PARTICLE_DTYPE)
    f["pos"] = rng.uniform(0.0, L, (N, 2))
    f["type"] = (rng.random(N) >= f_A).astype(np.int32)
    return f, L


# ---- the five configurations -------------------------------------------------

def nve_4096(seed: int = 1):
    """NVE N=4096, 65% A, square box at rho=0.8, 64x64 lattice +-0.1, T=1.0,
    dt=0.001 (1000 steps)."""
    f, Lx, Ly = lattice_frame(4096, 0.8, 1.0, 0.65, 1.0, seed)
    return f, config_dict(4096, Lx, Ly, dt=0.001, T=1.0)


def nvt_slab(N: int = 1048576, seed: int = 2):
    """Nose-Hoover interface slab: Lx = 2 Ly, rho=0.8, 90% A for x < Lx/2 and
    10% A above, T=0.7, Q=1.0, dt=0.002."""
    f, Lx, Ly = lattice_frame(N, 0.8, 2.0, lambda s: np.where(s < 0.5, 0.9, 0.1), 0.7, seed)
    return f, config_dict(N, Lx, Ly, dt=0.002, T=0.7, Q=1.0)


def nph_square(N: int = 4194304, seed: int = 3):
    """NPH: square box at rho=0.8, 65% A, P=1.0, W=10.0, dt=0.001."""
    f, Lx, Ly = lattice_frame(N, 0.8, 1.0, 0.65, 1.0, seed)
    return f, config_dict(N, Lx, Ly, dt=0.001, T=1.0, barostat_mass=10.0)


def fire_mix(n_systems: int = 512, seed: int = 4, n_min: int = 256, n_max: int = 16384):
    """Batched FIRE: N log-uniform in [n_min, n_max], f_A ~ U(0.2,0.8),
    rho ~ U(0.6,1.0), square boxes, uniform-random positions."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_systems):
        N = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        fa = float(rng.uniform(0.2, 0.8))
        rho = float(rng.uniform(0.6, 1.0))
        f, L = random_frame(N, rho, fa, seed * 100003 + k)
        out.append((f, config_dict(N, L, L, dt=0.001, T=0.0)))
    return out


FIRE_SETTINGS = dict(dt_init=0.001, dt_max=0.01, alpha0=0.1, f_inc=1.1, f_dec=0.5, N_min=5,
                     force_tol=1e-6, max_steps=20000)


def fire_params():
    """FireParams of the batched FIRE mix and the served FIRE quenches."""
    from . import FireParams

    s = FIRE_SETTINGS
    return FireParams(dt_init=s["dt_init"], dt_max=s["dt_max"], alpha0=s["alpha0"],
                      f_inc=s["f_inc"], f_dec=s["f_dec"], N_min=s["N_min"])


def served_stream(n_requests: int = 2000, rate: float = 200.0, seed: int = 5,
                  fire_fraction: float = 0.3, n_min: int = 1024, n_max: int = 262144):
    """Request specs of the served mixed stream: Poisson arrivals at `rate`
    per second; NVT segments (N log-uniform in [n_min, n_max], 1000-20000
    steps, T ~ U(0.5, 1.2)) or FIRE quenches (fire_fraction of requests, same
    N law), each from a jittered-lattice start with its own seed. Frames are
    made on demand by served_frame(spec)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(n_requests):
        t += float(rng.exponential(1.0 / rate))
        N = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        fire = bool(rng.random() < fire_fraction)
        steps = int(rng.integers(1000, 20001))
        T = float(rng.uniform(0.5, 1.2))
        out.append(dict(k=k, arrival=t, N=N, fire=fire, steps=steps, T=T,
                        seed=seed * 1000003 + k))
    return out


def served_frame(spec):
    """(frame, config dict) of one served request: rho = 0.8, 65% A, square
    box, lattice jitter +-0.1; FIRE quenches start at rest."""
    T = 0.0 if spec["fire"] else spec["T"]
    f, Lx, Ly = lattice_frame(spec["N"], 0.8, 1.0, 0.65, T, spec["seed"], jitter=0.1)
    return f, config_dict(spec["N"], Lx, Ly, dt=0.002 if not spec["fire"] else 0.001,
                          T=spec["T"], Q=1.0, n_cap=spec["N"])
