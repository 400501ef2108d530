"""Shared helpers of the test-suite (comparison metrics, small workloads)."""
import numpy as np


def min_image(d, L):
    L = np.asarray(L, dtype=np.float64)
    return d - L * np.round(d / L)


def rel_l2(a, b):
    """||a - b|| / ||b|| over all particles (the force-error metric)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def rel_err(a, b):
    return abs(a - b) / max(abs(b), 1e-300)
