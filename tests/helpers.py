"""Shared helpers of the parity tests: run the CUDA path and the FP64 oracle on one input."""
from __future__ import annotations

import numpy as np

import oracle as ora
from opentm_b200 import workloads as wl

# Tolerances of the parity gate (stated once here, used by every test).
KH_TOL = 1e-5     # max_ij |dK_ij| / max_ij |K_ij|, and per diagonal entry
SENS_TOL = 1e-4   # max |ds| / max |s| and ||ds||_2 / ||s||_2


def rel_c(c_gpu: np.ndarray, c_ref: np.ndarray) -> float:
    return float(np.abs(c_gpu - c_ref).max() / np.abs(c_ref).max())


def rel_diag(c_gpu: np.ndarray, c_ref: np.ndarray) -> float:
    d = np.diag(c_ref)
    return float((np.abs(np.diag(c_gpu) - d) / np.abs(d)).max())


def rel_entries(c_gpu: np.ndarray, c_ref: np.ndarray) -> np.ndarray:
    """Error of every K^H entry on its own scale: |dK_ij| / sqrt(|K_ii K_jj|) (for a diagonal entry
    that is |dK_ii| / |K_ii|)."""
    d = np.sqrt(np.abs(np.outer(np.diag(c_ref), np.diag(c_ref))))
    return np.abs(np.asarray(c_gpu) - c_ref) / d


def rel_field(a: np.ndarray, b: np.ndarray) -> tuple[float, float]:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    mx = float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
    l2 = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    return mx, l2


def random_k(shape, seed=0, p=3.0):
    """SIMP conductivity of i.i.d. U(0.001, 1) densities (configuration 1 distribution)."""
    n = int(np.prod(shape))
    rho = (0.001 + 0.999 * wl.uniform(seed, n)).reshape(shape).astype(np.float32)
    return wl.simp(rho, p), rho


def oracle_solution(k: np.ndarray, tol: float = 1e-12):
    return ora.homogenize(k.astype(np.float64), tol=tol, want_energy=True, want_chi=True)


DC_TEST = np.array([[1.0, 0.3, -0.2], [0.1, -0.5, 0.25], [0.4, -0.15, 0.8]])
