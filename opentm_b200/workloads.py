"""Seeded synthetic inputs of the benchmark configurations (host side, numpy).

One counter-based generator is used everywhere: value i of stream `seed` is
splitmix64(seed * 2^32 + i) mapped to [0, 1) with 53 bits; normals use Box-Muller on pairs.
Fields are returned as float32 arrays of shape (nz, ny, nx) (x fastest).

Configurations (SIMP k = kmin + rho^p (k0 - kmin), p = 3, k0 = 1, kmin = 1e-3 unless noted):
  1. plain solve 32^3: rho ~ U(0.001, 1), seed 0
  2. OC loop 128^3: rho0 = 0.3 + 0.05 U(-1, 1), seed 1
  3. mixed 256^3: s = periodic 3x3x3 box mean of N(0,1) (seed 2); rho = clamp(s >= q40(s) ? s : 0, 0.001, 1)
  4. MMA 384^3: rho0 = 0.25 + 0.02 U(-1, 1), seed 3
  5. serving: resolutions {32,48,64,96,128} with weights {.3,.25,.2,.15,.1}; rho ~ U(0.001,1)
     smoothed by a periodic 3x3x3 box mean, seed 4
"""
from __future__ import annotations

import numpy as np

_M = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(counter: np.ndarray) -> np.ndarray:
    z = counter.astype(np.uint64) + np.uint64(0x9E3779B97F4A7C15)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def uniform(seed: int, n: int, offset: int = 0) -> np.ndarray:
    """n values in [0, 1) (float64) of stream `seed`."""
    c = (np.uint64(seed) << np.uint64(32)) + np.arange(offset, offset + n, dtype=np.uint64)
    return (splitmix64(c) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def normal(seed: int, n: int) -> np.ndarray:
    m = (n + 1) // 2
    u1 = uniform(seed, m, 0)
    u2 = uniform(seed, m, m)
    r = np.sqrt(-2.0 * np.log1p(-u1))  # 1 - u1 in (0, 1]
    z = np.concatenate([r * np.cos(2 * np.pi * u2), r * np.sin(2 * np.pi * u2)])
    return z[:n]


def box_mean(a: np.ndarray, k: int = 1) -> np.ndarray:
    """Periodic (2k+1)^3 box mean."""
    out = np.zeros_like(a, dtype=np.float64)
    for dz in range(-k, k + 1):
        for dy in range(-k, k + 1):
            for dx in range(-k, k + 1):
                out += np.roll(a, (dz, dy, dx), axis=(0, 1, 2))
    return out / (2 * k + 1) ** 3


def simp(rho: np.ndarray, p: float = 3.0, k0: float = 1.0, kmin: float = 1e-3) -> np.ndarray:
    return (kmin + rho.astype(np.float64) ** p * (k0 - kmin)).astype(np.float32)


def config1_density(n: int = 32, seed: int = 0) -> np.ndarray:
    return (0.001 + 0.999 * uniform(seed, n ** 3)).reshape(n, n, n).astype(np.float32)


def config2_density(n: int = 128, seed: int = 1) -> np.ndarray:
    return (0.3 + 0.05 * (2.0 * uniform(seed, n ** 3) - 1.0)).reshape(n, n, n).astype(np.float32)


def config3_density(n: int = 256, seed: int = 2) -> np.ndarray:
    s = box_mean(normal(seed, n ** 3).reshape(n, n, n), 1)
    q = np.quantile(s, 0.4)
    rho = np.where(s >= q, s, 0.0)
    return np.clip(rho, 0.001, 1.0).astype(np.float32)


def config4_density(n: int = 384, seed: int = 3) -> np.ndarray:
    return (0.25 + 0.02 * (2.0 * uniform(seed, n ** 3) - 1.0)).reshape(n, n, n).astype(np.float32)


SERVE_RESOS = (32, 48, 64, 96, 128)
SERVE_WEIGHTS = (0.3, 0.25, 0.2, 0.15, 0.1)


def serving_requests(count: int = 2000, seed: int = 4, rate: float = 500.0):
    """(arrival_time_s, reso, rho) tuples: Poisson arrivals at `rate` req/s."""
    u = uniform(seed, 2 * count)
    cw = np.cumsum(SERVE_WEIGHTS)
    t = np.cumsum(-np.log1p(-u[:count]) / rate)
    out = []
    for i in range(count):
        n = SERVE_RESOS[int(np.searchsorted(cw, u[count + i] * cw[-1], side="right"))]
        out.append((float(t[i]), n, i))
    return out


def serving_density(n: int, index: int, seed: int = 4) -> np.ndarray:
    rho = 0.001 + 0.999 * uniform(seed * 1000003 + index + 1, n ** 3).reshape(n, n, n)
    return box_mean(rho, 1).astype(np.float32)
