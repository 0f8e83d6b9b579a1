"""CPU tests pinning the FP64 oracle to known answers derived from the mathematics (the
reference ships no golden vectors). These run without a GPU."""
import numpy as np
import pytest

import oracle as ora
from opentm_b200 import workloads as wl
from tests.helpers import random_k


def test_template_matrix_structure():
    n = 16
    KE, fe, dp = ora.template_matrix(n)
    h = 1.0 / n
    # trilinear Laplacian on a cube of side h: entries by Hamming distance 1/3, 0, -1/12, -1/12 (x h)
    expect = np.array([1 / 3, 0.0, -1 / 12, -1 / 12]) * h
    for i in range(8):
        for j in range(8):
            assert abs(KE[i, j] - expect[bin(i ^ j).count("1")]) < 1e-15
    # macro field: case 0 = +y, case 1 = -x, case 2 = +z in storage axes (mapping 1,3,2,0,5,7,6,4)
    for i in range(8):
        x, y, z = i & 1, (i >> 1) & 1, i >> 2
        np.testing.assert_allclose(dp[i], [h * y, -h * x, h * z], atol=1e-15)
    np.testing.assert_allclose(fe, KE @ dp, atol=1e-15)


def test_uniform_density_identity():
    r = ora.homogenize(np.ones((8, 8, 8)), tol=1e-12)
    np.testing.assert_allclose(r["C"], np.eye(3), atol=1e-12)


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_laminates(axis):
    n = 8
    k = np.ones((n, n, n))
    sl = [slice(None)] * 3
    sl[2 - axis] = slice(1, None, 2)  # array axes are (z, y, x)
    k[tuple(sl)] = 0.2
    r = ora.homogenize(k, tol=1e-12)
    k1, k2 = 1.0 + 1e-9, 0.2 + 1e-9
    arith, harm = (k1 + k2) / 2, 2 / (1 / k1 + 1 / k2)
    # reference load cases: 0 = y, 1 = x, 2 = z
    case_of_axis = {0: 1, 1: 0, 2: 2}
    d = np.diag(r["C"])
    for ax in range(3):
        c = case_of_axis[ax]
        want = harm if ax == axis else arith
        assert abs(d[c] - want) < 1e-10


def test_multigrid_matches_jacobi_pcg():
    k = wl.simp((0.001 + 0.999 * wl.uniform(3, 16 ** 3)).reshape(16, 16, 16).astype(np.float32))
    a = ora.homogenize(k, tol=1e-13, precond=1)
    b = ora.homogenize(k, tol=1e-13, precond=0, max_iter=50000)
    np.testing.assert_allclose(a["C"], b["C"], rtol=0, atol=1e-13)


def test_symmetry_and_positivity():
    k = wl.simp((0.001 + 0.999 * wl.uniform(4, 12 ** 3)).reshape(12, 12, 12).astype(np.float32))
    C = ora.homogenize(k, tol=1e-12)["C"]
    np.testing.assert_allclose(C, C.T, atol=1e-15)
    assert np.all(np.linalg.eigvalsh(C) > 0)
    # Voigt / Reuss bounds
    kk = k.astype(np.float64) + 1e-9
    assert np.all(np.diag(C) <= kk.mean() + 1e-12)
    assert np.all(np.diag(C) >= 1.0 / (1.0 / kk).mean() - 1e-12)


def test_sensitivity_finite_difference():
    n = 6
    k = wl.simp((0.1 + 0.9 * wl.uniform(5, n ** 3)).reshape(n, n, n).astype(np.float32)).astype(np.float64)
    dC = np.array([[1.0, 0.2, 0.0], [0.3, -0.7, 0.1], [0.0, 0.4, 0.5]])
    r = ora.homogenize(k, tol=1e-14, want_energy=True)
    s = ora.sensitivity(r["energy"], k, dC)
    f = lambda kk: float((ora.homogenize(kk, tol=1e-14)["C"] * dC).sum())
    for e in [(0, 0, 0), (2, 3, 1), (5, 5, 5)]:
        kp, km = k.copy(), k.copy()
        eps = 1e-5 * k[e]
        kp[e] += eps
        km[e] -= eps
        fd = (f(kp) - f(km)) / (2 * eps)
        assert abs(fd - s[e]) <= 1e-6 * max(1.0, abs(s).max())


def test_conv_adjoint_and_normalisation():
    shape = (7, 9, 11)
    x = wl.uniform(6, int(np.prod(shape))).reshape(shape)
    y = wl.uniform(7, int(np.prod(shape))).reshape(shape)
    for wtype, r, per in [(0, 1.5, False), (1, 2.0, True), (1, 2.0, False)]:
        fx, ws = ora.conv_forward(x, wtype, r, per)
        one, _ = ora.conv_forward(np.ones(shape), wtype, r, per)
        np.testing.assert_allclose(one, 1.0, atol=1e-14)  # renormalised by the in-bounds weight
        # <F x, y> = <x, F^T y>
        bt = ora.conv_backward(y, ws, wtype, r, per)
        assert abs((fx * y).sum() - (x * bt).sum()) < 1e-10


def test_oc_update_hits_volume():
    n = 4096
    rho = 0.3 + 0.1 * wl.uniform(8, n)
    s = -(wl.uniform(9, n) + 0.1)
    new, it = ora.oc_update(s, rho, 0.3, 0.001, 0.2, 0.5)
    assert abs(new.mean() - 0.3) <= 1e-4
    assert np.all(new >= 0.001) and np.all(new <= 1.0)
    assert np.all(np.abs(new - rho) <= 0.2 + 1e-12)


def test_mma_solves_small_convex_problem():
    # minimise sum (x - t)^2 s.t. sum x <= V, 0 <= x <= 1; KKT: x = clip(t - mu/2, 0, 1)
    n = 50
    t = wl.uniform(10, n)
    V = 0.3 * n
    x = np.full(n, 0.5)
    xmin, xmax = np.zeros(n), np.ones(n)
    xo1, xo2, low, upp = x.copy(), x.copy(), xmin.copy(), xmax.copy()
    for it in range(1, 60):
        df = 2 * (x - t)
        g = np.array([x.sum() / V - 1.0])
        dg = np.ones((1, n)) / V
        x, xo1, xo2, low, upp = ora.mmasub(it, x, xmin, xmax, xo1, xo2, df, g, dg, low, upp, 1.0,
                                           np.zeros(1), np.full(1, 1e3), np.ones(1), 1.0)
    # exact solution by bisection on mu
    lo, hi = 0.0, 10.0
    for _ in range(200):
        mu = (lo + hi) / 2
        if np.clip(t - mu / 2, 0, 1).sum() > V:
            lo = mu
        else:
            hi = mu
    x_star = np.clip(t - hi / 2, 0, 1)
    assert np.abs(x - x_star).max() < 1e-3


def test_warm_started_solve_matches_cold_and_reuses_the_guess():
    """homogenize_warm (the reference arm's OC-loop solve) converges to the same K^H as a cold solve
    and needs no iteration when started from that solution."""
    k, _ = random_k((16, 16, 16), seed=9)
    cold = ora.homogenize(k, tol=1e-12)
    chi = np.zeros((3, 16, 16, 16))
    warm = ora.homogenize_warm(k, chi, tol=1e-12)
    assert np.abs(warm["C"] - cold["C"]).max() <= 1e-12 * np.abs(cold["C"]).max()
    again = ora.homogenize_warm(k, chi, tol=1e-12)
    assert again["iters"] == [0, 0, 0]
    assert np.abs(again["C"] - cold["C"]).max() <= 1e-12 * np.abs(cold["C"]).max()
