"""Host-side checks of the design driver (no GPU): the convergence test and the volume governor
of the C ABI against their restatement, the driver's file formats, the openTM argument checks,
and known-answer checks that pin the oracle's initial fields and symmetrisations."""
import numpy as np
import pytest

from oracle import driver as od


def _lib_or_skip():
    from opentm_b200 import _lib
    try:
        return _lib.lib()
    except RuntimeError as e:  # library not built
        pytest.skip(str(e))


# ---------------------------------------------------------------------------------------
# ConvergeChecker / VolumeGovernor: C ABI == restatement
# ---------------------------------------------------------------------------------------
def test_converge_checker_matches_restatement():
    _lib_or_skip()
    from opentm_b200.driver import ConvergeChecker
    rng = np.random.default_rng(0)
    for trial in range(20):
        thres = [1e-3, 5e-4, 1e-2][trial % 3]
        a, b = ConvergeChecker(thres), od.ConvergeChecker(thres)
        # a decaying objective that flattens out, with noise of varying size
        val = 1.0
        for it in range(60):
            val = val * (1 - 0.3 * np.exp(-it / 5.0)) + rng.normal() * 10.0 ** rng.uniform(-7, -2)
            assert a.is_converge(it, val) == b.is_converge(it, val), (trial, it)


def test_converge_checker_needs_three_flat_steps():
    b = od.ConvergeChecker(1e-3)
    hits = [b.is_converge(it, 1.0 + (0.5 if it < 14 else 0.0)) for it in range(20)]
    assert not any(hits[:12])          # never before iteration 12
    assert hits[14:16] == [False, False] and hits[17] is True


def test_volume_governor_matches_restatement():
    _lib_or_skip()
    from opentm_b200.driver import VolumeGovernor
    rng = np.random.default_rng(1)
    for trial in range(30):
        a, b = VolumeGovernor(), od.VolumeGovernor()
        val = float(rng.uniform(0.01, 0.1))
        for itn in range(150):
            kind = trial % 3
            if kind == 0:    # oscillating objective: anti-vibration path
                val = val + (0.002 if itn % 2 else -0.002) * rng.uniform(0.5, 1.5)
            elif kind == 1:  # converging to below zero: shrink path
                val = val * 0.9 - 2e-4
            else:            # stalling: expansion path
                val = val - rng.uniform(0, 5e-5)
            low = float(rng.uniform(0.05, 0.3))
            volfrac = float(a.get_volume_bound() + rng.uniform(-0.012, 0.012))
            ra = a.volume_check(val, low, volfrac, itn)
            rb = b.volume_check(val, low, volfrac, itn)
            assert ra == rb
            assert np.float32(a.get_volume_bound()) == b.vb, (trial, itn)
            assert np.float32(a.get_current_decrease()) == b.get_current_decrease(), (trial, itn)


def test_volume_governor_shrink_known_answer():
    g = od.VolumeGovernor()
    # objective below zero: shrink to the lower bound, factor 1 -> 0.8
    g.volume_check(-1e-3, 0.25, 0.5, 0)
    assert g.vb == np.float32(0.25) and g.dec == np.float32(0.75) and g.df == np.float32(0.8)


# ---------------------------------------------------------------------------------------
# File formats
# ---------------------------------------------------------------------------------------
def test_density_binary_round_trip_and_layout(tmp_path):
    _lib_or_skip()
    from opentm_b200 import driver as dr
    rho = np.random.default_rng(2).random((5, 4, 3), dtype=np.float32)  # (nz, ny, nx)
    p = tmp_path / "rho.bin"
    dr.write_density_binary(str(p), rho)
    raw = p.read_bytes()
    assert np.array_equal(np.frombuffer(raw[:12], dtype=np.int32), [3, 4, 5])  # x, y, z sizes
    assert np.array_equal(np.frombuffer(raw[12:], dtype=np.float32), rho.ravel())  # x fastest
    assert np.array_equal(dr.read_density_binary(str(p)), rho)


def test_density_binary_rejects_bad_files(tmp_path):
    _lib_or_skip()
    from opentm_b200 import OtmError
    from opentm_b200 import driver as dr
    p = tmp_path / "short.bin"
    p.write_bytes(np.array([4, 4, 4], dtype=np.int32).tobytes() + b"\0" * 16)
    with pytest.raises(OtmError):
        dr.read_density_binary(str(p))
    p.write_bytes(np.array([0, 4, 4], dtype=np.int32).tobytes())
    with pytest.raises(OtmError):
        dr.read_density_binary(str(p))
    with pytest.raises(OtmError):
        dr.read_density_binary(str(tmp_path / "missing.bin"))


def test_vectors_interleaved_round_trip(tmp_path):
    _lib_or_skip()
    from opentm_b200 import driver as dr
    a, b, c = (np.arange(7, dtype=np.float32) + 10 * i for i in range(3))
    p = tmp_path / "vec"
    dr.write_vectors(str(p), [a, b, c])
    rec = np.frombuffer(p.read_bytes(), dtype=np.float32).reshape(7, 3)  # record j = (a_j, b_j, c_j)
    assert np.array_equal(rec, np.stack([a, b, c], axis=1))
    got = dr.read_vectors(str(p), 3)
    assert all(np.array_equal(x, y) for x, y in zip(got, (a, b, c)))
    dr.write_vectors(str(p), [a])
    assert np.array_equal(dr.read_vectors(str(p), 1)[0], a)


def test_heat_matrix_files(tmp_path):
    _lib_or_skip()
    from opentm_b200 import driver as dr
    K = np.arange(9, dtype=np.float32).reshape(3, 3) / 8
    dr.write_heat_matrix(str(tmp_path / "C"), K)
    assert np.array_equal(np.frombuffer((tmp_path / "C").read_bytes(), dtype=np.float32), K.ravel())
    dr.write_heat_matrix(str(tmp_path / "C.txt"), K, text=True)
    rows = [[float(v) for v in line.split()] for line in (tmp_path / "C.txt").read_text().splitlines()]
    assert np.allclose(rows, K)


def test_openTM_argument_checks():
    from opentm_b200 import openTM
    with pytest.raises(ValueError):
        openTM.runInstance(16, [1.0], [0.3, 0.2, 0.1, 0, 0, 0])
    h = openTM.homo()
    with pytest.raises(ValueError):
        h.setConfig(16, [1, 2, 3], [0.3, 0.2, 0.1, 0, 0, 0])
    h.setConfig(16, [1, 1e-4], [0.3, 0.2, 0.1, 0, 0, 0])
    with pytest.raises(ValueError):
        h.optimize()  # no density set


# ---------------------------------------------------------------------------------------
# Known answers that pin the oracle's restatement
# ---------------------------------------------------------------------------------------
def test_randtri_basis_index_convention():
    """Single coefficients select the functions the reference's index arithmetic names
    (Framework.cuh:180-205): first-order i < 3n is cos of axis i % 3 at frequency i / 3 + 1,
    i in [3n, 6n) the sin; second-order 6n + j 6n + k is g_j g_k with g_j = cos of axis j / n
    at frequency j % n + 1 (j < 3n), sin beyond."""
    n, npd = 9, 2
    x, y, z = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")[::-1]
    p = [x / (n - 1.0), y / (n - 1.0), z / (n - 1.0)]
    cnt = od.randtri_count(npd, False)

    def field(idx):
        c = np.zeros(cnt)
        c[idx] = 1.0
        return od.randtri_field(n, npd, c, False)

    w = 2 * np.pi
    assert np.allclose(field(0), np.cos(w * p[0]))
    assert np.allclose(field(1), np.cos(w * p[1]))
    assert np.allclose(field(3), np.cos(2 * w * p[0]))        # axis 0, frequency 2
    assert np.allclose(field(3 * npd + 2), np.sin(w * p[2]))  # sin, axis 2, frequency 1
    j, k = 1, 3 * npd + 2 * npd + 1                            # cos(4 pi x) * sin(4 pi z)
    assert np.allclose(field(6 * npd + j * 6 * npd + k), np.cos(2 * w * p[0]) * np.sin(2 * w * p[2]))


def test_symmetrize_results_are_invariant_and_idempotent():
    rng = np.random.default_rng(3)
    f = rng.random((8, 8, 8), dtype=np.float32)
    r3 = od.symmetrize(f, od.SYM_REFLECT3)
    for ax in range(3):
        assert np.allclose(r3, np.flip(r3, axis=ax))
    r6 = od.symmetrize(f, od.SYM_REFLECT6)
    assert np.allclose(r6, np.transpose(r6, (1, 0, 2))) and np.allclose(r6, np.transpose(r6, (2, 1, 0)))
    assert np.allclose(r6, np.flip(r6, axis=0))
    rot = od.symmetrize(f, od.SYM_ROTATE3)
    # 90-degree rotations about the centre: (x, y) -> (y, -x) and the cyclic axis permutation
    assert np.allclose(rot, np.rot90(rot, k=1, axes=(1, 2)))
    assert np.allclose(rot, np.transpose(rot, (1, 2, 0)))
    r2 = od.symmetrize(f, od.SYM_ROTATE2)
    assert np.allclose(r2, r2[::-1, ::-1, ::-1])
    for s in (od.SYM_REFLECT3, od.SYM_REFLECT6, od.SYM_ROTATE3, od.SYM_ROTATE2):
        once = od.symmetrize(f, s)
        assert np.allclose(od.symmetrize(once, s), once)
        if s in (od.SYM_REFLECT3, od.SYM_ROTATE2):  # disjoint orbits of equal size: the mean stays
            assert np.isclose(once.astype(np.float64).mean(), f.astype(np.float64).mean(), rtol=1e-6)


def test_tpms_fields_have_their_symmetries():
    P, D, IWP = (od.init_closed(w, 16) for w in (od.INIT_P, od.INIT_D, od.INIT_IWP))
    for f in (P, IWP):  # symmetric under any exchange of axes
        assert np.allclose(f, np.transpose(f, (1, 0, 2)), atol=1e-5)
        assert np.allclose(f, np.transpose(f, (2, 1, 0)), atol=1e-5)
    assert np.allclose(D, np.transpose(D, (1, 2, 0)), atol=1e-5)
    for f in (P, D, IWP):
        assert f.min() >= np.float32(0.001) and f.max() <= 1.0
    ex = od.init_closed(od.INIT_EXAMPLE, 12)
    assert set(np.unique(ex)) == {np.float32(0.0), np.float32(0.3)} and ex[6, 6, 6] == 0 and ex[0, 0, 0] == np.float32(0.3)


def test_randtri_init_meets_volume():
    co = od.randtri_coefficients(5, 2, False)
    f = od.randtri_init(12, 2, co, False, od.SYM_NONE, 0.3)
    assert abs(f.astype(np.float64).mean() - 0.3) / 0.3 < 1e-3
