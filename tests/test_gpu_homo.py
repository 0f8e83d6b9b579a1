"""GPU parity of the homogenization path (K^H, element energies, sensitivity) against the FP64
oracle, through the C ABI. Tolerances: K^H 1e-5 (norm-relative and per diagonal entry),
sensitivity 1e-4 (max-relative and relative L2); see tests/helpers.py."""
import numpy as np
import pytest

import oracle as ora
from opentm_b200 import workloads as wl
from tests.helpers import (DC_TEST, KH_TOL, SENS_TOL, oracle_solution, random_k, rel_c, rel_diag, rel_entries,
                           rel_field)

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def gpu_run(k, tol=1e-6, pre=2, post=2, dC=DC_TEST, pitchT=-1, **kw):
    from opentm_b200 import HomoConfig, Homogenization_H
    nz, ny, nx = k.shape
    H = Homogenization_H(HomoConfig(reso=(nx, ny, nz), femRelThres=tol, pre_smooth=pre, post_smooth=post,
                                    max_iter=kw.pop("max_iter", 200), **kw))
    if pitchT > 0:
        kp = torch.zeros((nz, ny, pitchT), dtype=torch.float32, device="cuda")
        kp[:, :, :nx] = torch.from_numpy(k).cuda()
        H.update(kp, pitchT)
    else:
        H.update(torch.from_numpy(np.ascontiguousarray(k)).cuda())
    C = H.heatMatrix()
    E = H.element_energy().cpu().numpy()
    sens = torch.empty(k.shape, dtype=torch.float32, device="cuda")
    H.Sensitivity(dC, sens, -1, False)
    torch.cuda.synchronize()
    return H, C, E, sens.cpu().numpy()


def check_against_oracle(k, C, E, sens, dC=DC_TEST):
    ref = oracle_solution(k)
    assert rel_c(C, ref["C"]) <= KH_TOL, (C, ref["C"])
    assert rel_diag(C, ref["C"]) <= KH_TOL
    assert rel_entries(C, ref["C"]).max() <= KH_TOL, rel_entries(C, ref["C"])
    for a in range(6):
        mx, l2 = rel_field(E[a], ref["energy"][a])
        assert mx <= SENS_TOL and l2 <= SENS_TOL, (a, mx, l2)
    s_ref = ora.sensitivity(ref["energy"], k, dC)
    mx, l2 = rel_field(sens, s_ref)
    assert mx <= SENS_TOL and l2 <= SENS_TOL, (mx, l2)
    return ref


def test_uniform_density_gives_identity():
    k = np.ones((16, 16, 16), dtype=np.float32)
    _, C, _, _ = gpu_run(k)
    np.testing.assert_allclose(C, np.eye(3), atol=1e-6)


def test_laminate_closed_form():
    # layers along storage x: reference K[1][1] (load case -x) is the harmonic mean,
    # K[0][0] and K[2][2] the arithmetic mean (templateMatrix.cpp:74-85 axis convention)
    k = np.ones((16, 16, 16), dtype=np.float32)
    k[:, :, 0::2] = 1.0
    k[:, :, 1::2] = 0.1
    _, C, _, _ = gpu_run(k, tol=1e-7)
    k1, k2 = 1.0 + 1e-9, 0.1 + 1e-9
    arith, harm = (k1 + k2) / 2, 2.0 / (1 / k1 + 1 / k2)
    assert abs(C[0, 0] - arith) / arith < 1e-5
    assert abs(C[2, 2] - arith) / arith < 1e-5
    assert abs(C[1, 1] - harm) / harm < 1e-5


def test_config1_32_parity():
    """Configuration 1: 32^3, rho ~ U(0.001,1) seed 0, SIMP p=3, V(2,2), tol 1e-6."""
    k, _ = random_k((32, 32, 32), seed=0)
    H, C, E, sens = gpu_run(k, tol=1e-6)
    check_against_oracle(k, C, E, sens)
    st = H.stats()
    assert st.levels >= 3 and max(st.rel_res) <= 1e-6


@pytest.mark.parametrize("shape", [(8, 8, 8), (16, 16, 16), (32, 16, 8), (24, 24, 24), (20, 20, 20), (4, 4, 4),
                                   (6, 6, 6)])
def test_shapes_parity(shape):
    k, _ = random_k(shape, seed=sum(shape))
    _, C, E, sens = gpu_run(k, tol=1e-7)
    check_against_oracle(k, C, E, sens)


def test_vcycle_solver_parity():
    k, _ = random_k((16, 16, 16), seed=5)
    _, C, E, sens = gpu_run(k, tol=1e-7, solver="vcycle")
    check_against_oracle(k, C, E, sens)


def test_v11_and_v33_cycles():
    k, _ = random_k((16, 16, 16), seed=6)
    for s in (1, 3):
        _, C, E, sens = gpu_run(k, tol=1e-7, pre=s, post=s)
        check_against_oracle(k, C, E, sens)


def test_graphs_match_direct_launches_bitwise():
    k, _ = random_k((16, 16, 16), seed=7)
    _, C1, E1, s1 = gpu_run(k, use_graphs=True)
    _, C2, E2, s2 = gpu_run(k, use_graphs=False)
    assert np.array_equal(C1, C2) and np.array_equal(E1, E2) and np.array_equal(s1, s2)


def test_deterministic_repeat():
    k, _ = random_k((32, 32, 32), seed=8)
    _, C1, _, s1 = gpu_run(k)
    _, C2, _, s2 = gpu_run(k)
    assert np.array_equal(C1, C2) and np.array_equal(s1, s2)


def test_pitched_input_and_lexi_sensitivity():
    k, _ = random_k((16, 16, 16), seed=9)
    H, C, E, sens = gpu_run(k, pitchT=128)
    check_against_oracle(k, C, E, sens)
    pitched = torch.full((16, 16, 128), 7.0, dtype=torch.float32, device="cuda")
    H.Sensitivity(DC_TEST, pitched, 128, True)
    p = pitched.cpu().numpy()
    np.testing.assert_array_equal(p[:, :, :16], sens)
    assert np.all(p[:, :, 16:] == 0.0)  # pitch padding zeroed like init_array in the reference


def test_warm_start_reduces_iterations():
    from opentm_b200 import HomoConfig, Homogenization_H
    k, _ = random_k((32, 32, 32), seed=10)
    H = Homogenization_H(HomoConfig(reso=32, femRelThres=1e-6, pre_smooth=2, post_smooth=2))
    H.update(torch.from_numpy(k).cuda())
    H.heatMatrix()
    cold = H.stats().iterations
    k2 = (k * (1.0 + 0.01 * np.cos(np.arange(k.size)).reshape(k.shape))).astype(np.float32)
    H.update(torch.from_numpy(k2).cuda())
    C = H.heatMatrix()
    warm = H.stats().iterations
    assert warm < cold
    ref = oracle_solution(k2)
    assert rel_c(C, ref["C"]) <= KH_TOL


def test_power_penal_sensitivity():
    # power_penal != 1: solver uses 1e-9 + k^p, sensitivity carries p k^(p-1)
    k, _ = random_k((8, 8, 8), seed=11)
    from opentm_b200 import HomoConfig, Homogenization_H
    H = Homogenization_H(HomoConfig(reso=8, femRelThres=1e-6, pre_smooth=2, post_smooth=2, power_penal=2.0))
    H.update(torch.from_numpy(k).cuda())
    C = H.heatMatrix()
    sens = torch.empty(k.shape, dtype=torch.float32, device="cuda")
    H.Sensitivity(DC_TEST, sens)
    ref = ora.homogenize(k.astype(np.float64), power_penal=2.0, tol=1e-12, want_energy=True)
    assert rel_c(C, ref["C"]) <= KH_TOL
    s_ref = ora.sensitivity(ref["energy"], k, DC_TEST, power_penal=2.0)
    mx, l2 = rel_field(sens.cpu().numpy(), s_ref)
    assert mx <= SENS_TOL and l2 <= SENS_TOL


def test_nan_input_is_rejected():
    from opentm_b200 import HomoConfig, Homogenization_H, OtmError
    k = np.ones((8, 8, 8), dtype=np.float32)
    k[3, 3, 3] = np.nan
    H = Homogenization_H(HomoConfig(reso=8))
    H.update(torch.from_numpy(k).cuda())
    with pytest.raises(OtmError) as ei:
        H.heatMatrix()
    assert ei.value.status == 7  # OTM_ERR_NAN
    # the status belongs to the imported field: a valid field afterwards solves normally
    good, _ = random_k((8, 8, 8), seed=13)
    H.update(torch.from_numpy(good).cuda())
    H.reset_displacement()
    assert np.all(np.isfinite(H.heatMatrix()))


def test_iteration_cap_reports_not_converged():
    from opentm_b200 import HomoConfig, Homogenization_H, OtmError
    k, _ = random_k((16, 16, 16), seed=12)
    H = Homogenization_H(HomoConfig(reso=16, femRelThres=1e-12, max_iter=2, pre_smooth=1, post_smooth=1))
    H.update(torch.from_numpy(k).cuda())
    with pytest.raises(OtmError) as ei:
        H.heatMatrix()
    assert ei.value.status == 5  # OTM_ERR_NOT_CONVERGED
    C = H.heatMatrix(allow_not_converged=True)
    assert np.all(np.isfinite(C))


def test_two_handles_are_independent():
    from opentm_b200 import HomoConfig, Homogenization_H
    ka, _ = random_k((16, 16, 16), seed=13)
    kb, _ = random_k((8, 8, 8), seed=14)
    Ha = Homogenization_H(HomoConfig(reso=16, femRelThres=1e-7, pre_smooth=2, post_smooth=2))
    Hb = Homogenization_H(HomoConfig(reso=8, femRelThres=1e-7, pre_smooth=2, post_smooth=2))
    Ha.update(torch.from_numpy(ka).cuda())
    Hb.update(torch.from_numpy(kb).cuda())
    Ca, Cb = Ha.heatMatrix(), Hb.heatMatrix()
    assert rel_c(Ca, oracle_solution(ka)["C"]) <= KH_TOL
    assert rel_c(Cb, oracle_solution(kb)["C"]) <= KH_TOL


def test_profile_events_inside_graphs():
    from opentm_b200 import HomoConfig, Homogenization_H
    k, _ = random_k((32, 32, 32), seed=15)
    for graphs in (True, False):
        H = Homogenization_H(HomoConfig(reso=32, femRelThres=1e-6, pre_smooth=2, post_smooth=2, profile=True,
                                        use_graphs=graphs, smoother="tiled"))
        H.update(torch.from_numpy(k).cuda())
        H.heatMatrix()
        pr = H.profile()
        assert pr.sweeps == H.stats().iterations > 0
        # the tiled smoother's timed region is its post-smoothing leg, one launch per sweep: each
        # reads u, k, f and writes u (3 cases, FP32), the first also reads the coarse correction
        assert pr.kernel_kind == 1 and pr.launches_per_sweep == 2
        assert pr.sweep_ms > 0 and pr.sweep_bytes == 32 ** 3 * (2 * (12 + 4 + 12 + 12) + 1.5)
        # a following library call still works (no stale error from the event queries)
        H.heatMatrix_nosolve()


@pytest.mark.parametrize("precision", ["bf16", "fp16"])
@pytest.mark.parametrize("shape", [(32, 32, 32), (16, 16, 16), (24, 24, 24)])
def test_mixed_precision_parity(precision, shape):
    """16-bit fine-level storage with FP64 refinement meets the same K^H / sensitivity gates."""
    k, _ = random_k(shape, seed=20 + shape[0])
    H, C, E, sens = gpu_run(k, tol=1e-6, precision=precision)
    check_against_oracle(k, C, E, sens)
    st = H.stats()
    # PCG iterations with at least the start and the converged FP64 residual evaluations
    assert st.iterations > 0 and 2 <= st.refinements <= st.iterations + 1 and max(st.rel_res) <= 1e-6


def test_mixed_precision_warm_start_and_reset():
    from opentm_b200 import HomoConfig, Homogenization_H
    k, _ = random_k((32, 32, 32), seed=30)
    H = Homogenization_H(HomoConfig(reso=32, femRelThres=1e-6, pre_smooth=2, post_smooth=2, precision="bf16"))
    H.update(torch.from_numpy(k).cuda())
    H.heatMatrix()
    cold = H.stats().iterations
    H.update(torch.from_numpy(k).cuda())
    C = H.heatMatrix()
    assert H.stats().iterations < cold  # the FP64 solution is reused
    H.reset_displacement()
    H.update(torch.from_numpy(k).cuda())
    C2 = H.heatMatrix()
    assert H.stats().iterations == cold
    assert rel_c(C2, C) <= KH_TOL


@pytest.mark.parametrize("shape", [(32, 32, 32), (64, 64, 64), (48, 48, 48), (48, 32, 64)])
def test_cluster_cycle_matches_per_level_kernels(shape):
    """The lower levels run as one thread-block-cluster launch (distributed shared memory,
    cluster barriers); the result equals the per-level kernels' and meets the oracle gates."""
    nz, ny, nx = shape
    k, _ = random_k(shape, seed=40 + nx + ny + nz)
    H1, C1, E1, s1 = gpu_run(k, tol=1e-7, cluster_cycle=True)
    H2, C2, E2, s2 = gpu_run(k, tol=1e-7, cluster_cycle=False)
    assert H1.stats().cluster_level >= 1 and H2.stats().cluster_level == -1
    assert rel_c(C1, C2) <= 1e-6
    assert abs(H1.stats().iterations - H2.stats().iterations) <= 1
    mx, l2 = rel_field(s1, s2)
    assert mx <= SENS_TOL and l2 <= SENS_TOL
    check_against_oracle(k, C1, E1, s1)


@pytest.mark.parametrize("shape,auto_level", [((64, 64, 64), 2), ((48, 48, 48), 1)])
def test_cluster_from_16_cubed(shape, auto_level):
    """cluster_cycle 2: the cluster launch starts at the level with <= 16^3 unknowns and the
    level above it is smoothed by the coarse tile kernels (64^3) or colour passes (48^3). The
    automatic choice (cluster_cycle 1) takes that level only where the level above is tiled."""
    nz, ny, nx = shape
    k, _ = random_k(shape, seed=50 + nx)
    H1, C1, E1, s1 = gpu_run(k, tol=1e-7, cluster_cycle=2)
    H2, C2, E2, s2 = gpu_run(k, tol=1e-7, cluster_cycle=0)
    H3, C3, E3, s3 = gpu_run(k, tol=1e-7, cluster_cycle=1)
    assert H1.stats().cluster_level == 2 and H2.stats().cluster_level == -1
    assert H3.stats().cluster_level == auto_level
    assert rel_c(C1, C2) <= 1e-6 and rel_c(C3, C2) <= 1e-6
    assert abs(H1.stats().iterations - H2.stats().iterations) <= 1
    check_against_oracle(k, C1, E1, s1)


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_heat_matrix_sensitivity_one_pass(precision):
    """heatMatrixSensitivity (K^H and the sensitivity in one element pass) returns what
    heatMatrix + Sensitivity return, bit for bit, pitched output with zeroed padding included; x
    not a multiple of the 8-element runs of the element pass."""
    from opentm_b200 import HomoConfig, Homogenization_H
    shape = (16, 12, 20)
    nz, ny, nx = shape
    k, _ = random_k(shape, seed=77)
    kd = torch.from_numpy(k).cuda()
    out = []
    for fused in (False, True):
        H = Homogenization_H(HomoConfig(reso=(nx, ny, nz), femRelThres=1e-7, pre_smooth=2, post_smooth=2,
                                        precision=precision))
        H.update(kd)
        s = torch.full((nz, ny, nx + 5), 7.0, dtype=torch.float32, device="cuda")
        if fused:
            C = H.heatMatrixSensitivity(DC_TEST, s, nx + 5, True)
        else:
            C = H.heatMatrix()
            H.Sensitivity(DC_TEST, s, nx + 5, True)
        torch.cuda.synchronize()
        out.append((C, s.cpu().numpy()))
    (C1, s1), (C2, s2) = out
    assert np.array_equal(C1, C2) and np.array_equal(s1, s2)
    assert np.all(s2[:, :, nx:] == 0)
    ref = oracle_solution(k)
    assert rel_entries(C2, ref["C"]).max() <= KH_TOL
    mx, l2 = rel_field(s2[:, :, :nx], ora.sensitivity(ref["energy"], k, DC_TEST))
    assert mx <= SENS_TOL and l2 <= SENS_TOL, (mx, l2)


def test_mixed_precision_stationary_refinement():
    """The stationary form (solver "vcycle"): FP64 refinement around one 16-bit V-cycle per step."""
    k, _ = random_k((32, 32, 32), seed=33)
    H, C, E, sens = gpu_run(k, tol=1e-6, precision="bf16", solver="vcycle")
    check_against_oracle(k, C, E, sens)
    st = H.stats()
    assert st.refinements == st.iterations > 0 and max(st.rel_res) <= 1e-6


def test_pinned_host_arrays_and_copies():
    """otm_host_alloc arrays and the library's host<->device copies round-trip exactly, on the
    current stream, and report size mismatches."""
    from opentm_b200 import copy_to_device, copy_to_host, pinned_empty
    a = pinned_empty((16, 8, 4))
    a[...] = np.random.default_rng(3).random(a.shape, dtype=np.float32)
    t = torch.empty(a.shape, dtype=torch.float32, device="cuda")
    copy_to_device(t, a)
    t.mul_(2.0)
    b = pinned_empty(a.shape)
    copy_to_host(b, t)
    torch.cuda.current_stream().synchronize()
    assert np.array_equal(b, 2.0 * a)
    assert torch.from_numpy(a).is_pinned()
    with pytest.raises(ValueError):
        copy_to_device(t, pinned_empty((3,)))


@pytest.mark.parametrize("precision", ["fp32", "bf16", "fp16"])
@pytest.mark.parametrize("shape", [(32, 32, 32), (16, 16, 16), (48, 32, 64), (64, 64, 64)])
def test_tiled_smoother_matches_color_passes(precision, shape):
    """The fine level in 16^3 shared-memory tiles (one launch per smoothing leg, block Jacobi across
    tile faces) meets the oracle gates, agrees with the global colour-pair passes, and needs at most
    a few more PCG iterations."""
    nz, ny, nx = shape
    k, _ = random_k(shape, seed=60 + nx + 2 * ny + 3 * nz)
    H1, C1, E1, s1 = gpu_run(k, tol=1e-7, precision=precision, smoother="tiled")
    H2, C2, E2, s2 = gpu_run(k, tol=1e-7, precision=precision, smoother="color")
    assert rel_c(C1, C2) <= 2e-6
    assert H1.stats().iterations <= H2.stats().iterations + 3
    check_against_oracle(k, C1, E1, s1)


def test_vcycle_solver_keeps_color_passes():
    """Stationary V-cycles (MG_H::solveEquation) keep the global colour passes even when the tiled
    smoother is asked for: block Jacobi across tile faces would not damp every error mode."""
    k, _ = random_k((16, 16, 16), seed=5)
    H, C, E, sens = gpu_run(k, tol=1e-7, solver="vcycle", smoother="tiled")
    assert H.stats().smoother == 0
    check_against_oracle(k, C, E, sens)
    H, _, _, _ = gpu_run(k, tol=1e-7, smoother="tiled")
    assert H.stats().smoother == 1


def test_single_sweep_legs_keep_color_passes():
    """With one smoothing sweep per leg the tilings of the tile smoother could not alternate (the
    post leg mirrors the pre leg), so V(1,1) uses the colour passes on every level."""
    k, _ = random_k((32, 32, 32), seed=6)
    H, C, E, sens = gpu_run(k, tol=1e-7, pre=1, post=1, smoother="tiled")
    assert H.stats().smoother == 0
    check_against_oracle(k, C, E, sens)


def test_tiled_graphs_and_repeat_bitwise():
    k, _ = random_k((32, 32, 32), seed=72)
    _, C1, E1, s1 = gpu_run(k, use_graphs=True, smoother="tiled")
    _, C2, E2, s2 = gpu_run(k, use_graphs=False, smoother="tiled")
    _, C3, E3, s3 = gpu_run(k, use_graphs=True, smoother="tiled")
    assert np.array_equal(C1, C2) and np.array_equal(E1, E2) and np.array_equal(s1, s2)
    assert np.array_equal(C1, C3) and np.array_equal(s1, s3)


@pytest.mark.parametrize("smoother", ["tiled", "color"])
def test_single_v_cycle_reduces_the_residual(smoother):
    """MG_H::v_cycle through otm_homo_v_cycle: one V(2,2) cycle from a zero correction on random
    mean-free right-hand sides leaves a residual f - A u (FP64 operator of the oracle) of at most a
    third of f, for both fine smoothers; the level description names the smoother."""
    from opentm_b200 import HomoConfig, Homogenization_H
    n = 32
    k = (0.5 + 0.5 * wl.uniform(81, n ** 3)).astype(np.float32).reshape(n, n, n)
    H = Homogenization_H(HomoConfig(reso=n, femRelThres=1e-6, pre_smooth=2, post_smooth=2, smoother=smoother))
    H.update(torch.from_numpy(k).cuda())
    f = np.random.default_rng(1).standard_normal((3, n, n, n)).astype(np.float32)
    f -= f.mean(axis=(1, 2, 3), keepdims=True)
    u = H.v_cycle(torch.from_numpy(f).cuda(), pre=2, post=2).cpu().numpy().astype(np.float64)
    ks = 1e-9 + k.astype(np.float64)
    for c in range(3):
        r = f[c] - ora.apply(ks, u[c])
        assert np.linalg.norm(r) <= np.linalg.norm(f[c]) / 3.0, (c, np.linalg.norm(r) / np.linalg.norm(f[c]))
    info = H.level(0)
    assert info.levels == H.stats().levels and list(info.reso) == [n, n, n] and info.stencil == 0
    assert info.smoother == (1 if smoother == "tiled" else 0)
