"""GPU parity of the design driver against its restatement (oracle/driver.py): initial fields,
symmetrisation (bit for bit), the random trigonometric basis, and the runCustom loop for both
models against the FP64 oracle loop.

Tolerances: closed-form fields 1e-4 absolute (CUDA's cosf / tanhf against numpy's float32 ones,
amplified by the tanh projection's slope of at most 10); random-basis fields 2e-3 absolute
(FP32 products against FP64); design loop: objective history 2e-4 relative, densities 2e-3
absolute after the iterations run (FP32 solves to 1e-6 against FP64 to 1e-10)."""
import numpy as np
import pytest

from oracle import driver as od

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _cfg(**kw):
    from opentm_b200.driver import DesignConfig
    return DesignConfig(**kw)


def _init(cfg):
    from opentm_b200.driver import init_density
    out = torch.empty((cfg.reso,) * 3, dtype=torch.float32, device="cuda")
    co = init_density(cfg, out)
    return out.cpu().numpy(), co


@pytest.mark.parametrize("way", [od.INIT_P, od.INIT_G, od.INIT_D, od.INIT_IWP, od.INIT_EXAMPLE])
@pytest.mark.parametrize("n", [16, 15])
def test_closed_form_initial_fields(way, n):
    got, _ = _init(_cfg(reso=n, winit=way))
    ref = od.init_density(way, n)
    assert np.abs(got - ref).max() <= 1e-4


def test_noise_initial_field_with_symmetry():
    got, _ = _init(_cfg(reso=16, winit=od.INIT_NOISE, sym=od.SYM_REFLECT3, seed=7, volRatio=0.35))
    ref = od.init_density(od.INIT_NOISE, 16, sym=od.SYM_REFLECT3, vol=0.35, seed=7)
    assert np.abs(got - ref).max() <= 1e-6


@pytest.mark.parametrize("way", [od.INIT_RANDOM, od.INIT_RANDCENTER])
def test_random_basis_initial_fields(way):
    got, co = _init(_cfg(reso=16, winit=way, initperiod=3, seed=11, volRatio=0.3))
    ref_co = od.randtri_coefficients(11, 3, way != od.INIT_RANDOM)
    assert np.array_equal(co, ref_co)
    ref = od.init_density(way, 16, vol=0.3, n_period=3, seed=11)
    assert np.abs(got - ref).max() <= 2e-3
    # before the clamp to [0.1, 1] the level set meets the volume ratio to 1e-3
    assert got.min() >= np.float32(0.1)


def test_randtri_field_default_period():
    from opentm_b200.driver import randtri_coefficients, randtri_field
    co = randtri_coefficients(3, 10, True)
    f = torch.empty((12, 12, 12), dtype=torch.float32, device="cuda")
    randtri_field(f, 10, co, True)
    torch.cuda.synchronize()
    ref = od.randtri_field(12, 10, co, True)
    assert np.abs(f.cpu().numpy() - ref).max() <= 2e-3 * max(1.0, np.abs(ref).max() / 10)


@pytest.mark.parametrize("sym", [od.SYM_REFLECT3, od.SYM_REFLECT6, od.SYM_ROTATE3, od.SYM_ROTATE2])
@pytest.mark.parametrize("shape", [(16, 16, 16), (10, 10, 10), (15, 15, 15), (12, 10, 8)])
def test_symmetrize_bitwise(sym, shape):
    from opentm_b200 import OtmError
    from opentm_b200.driver import symmetrize
    cube = shape[0] == shape[1] == shape[2]
    f = np.random.default_rng(sum(shape) + sym).random(shape, dtype=np.float32)
    t = torch.from_numpy(f).cuda()
    if (sym == od.SYM_REFLECT6 and not cube) or (sym == od.SYM_ROTATE3 and (not cube or shape[0] % 2)):
        with pytest.raises(OtmError):
            symmetrize(t, sym)
        return
    symmetrize(t, sym)
    torch.cuda.synchronize()
    assert np.array_equal(t.cpu().numpy(), od.symmetrize(f, sym))


def test_symmetrize_without_average():
    from opentm_b200.driver import symmetrize
    f = np.random.default_rng(5).random((9, 8, 7), dtype=np.float32)
    for sym in (od.SYM_REFLECT3, od.SYM_ROTATE2):
        t = torch.from_numpy(f).cuda()
        symmetrize(t, sym, average=False)
        torch.cuda.synchronize()
        assert np.array_equal(t.cpu().numpy(), od.symmetrize(f, sym, average=False))


def _rho0(n):
    return od.init_density(od.INIT_P, n)


@pytest.mark.parametrize("model,sym", [("oc", od.SYM_NONE), ("oc", od.SYM_REFLECT3), ("mma", od.SYM_NONE)])
def test_design_loop_matches_oracle(model, sym):
    from opentm_b200.driver import Model, run_custom
    n, iters = 16, 4
    rho0 = _rho0(n)
    tt = (0.3, 0.2, 0.1, 0.02, 0.01, 0.01)
    cfg = _cfg(reso=n, model=Model.oc if model == "oc" else Model.mma, max_iter=iters, femRelThres=1e-6,
               heatRatio=(1.0, 1e-3), target_tensor=tt, sym=sym)
    rho, info = run_custom(cfg, rho0=rho0)
    ref_rho, ref_hist = od.run_custom(rho0, model, heat_ratio=(1.0, 1e-3), target=tt, iters=iters, sym=sym)
    assert info["iterations"] == iters == len(ref_hist)
    assert np.allclose(info["history"], ref_hist, rtol=2e-4, atol=1e-7), (info["history"], ref_hist)
    assert np.abs(rho - ref_rho).max() <= 2e-3
    assert abs(info["volume"] - rho.astype(np.float64).mean()) <= 1e-6


def test_run_custom_from_init_and_outputs(tmp_path):
    from opentm_b200 import driver as dr
    n = 16
    cfg = _cfg(reso=n, winit=od.INIT_RANDCENTER, initperiod=2, seed=4, max_iter=2, femRelThres=1e-6,
               outprefix=str(tmp_path) + "/")
    rho, info = dr.run_custom(cfg)
    co = dr.read_vectors(str(tmp_path / "coeff"))[0]
    assert np.array_equal(co, od.randtri_coefficients(4, 2, True))
    init = dr.read_density_binary(str(tmp_path / "init_rand"))
    ref_init = od.init_density(od.INIT_RANDCENTER, n, n_period=2, seed=4)
    assert np.abs(init - ref_init).max() <= 2e-3
    assert np.array_equal(dr.read_density_binary(str(tmp_path / f"density{n}")), rho)
    assert (tmp_path / "oc_v_log.txt").exists() and info["iterations"] == 2
    # the same coefficients read back from the file reproduce the initial field
    cfg2 = _cfg(reso=n, winit=od.INIT_REP_RANDCENTER, initperiod=2, inputrho=str(tmp_path / "coeff"))
    again, _ = _init(cfg2)
    assert np.array_equal(again, init)
    # manual: the density file itself
    cfg3 = _cfg(reso=n, winit=od.INIT_MANUAL, inputrho=str(tmp_path / "init_rand"))
    manual, _ = _init(cfg3)
    assert np.array_equal(manual, np.clip(init, 0.1, 1.0))


def test_openTM_entry_points():
    from opentm_b200 import openTM
    rho = openTM.runInstance(16, [1, 1e-3], [0.3, 0.2, 0.1, 0.0, 0.0, 0.0], openTM.InitWay.IWP, openTM.Model.oc,
                             max_iter=2)
    assert len(rho) == 16 ** 3 and min(rho) >= 0.001 and max(rho) <= 1.0
    h = openTM.homo()
    h.setConfig(16, [1, 1e-3], [0.3, 0.2, 0.1, 0.0, 0.0, 0.0], openTM.Model.mma)
    h.config.max_iter = 2
    h.setDensity(rho)
    out = h.optimize()
    assert len(out) == 16 ** 3 and h.info["iterations"] == 2
    assert min(out) >= 1e-4 - 1e-7 and max(out) <= 1.0


def test_unsupported_initialisation():
    from opentm_b200 import OtmError
    with pytest.raises(OtmError) as ei:
        _init(_cfg(reso=16, winit=od.INIT_INTERP))
    assert ei.value.status == 2  # OTM_ERR_UNSUPPORTED
