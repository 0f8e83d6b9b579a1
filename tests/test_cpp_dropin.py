"""The C++ drop-in header compiles against the library (CPU test) and, on a GPU, reproduces the
Python path's K^H (GPU test)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "dropin_main.cpp")
CUDA = "/usr/local/cuda"


def _build(tmp_path):
    exe = os.path.join(str(tmp_path), "dropin")
    gxx = shutil.which("g++")
    cmd = [gxx, "-std=c++17", "-O2", SRC, "-o", exe, "-I", os.path.join(ROOT, "include"), "-I",
           os.path.join(CUDA, "include"), "-L", os.path.join(ROOT, "opentm_b200"), "-lopentm_b200",
           "-Wl,-rpath," + os.path.join(ROOT, "opentm_b200"), "-L", os.path.join(CUDA, "lib64"), "-lcudart",
           "-Wl,-rpath," + os.path.join(CUDA, "lib64")]
    subprocess.run(cmd, check=True)
    return exe


def test_dropin_header_compiles_and_links(tmp_path):
    exe = _build(tmp_path)
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_dropin_program_matches_python_path(tmp_path):
    import torch

    from opentm_b200 import HomoConfig, Homogenization_H
    from opentm_b200 import workloads as wl
    exe = _build(tmp_path)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    vals = {l.split()[0]: [float(v) for v in l.split()[1:]] for l in out.strip().splitlines() if l != "ok"}
    n = 16
    rho = (0.001 + 0.999 * wl.uniform(0, n ** 3)).astype(np.float32)
    k = (1e-3 + rho * rho * rho * (1 - 1e-3)).astype(np.float32).reshape(n, n, n)
    H = Homogenization_H(HomoConfig(reso=n, femRelThres=1e-6, pre_smooth=2, post_smooth=2))
    H.update(torch.from_numpy(k).cuda())
    C = H.heatMatrix()
    got = np.array(vals["C"])
    want = np.array([C[0, 0], C[0, 1], C[0, 2], C[1, 1], C[1, 2], C[2, 2]])
    # the C++ program forms k in float arithmetic, numpy in double: inputs differ in the last
    # bits, so the two solves agree to the solver tolerance, not bitwise
    assert np.abs(got - want).max() / np.abs(want).max() <= 1e-6
    assert vals["relres"][0] <= 1e-7
    assert vals["fused_same"] == [1.0]  # heatMatrix(C, dC, sens, ...) == heatMatrix + Sensitivity, bit for bit
    # same OC inputs through the oracle: filtered sensitivities, then the 20-step bisection
    import oracle as ora
    n3 = n ** 3
    g = -(0.1 + wl.uniform(0, 2 * n3)[n3:].astype(np.float32)).reshape(n, n, n)
    s = ora.oc_filter_sens(g, np.full((n, n, n), 0.3), 2.0)
    want_vol = ora.oc_update(s, np.full((n, n, n), 0.3), 0.25, 0.001, 0.2, 0.5)[0].mean()
    assert abs(vals["oc_vol"][0] - want_vol) <= 1e-5
    assert abs(vals["mma_mean"][0] - 0.3) <= 2e-3
    # runCustom through the C++ layer equals the Python driver bit for bit (same library calls)
    from opentm_b200.driver import DesignConfig, InitWay, Model, run_custom
    rho, _ = run_custom(DesignConfig(reso=16, max_iter=2, heatRatio=(1.0, 1e-4), winit=InitWay.IWP, model=Model.oc))
    assert vals["design_sum"][0] == pytest.approx(float(rho.astype(np.float64).sum()), rel=1e-9)
    assert vals["governor"] == [pytest.approx(0.25, abs=1e-7), 0.0]
    # heat_tensor_t eval / backward = density filter -> update -> heatMatrix -> Sensitivity -> filter
    # adjoint through the Python path on the same density (the same library calls)
    from opentm_b200 import DensityFilter
    rho_h = wl.uniform(0, 6 * n3)[5 * n3:].astype(np.float32).reshape(n, n, n)
    df = DensityFilter((n, n, n), 2.0, 1, True, 3.0, 1.0, 1e-3)
    H2 = Homogenization_H(HomoConfig(reso=n, femRelThres=1e-6, pre_smooth=2, post_smooth=2))
    H2.update(df.forward(torch.from_numpy(rho_h).cuda()))
    C2 = H2.heatMatrix()
    g_k = torch.empty((n, n, n), dtype=torch.float32, device="cuda")
    H2.Sensitivity(-np.eye(3), g_k)
    g_rho = df.backward(g_k)
    want = [C2[0, 0], C2[0, 1], C2[0, 2], C2[1, 1], C2[1, 2], C2[2, 2]]
    assert np.allclose(vals["ht_C"], want, rtol=1e-7, atol=1e-12)
    assert vals["ht_grad_sum"][0] == pytest.approx(float(g_rho.double().sum()), rel=1e-6)
    # MG_H: one V(2,2) cycle on the same right-hand sides
    lv = [H2.level(l) for l in range(H2.level(0).levels)]
    assert vals["mg_levels"] == [len(lv), n, 1.0]
    f = (wl.uniform(0, 10 * n3)[7 * n3:].astype(np.float32) - np.float32(0.5)).reshape(3, n, n, n)
    u = H2.v_cycle(torch.from_numpy(f).cuda(), pre=2, post=2)
    assert vals["vc_norm"][0] == pytest.approx(float(u.double().norm()), rel=1e-6)
