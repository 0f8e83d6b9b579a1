"""GPU parity of the FP64 device MMA (mmasubDevice / MMAOptimizer) against the oracle's
restatement of the same algorithm."""
import ctypes

import numpy as np
import pytest

import oracle as ora
from opentm_b200 import _lib
from opentm_b200 import workloads as wl

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

MMA_TOL = 1e-7  # FP64 device vs FP64 host, max |dx| after each step (different summation order)


def _problem(n, m, seed):
    t = wl.uniform(seed, n)
    w = 0.5 + wl.uniform(seed + 1, n)
    A = 0.5 + wl.uniform(seed + 2, m * n).reshape(m, n)
    return t, w, A


def test_mmasub_device_matches_oracle():
    n, m = 3000, 2
    t, w, A = _problem(n, m, 40)
    V = np.array([0.3 * n, 0.35 * n])
    x = np.full(n, 0.5)
    xmin, xmax = np.zeros(n), np.ones(n)
    st = dict(x=x.copy(), o1=x.copy(), o2=x.copy(), lo=xmin.copy(), up=xmax.copy())
    dev = {k: torch.from_numpy(v.copy()).cuda() for k, v in st.items()}
    dmin, dmax = torch.from_numpy(xmin).cuda(), torch.from_numpy(xmax).cuda()
    a = np.zeros(m)
    c = np.full(m, 1e3)
    d = np.ones(m)
    da, dc, dd = (torch.from_numpy(v).cuda() for v in (a, c, d))
    L = _lib.lib()
    for it in range(1, 8):
        xc = st["x"]
        df = 2 * w * (xc - t)
        g = (A @ xc) / V - 1.0
        dg = A / V[:, None]
        st["x"], st["o1"], st["o2"], st["lo"], st["up"] = ora.mmasub(
            it, xc, xmin, xmax, st["o1"], st["o2"], df, g, dg, st["lo"], st["up"], 1.0, a, c, d, 1.0)
        xd = dev["x"].cpu().numpy()
        ddf = torch.from_numpy(2 * w * (xd - t)).cuda()
        dgv = torch.from_numpy((A @ xd) / V - 1.0).cuda()
        dgd = torch.from_numpy(np.ascontiguousarray(A / V[:, None])).cuda()
        pp = _lib.PitchedPtr(dgd.data_ptr(), n * 8, n * 8, m)
        P = ctypes.c_void_p
        s = L.otm_mmasub_device(m, n, it, P(dev["x"].data_ptr()), P(dmin.data_ptr()), P(dmax.data_ptr()),
                                P(dev["o1"].data_ptr()), P(dev["o2"].data_ptr()), 1.0, P(ddf.data_ptr()),
                                P(dgv.data_ptr()), pp, P(dev["lo"].data_ptr()), P(dev["up"].data_ptr()), 1.0,
                                P(da.data_ptr()), P(dc.data_ptr()), P(dd.data_ptr()), 1.0,
                                P(torch.cuda.current_stream().cuda_stream))
        assert s == 0, _lib.last_error()
        torch.cuda.synchronize()
        for k in ("x", "lo", "up"):
            assert np.abs(dev[k].cpu().numpy() - st[k]).max() <= MMA_TOL, (it, k)


def test_mma_optimizer_float_interface():
    from opentm_b200 import MMAOptimizer
    n = 4096
    t, w, A = _problem(n, 1, 50)
    V = 0.3 * n
    mma = MMAOptimizer(1, n, 1.0, 0.0, 1e3, 1.0)
    mma.setBound(0.0, 1.0)
    x = torch.full((n,), 0.5, dtype=torch.float32, device="cuda")
    xr = np.full(n, 0.5)
    o1, o2, lo, up = xr.copy(), xr.copy(), np.zeros(n), np.ones(n)
    for it in range(1, 6):
        xd = x.double().cpu().numpy()
        df = torch.from_numpy((2 * w * (xd - t)).astype(np.float32)).cuda()
        dg = torch.from_numpy((A[0] / V).astype(np.float32)).cuda()
        g = [float(A[0] @ xd / V - 1.0)]
        mma.update(it, x, df, g, [dg])
        xr, o1, o2, lo, up = ora.mmasub(it, xd, np.zeros(n), np.ones(n), o1, o2,
                                        (2 * w * (xd - t)).astype(np.float32).astype(np.float64),
                                        np.array([np.float32(g[0])], dtype=np.float64),
                                        (A[0:1] / V).astype(np.float32).astype(np.float64), lo, up, 1.0,
                                        np.zeros(1), np.full(1, 1e3), np.ones(1), 1.0)
        torch.cuda.synchronize()
        assert np.abs(x.cpu().numpy() - xr).max() <= 1e-6
