"""GPU test of otm_oc_filter_sens_noalloc, the filter entry point that allocates no device
memory (for callers whose allocator already owns the GPU's memory, or whose loop may not call
cudaMalloc/cudaFree). Called through the C ABI twice in a row; each call must give the same
result as the allocating otm_oc_filter_sens on the same input, within the filter tolerance
used by the other filter tests. The file name sorts last so that a run that stops at the
first failure has already run every other test."""
import ctypes

import numpy as np
import pytest

from opentm_b200 import _lib
from opentm_b200 import workloads as wl

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

FILTER_TOL = 1e-5


def _call(fn, sens, rho, n):
    L = _lib.lib()
    s = getattr(L, fn)(ctypes.c_void_p(sens.data_ptr()), ctypes.c_void_p(rho.data_ptr()), n, _lib.i3((n, n, n)),
                       ctypes.c_float(2.0), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert s == 0, _lib.last_error()


@pytest.mark.parametrize("n", [24, 40])
def test_noalloc_filter_matches_allocating_filter_twice(n):
    for call in range(2):  # the second call reuses the scratch array the first one left behind
        rho = (0.1 + 0.9 * wl.uniform(200 + 10 * call + n, n ** 3)).reshape(n, n, n).astype(np.float32)
        sens = -wl.uniform(300 + 10 * call + n, n ** 3).reshape(n, n, n).astype(np.float32)
        r = torch.from_numpy(rho).cuda()
        a = torch.from_numpy(sens).cuda()
        b = a.clone()
        _call("otm_oc_filter_sens", a, r, n)
        _call("otm_oc_filter_sens_noalloc", b, r, n)
        torch.cuda.synchronize()
        x, y = a.cpu().numpy(), b.cpu().numpy()
        assert np.abs(x - y).max() <= FILTER_TOL * np.abs(x).max()


def test_noalloc_rejects_cells_above_the_limit():
    L = _lib.lib()
    dummy = ctypes.c_void_p(256)
    st = L.otm_oc_filter_sens_noalloc(dummy, dummy, 0, _lib.i3((129, 128, 128)), ctypes.c_float(2.0), None)
    assert st == 2  # OTM_ERR_UNSUPPORTED: more than OTM_NOALLOC_MAX_CELLS voxels
    assert "OTM_NOALLOC_MAX_CELLS" in _lib.last_error()
