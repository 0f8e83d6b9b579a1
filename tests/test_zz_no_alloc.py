"""GPU test of otm_oc_filter_sens_noalloc, the filter entry point that allocates no device
memory (for callers whose allocator already owns the GPU's memory, or whose loop may not call
cudaMalloc/cudaFree). Called through the C ABI twice in a row; each call must give the same
result as the allocating otm_oc_filter_sens on the same input, within the filter tolerance
used by the other filter tests, and must take nothing from the library's scratch memory pool.
The file name sorts last so that a run that stops at the first failure has already run every
other test."""
import ctypes

import numpy as np
import pytest

from opentm_b200 import _lib
from opentm_b200 import workloads as wl

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

FILTER_TOL = 1e-5


def _call(fn, sens, rho, reso):
    L = _lib.lib()
    return getattr(L, fn)(ctypes.c_void_p(sens.data_ptr()), ctypes.c_void_p(rho.data_ptr()), reso[0],
                          _lib.i3(reso), ctypes.c_float(2.0),
                          ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))


@pytest.mark.parametrize("n", [24, 40])
def test_noalloc_filter_matches_allocating_filter_twice(n):
    L = _lib.lib()
    for call in range(2):  # the second call reuses the scratch array the first one left behind
        rho = (0.1 + 0.9 * wl.uniform(200 + 10 * call + n, n ** 3)).reshape(n, n, n).astype(np.float32)
        sens = -wl.uniform(300 + 10 * call + n, n ** 3).reshape(n, n, n).astype(np.float32)
        r = torch.from_numpy(rho).cuda()
        a = torch.from_numpy(sens).cuda()
        b = a.clone()
        assert _call("otm_oc_filter_sens", a, r, (n, n, n)) == 0, _lib.last_error()
        torch.cuda.synchronize()
        before = L.otm_scratch_alloc_count()
        assert _call("otm_oc_filter_sens_noalloc", b, r, (n, n, n)) == 0, _lib.last_error()
        torch.cuda.synchronize()
        assert L.otm_scratch_alloc_count() == before, "the allocation-free filter took scratch memory"
        x, y = a.cpu().numpy(), b.cpu().numpy()
        assert np.abs(x - y).max() <= FILTER_TOL * np.abs(x).max()


def test_allocating_filter_is_seen_by_the_counter():
    """The counter the test above relies on does move for the allocating entry point."""
    L = _lib.lib()
    n = 16
    r = torch.full((n, n, n), 0.5, device="cuda")
    a = torch.full((n, n, n), -1.0, device="cuda")
    before = L.otm_scratch_alloc_count()
    assert _call("otm_oc_filter_sens", a, r, (n, n, n)) == 0, _lib.last_error()
    torch.cuda.synchronize()
    assert L.otm_scratch_alloc_count() > before


def test_noalloc_rejects_cells_above_the_limit():
    # real device buffers of the rejected size: if the size check ever ran after a launch, the
    # kernels would still stay inside these arrays
    reso = (129, 128, 128)
    rho = torch.full(reso[::-1], 0.5, device="cuda")
    sens = torch.full(reso[::-1], -1.0, device="cuda")
    keep = sens.clone()
    st = _call("otm_oc_filter_sens_noalloc", sens, rho, reso)
    torch.cuda.synchronize()
    assert st == 2  # OTM_ERR_UNSUPPORTED: more than OTM_NOALLOC_MAX_CELLS voxels
    assert "OTM_NOALLOC_MAX_CELLS" in _lib.last_error()
    assert torch.equal(sens, keep)  # nothing was written
