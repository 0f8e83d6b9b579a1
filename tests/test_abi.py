"""CPU tests of the C ABI library: it loads without a GPU, exports every symbol the public
headers declare, and its host-side argument checks answer without touching the device."""
import ctypes
import os

import pytest

from opentm_b200 import _lib


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = _lib.header_symbols()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_signatures_cover_headers():
    # every declared entry point has a ctypes signature in the Python binding
    names = set(_lib.header_symbols())
    assert names <= set(_lib.SIGNATURES), sorted(names - set(_lib.SIGNATURES))


def test_config_defaults_mirror_homoconfig():
    cfg = _lib.default_config()
    assert list(cfg.reso) == [128, 128, 128]      # cmdline.cpp:6-8
    assert cfg.fem_rel_thres == pytest.approx(0.01)  # cmdline.cpp:28
    assert cfg.max_iter == 200                    # MG.cpp:382
    assert cfg.pre_smooth == 1 and cfg.post_smooth == 1
    assert cfg.power_penal == pytest.approx(1.0)
    assert cfg.warm_start == 1


def test_status_strings_and_version():
    L = _lib.lib()
    assert L.otm_abi_version() == 2
    assert L.otm_status_string(0) == b"ok"
    assert L.otm_status_string(5) == b"not converged"


@pytest.mark.parametrize("kw,status", [
    (dict(reso=(2048, 16, 16)), 2),          # > 1024 per axis (grid.cpp:23-25)
    (dict(reso=(16, 16, 16), max_iter=0), 1),
    (dict(reso=(16, 16, 16), pre_smooth=0, post_smooth=0), 1),
    (dict(reso=(16, 16, 16), pre_smooth=1, post_smooth=2), 1),  # PCG needs a symmetric cycle
    (dict(reso=(16, 16, 16), solver=7), 1),
    (dict(reso=(16, 16, 16), precision=9), 1),
    (dict(reso=(1024, 1024, 4)), 2),          # coarsest level too large for the dense solve
])
def test_create_rejects_bad_configs_before_touching_the_device(kw, status):
    reso = kw.pop("reso")
    cfg = _lib.default_config(reso, **kw)
    h = ctypes.c_void_p()
    assert _lib.lib().otm_homo_create(ctypes.byref(cfg), ctypes.byref(h)) == status
    assert not h.value


def test_null_handles_are_rejected():
    L = _lib.lib()
    assert L.otm_homo_update(None, None, 0) == 1
    assert L.otm_homo_destroy(None) == 1
    assert L.otm_oc_update(0, None, None, 0.3, 0.001, 0.02, 0.5, None, None) == 1


def test_filter_rejects_bad_radius_without_device():
    L = _lib.lib()
    dummy = ctypes.c_void_p(16)
    st = L.otm_filter_forward(_lib.i3((8, 8, 8)), dummy, -1, dummy, -1, None, 1, ctypes.c_float(9.0), 1, None)
    assert st == 2  # half width above the supported 6
    st = L.otm_filter_forward(_lib.i3((8, 8, 8)), dummy, -1, dummy, -1, None, 5, ctypes.c_float(2.0), 1, None)
    assert st == 1
