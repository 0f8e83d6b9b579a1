"""The design driver around the homogenization path (include/opentm_b200_driver.h).

Initial densities (initDensity, Framework.cu:63-145; randTri, homogenization/Framework.cuh:237-310),
field symmetrisation (AutoDiff/TensorExpression.cuh:70-280), the tensor-matching loop (runCustom,
Framework.cu:147-244) with its convergence test and volume governor (Framework.cuh:312-411), and
the driver's file formats (homogenization/utils.h:47-91, grid.cpp:336-344, homoExpression.h:130-146).
Device fields are CUDA tensors of shape (nz, ny, nx), x fastest.
"""
from __future__ import annotations

import ctypes
import enum
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check, i3, lib


class Symmetry(enum.IntEnum):
    """cfg::Symmetry (cmdline.h:9)."""
    reflect3 = 0
    reflect6 = 1
    rotate3 = 2
    rotate2 = 3
    NONE = 4


class InitWay(enum.IntEnum):
    """cfg::InitWay (cmdline.h:10)."""
    random = 0
    randcenter = 1
    noise = 2
    manual = 3
    interp = 4
    rep_randcenter = 5
    P = 6
    G = 7
    D = 8
    IWP = 9
    example = 10


class Model(enum.IntEnum):
    """cfg::Model (cmdline.h:11)."""
    mma = 0
    oc = 1


@dataclass
class DesignConfig:
    """The cfg::HomoConfig fields the driver reads (cmdline.h:12-33) with HomoConfig::init()
    defaults (cmdline.cpp:4-35); `seed` selects the random stream of the random initialisers."""
    reso: int = 128
    sym: Symmetry = Symmetry.NONE
    winit: InitWay = InitWay.IWP
    model: Model = Model.oc
    volRatio: float = 0.3
    heatRatio: tuple = (1.0, 0.0)
    finthres: float = 5e-4
    femRelThres: float = 0.01
    target_tensor: tuple = (0.3, 0.2, 0.1, 0.0, 0.0, 0.0)
    max_iter: int = 500
    initperiod: int = 10
    seed: int = 0
    inputrho: str | None = None
    outprefix: str | None = None

    def to_c(self) -> tuple[_lib.DriverConfig, list]:
        c = _lib.DriverConfig()
        check(lib().otm_driver_config_init(ctypes.byref(c)), "otm_driver_config_init")
        c.reso = int(self.reso)
        c.sym = int(self.sym)
        c.winit = int(self.winit)
        c.model = int(self.model)
        c.vol_ratio = float(self.volRatio)
        if len(self.heatRatio) != 2:
            raise ValueError("heatRatio needs 2 values")
        if len(self.target_tensor) != 6:
            raise ValueError("target_tensor needs 6 values")
        for i in range(2):
            c.heat_ratio[i] = float(self.heatRatio[i])
        for i in range(6):
            c.target_tensor[i] = float(self.target_tensor[i])
        c.finthres = float(self.finthres)
        c.fem_rel_thres = float(self.femRelThres)
        c.max_iter = int(self.max_iter)
        c.init_period = int(self.initperiod)
        c.seed = int(self.seed)
        keep = []  # the encoded strings must outlive the call
        if self.inputrho is not None:
            keep.append(str(self.inputrho).encode())
            c.input_path = keep[-1]
        if self.outprefix is not None:
            keep.append(str(self.outprefix).encode())
            c.output_prefix = keep[-1]
        return c, keep


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _dev(t) -> int:
    if not getattr(t, "is_cuda", False):
        raise ValueError("device fields must be CUDA tensors")
    return t.data_ptr()


def _stream(stream=None) -> int:
    if stream is not None:
        return stream if isinstance(stream, int) else stream.cuda_stream
    import torch
    return torch.cuda.current_stream().cuda_stream


def run_custom(config: DesignConfig, rho0=None):
    """runCustom: returns (rho as a float32 array (n, n, n), info) where info holds iterations,
    converged, objective, volume, volume_bound, K (3x3) and history (objective per iteration)."""
    c, keep = config.to_c()
    n = int(config.reso)
    rho_out = np.empty((n, n, n), dtype=np.float32)
    hist = np.zeros(max(int(config.max_iter), 1), dtype=np.float64)
    r0 = None
    if rho0 is not None:
        r0 = np.ascontiguousarray(np.asarray(rho0, dtype=np.float32).reshape(n, n, n))
    res = _lib.DriverResult()
    check(lib().otm_run_custom(ctypes.byref(c), _fptr(r0) if r0 is not None else None, _fptr(rho_out),
                               hist.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(res)),
          "otm_run_custom")
    del keep
    info = {"iterations": res.iterations, "converged": bool(res.converged), "objective": res.objective,
            "volume": res.volume, "volume_bound": res.volume_bound,
            "K": np.array(res.K[:], dtype=np.float32).reshape(3, 3), "history": hist[:res.iterations].copy(),
            "init_seconds": res.init_seconds, "loop_seconds": res.loop_seconds}
    return rho_out, info


def init_density(config: DesignConfig, out, stream=None):
    """initDensity into the CUDA tensor `out` (reso^3 values); returns the random-basis
    coefficients for the random forms, else None. Waits for the work."""
    c, keep = config.to_c()
    co = None
    if config.winit in (InitWay.random, InitWay.randcenter, InitWay.rep_randcenter):
        co = np.zeros(randtri_coeff_count(config.initperiod, config.winit != InitWay.random), dtype=np.float32)
    check(lib().otm_init_density(ctypes.byref(c), ctypes.c_void_p(_dev(out)), int(config.reso),
                                 _fptr(co) if co is not None else None, ctypes.c_void_p(_stream(stream))),
          "otm_init_density")
    del keep
    return co


def symmetrize(field, sym: Symmetry, average: bool = True, stream=None):
    """Tensor::symmetrize on a CUDA tensor of shape (nz, ny, nx), in place."""
    nz, ny, nx = field.shape
    check(lib().otm_symmetrize(i3((nx, ny, nz)), ctypes.c_void_p(_dev(field)), nx, int(sym), int(bool(average)),
                               ctypes.c_void_p(_stream(stream))), "otm_symmetrize")


def randtri_coeff_count(n_period: int, centered: bool) -> int:
    return int(lib().otm_randtri_coeff_count(int(n_period), int(bool(centered))))


def randtri_coefficients(seed: int, n_period: int, centered: bool) -> np.ndarray:
    co = np.zeros(randtri_coeff_count(n_period, centered), dtype=np.float32)
    check(lib().otm_randtri_coefficients(int(seed), int(n_period), int(bool(centered)), _fptr(co)),
          "otm_randtri_coefficients")
    return co


def randtri_field(field, n_period: int, coeffs, centered: bool, stream=None):
    """The random trigonometric basis sum into a CUDA tensor of shape (nz, ny, nx)."""
    nz, ny, nx = field.shape
    co = np.ascontiguousarray(np.asarray(coeffs, dtype=np.float32))
    if co.size < randtri_coeff_count(n_period, centered):
        raise ValueError("too few coefficients")
    check(lib().otm_randtri_field(i3((nx, ny, nz)), ctypes.c_void_p(_dev(field)), nx, int(n_period), _fptr(co),
                                  int(bool(centered)), ctypes.c_void_p(_stream(stream))), "otm_randtri_field")


class ConvergeChecker:
    """ConvergeChecker (Framework.cuh:312-345)."""

    def __init__(self, thres: float = 1e-3):
        self._c = _lib.ConvergeChecker()
        lib().otm_converge_checker_init(ctypes.byref(self._c), float(thres))

    def is_converge(self, iter: int, obj: float) -> bool:
        return bool(lib().otm_converge_checker_step(ctypes.byref(self._c), int(iter), float(obj)))


class VolumeGovernor:
    """VolumeGovernor (Framework.cuh:347-411)."""

    def __init__(self):
        self._g = _lib.VolumeGovernor()
        lib().otm_volume_governor_init(ctypes.byref(self._g))

    def get_volume_bound(self) -> float:
        return float(self._g.volume_bound)

    def volume_check(self, value: float, low_bound: float, volfrac: float, itn: int) -> int:
        return int(lib().otm_volume_governor_check(ctypes.byref(self._g), float(value), float(low_bound),
                                                   float(volfrac), int(itn)))

    def get_current_decrease(self) -> float:
        return float(lib().otm_volume_governor_decrease(ctypes.byref(self._g)))


def write_density_binary(path: str, rho: np.ndarray):
    """Grid_H::writeDensity binary form: int32 (nx, ny, nz), then the densities, x fastest."""
    r = np.ascontiguousarray(np.asarray(rho, dtype=np.float32))
    nz, ny, nx = r.shape
    check(lib().otm_write_density_binary(str(path).encode(), i3((nx, ny, nz)), _fptr(r)), "otm_write_density_binary")


def read_density_binary(path: str) -> np.ndarray:
    reso = (ctypes.c_int * 3)()
    check(lib().otm_read_density_binary(str(path).encode(), reso, None, 0), "otm_read_density_binary")
    out = np.empty((reso[2], reso[1], reso[0]), dtype=np.float32)
    check(lib().otm_read_density_binary(str(path).encode(), reso, _fptr(out), out.size), "otm_read_density_binary")
    return out


def write_vectors(path: str, vecs) -> None:
    """homoutils::writeVectors: equal-length vectors interleaved element by element."""
    arrs = [np.ascontiguousarray(np.asarray(v, dtype=np.float32)) for v in vecs]
    if not arrs or any(a.size != arrs[0].size for a in arrs):
        raise ValueError("vectors must be non-empty and of equal length")
    ptrs = (ctypes.POINTER(ctypes.c_float) * len(arrs))(*[_fptr(a) for a in arrs])
    check(lib().otm_write_vectors(str(path).encode(), len(arrs), arrs[0].size, ptrs), "otm_write_vectors")


def read_vectors(path: str, n_vec: int = 1) -> list[np.ndarray]:
    n = ctypes.c_size_t(0)
    check(lib().otm_read_vectors(str(path).encode(), int(n_vec), ctypes.byref(n), None, 0), "otm_read_vectors")
    arrs = [np.empty(n.value, dtype=np.float32) for _ in range(n_vec)]
    ptrs = (ctypes.POINTER(ctypes.c_float) * n_vec)(*[_fptr(a) for a in arrs])
    check(lib().otm_read_vectors(str(path).encode(), int(n_vec), ctypes.byref(n), ptrs, n.value), "otm_read_vectors")
    return arrs


def write_heat_matrix(path: str, K, text: bool = False) -> None:
    """heat_tensor_t::writeTo (9 raw float32) or writeToTxt."""
    k = np.ascontiguousarray(np.asarray(K, dtype=np.float32).reshape(9))
    check(lib().otm_write_heat_matrix(str(path).encode(), _fptr(k), int(bool(text))), "otm_write_heat_matrix")
