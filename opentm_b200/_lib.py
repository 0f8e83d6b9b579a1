"""ctypes binding of ``libopentm_b200.so`` (the C ABI declared in include/opentm_b200*.h).

The library is loaded from the package directory. If it is missing the import of the
product entry points fails loudly: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "libopentm_b200.so")
HEADERS = [os.path.join(ROOT, "include", f)
           for f in ("opentm_b200.h", "opentm_b200_mma.h", "opentm_b200_server.h", "opentm_b200_noalloc.h",
                     "opentm_b200_driver.h")]

OTM_OK = 0
STATUS_NAMES = {
    0: "OTM_OK", 1: "OTM_ERR_INVALID_ARGUMENT", 2: "OTM_ERR_UNSUPPORTED", 3: "OTM_ERR_CUDA",
    4: "OTM_ERR_OUT_OF_MEMORY", 5: "OTM_ERR_NOT_CONVERGED", 6: "OTM_ERR_DIVERGED", 7: "OTM_ERR_NAN",
    8: "OTM_ERR_BUDGET", 9: "OTM_ERR_STATE", 10: "OTM_ERR_TIMEOUT", 11: "OTM_ERR_CANCELLED",
    12: "OTM_ERR_NOT_READY",
}
OTM_ERR_NOT_CONVERGED = 5
OTM_ERR_NOT_READY = 12

PRECISION = {"fp32": 0, "bf16": 1, "fp16": 2}
SOLVER = {"pcg": 0, "vcycle": 1}
SMOOTHER = {"color": 0, "tiled": 1}


class OtmError(RuntimeError):
    def __init__(self, status: int, where: str, message: str = ""):
        self.status = status
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)} ({message})")


class Config(ctypes.Structure):
    _fields_ = [
        ("reso", ctypes.c_int * 3),
        ("fem_rel_thres", ctypes.c_double),
        ("max_iter", ctypes.c_int),
        ("pre_smooth", ctypes.c_int),
        ("post_smooth", ctypes.c_int),
        ("solver", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("coarsest_max_dof", ctypes.c_int),
        ("power_penal", ctypes.c_float),
        ("warm_start", ctypes.c_int),
        ("check_every", ctypes.c_int),
        ("use_graphs", ctypes.c_int),
        ("profile", ctypes.c_int),
        ("cluster_cycle", ctypes.c_int),
        ("smoother", ctypes.c_int),
    ]


class LevelInfo(ctypes.Structure):
    _fields_ = [("levels", ctypes.c_int), ("reso", ctypes.c_int * 3), ("stencil", ctypes.c_int),
                ("smoother", ctypes.c_int)]


class SolveStats(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int),
        ("refinements", ctypes.c_int),
        ("rel_res", ctypes.c_double * 3),
        ("status", ctypes.c_int),
        ("levels", ctypes.c_int),
        ("coarsest_reso", ctypes.c_int * 3),
        ("cluster_level", ctypes.c_int),
        ("smoother", ctypes.c_int),
    ]


class Profile(ctypes.Structure):
    _fields_ = [("sweeps", ctypes.c_int), ("sweep_ms", ctypes.c_double), ("sweep_bytes", ctypes.c_double),
                ("launches_per_sweep", ctypes.c_int), ("kernel_kind", ctypes.c_int)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_size_t), ("max_active", ctypes.c_int), ("fem_rel_thres", ctypes.c_double),
                ("max_iter", ctypes.c_int), ("pre_smooth", ctypes.c_int), ("iters_per_step", ctypes.c_int),
                ("power_penal", ctypes.c_float), ("batched", ctypes.c_int), ("streams", ctypes.c_int),
                ("host_stage_bytes", ctypes.c_size_t)]


class RequestInfo(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int), ("status", ctypes.c_int), ("submit_s", ctypes.c_double),
                ("admit_s", ctypes.c_double), ("done_s", ctypes.c_double), ("stats", SolveStats)]


class PitchedPtr(ctypes.Structure):
    _fields_ = [("ptr", ctypes.c_void_p), ("pitch", ctypes.c_size_t), ("xsize", ctypes.c_size_t),
                ("ysize", ctypes.c_size_t)]


class DriverConfig(ctypes.Structure):
    _fields_ = [("reso", ctypes.c_int), ("sym", ctypes.c_int), ("winit", ctypes.c_int), ("model", ctypes.c_int),
                ("vol_ratio", ctypes.c_double), ("heat_ratio", ctypes.c_double * 2), ("finthres", ctypes.c_double),
                ("fem_rel_thres", ctypes.c_double), ("target_tensor", ctypes.c_double * 6),
                ("max_iter", ctypes.c_int), ("init_period", ctypes.c_int), ("seed", ctypes.c_uint64),
                ("input_path", ctypes.c_char_p), ("output_prefix", ctypes.c_char_p)]


class DriverResult(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("converged", ctypes.c_int), ("objective", ctypes.c_double),
                ("volume", ctypes.c_double), ("volume_bound", ctypes.c_double), ("K", ctypes.c_float * 9),
                ("init_seconds", ctypes.c_double), ("loop_seconds", ctypes.c_double)]


class ConvergeChecker(ctypes.Structure):
    _fields_ = [("thres", ctypes.c_double), ("obj", ctypes.c_double * 10), ("p", ctypes.c_int)]


class VolumeGovernor(ctypes.Structure):
    _fields_ = [("low_bound", ctypes.c_float), ("volume_bound", ctypes.c_float), ("decrease", ctypes.c_float),
                ("decrease_factor", ctypes.c_float), ("val_last", ctypes.c_float), ("vibrate", ctypes.c_float),
                ("vibrate_count", ctypes.c_int), ("count", ctypes.c_int)]


_P = ctypes.c_void_p
_I3 = ctypes.POINTER(ctypes.c_int)
_D = ctypes.POINTER(ctypes.c_double)
_F = ctypes.POINTER(ctypes.c_float)
_S = ctypes.c_int  # otm_status

# name -> (restype, argtypes)
SIGNATURES = {
    "otm_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "otm_last_error": (ctypes.c_char_p, []),
    "otm_abi_version": (ctypes.c_int, []),
    "otm_config_init": (_S, [ctypes.POINTER(Config)]),
    "otm_homo_create": (_S, [ctypes.POINTER(Config), ctypes.POINTER(_P)]),
    "otm_homo_destroy": (_S, [_P]),
    "otm_homo_set_stream": (_S, [_P, _P]),
    "otm_homo_get_config": (_S, [_P, ctypes.POINTER(Config)]),
    "otm_homo_set_tolerance": (_S, [_P, ctypes.c_double]),
    "otm_homo_update": (_S, [_P, _P, ctypes.c_int]),
    "otm_homo_update_density": (_S, [_P, _I3, _P, ctypes.c_int, _P, _P, _P, ctypes.c_int, ctypes.c_float,
                                     ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float]),
    "otm_homo_solve": (_S, [_P, ctypes.POINTER(SolveStats)]),
    "otm_homo_heat_matrix": (_S, [_P, _D]),
    "otm_homo_heat_matrix_nosolve": (_S, [_P, _D]),
    "otm_homo_sensitivity": (_S, [_P, _F, _P, ctypes.c_int, ctypes.c_int]),
    "otm_homo_heat_matrix_sensitivity": (_S, [_P, _D, _F, _P, ctypes.c_int, ctypes.c_int]),
    "otm_homo_element_energy": (_S, [_P, _P]),
    "otm_homo_get_solution": (_S, [_P, ctypes.c_int, _P]),
    "otm_homo_v_cycle": (_S, [_P, _P, _P, ctypes.c_int, ctypes.c_int]),
    "otm_homo_level": (_S, [_P, ctypes.c_int, ctypes.POINTER(LevelInfo)]),
    "otm_homo_set_solution": (_S, [_P, ctypes.c_int, _P]),
    "otm_homo_reset_displacement": (_S, [_P]),
    "otm_homo_get_stats": (_S, [_P, ctypes.POINTER(SolveStats)]),
    "otm_homo_get_profile": (_S, [_P, ctypes.POINTER(Profile), ctypes.c_int]),
    "otm_launch_count": (ctypes.c_uint64, []),
    "otm_scratch_alloc_count": (ctypes.c_uint64, []),
    "otm_host_alloc": (_S, [ctypes.c_size_t, ctypes.POINTER(_P)]),
    "otm_host_free": (_S, [_P]),
    "otm_copy_to_device": (_S, [_P, _P, ctypes.c_size_t, _P]),
    "otm_copy_to_host": (_S, [_P, _P, ctypes.c_size_t, _P]),
    "otm_filter_forward": (_S, [_I3, _P, ctypes.c_int, _P, ctypes.c_int, _P, ctypes.c_int, ctypes.c_float,
                                ctypes.c_int, _P]),
    "otm_filter_backward": (_S, [_I3, _P, ctypes.c_int, _P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                 ctypes.c_int, _P]),
    "otm_density_forward": (_S, [_I3, _P, ctypes.c_int, _P, _P, _P, _P, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                 ctypes.c_float, ctypes.c_float, ctypes.c_float, _P]),
    "otm_density_backward": (_S, [_I3, _P, _P, _P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                  _P]),
    "otm_oc_filter_sens": (_S, [_P, _P, ctypes.c_size_t, _I3, ctypes.c_float, _P]),
    "otm_oc_update": (_S, [ctypes.c_int, _P, _P, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                           _P, ctypes.POINTER(ctypes.c_int)]),
    # MMA (include/opentm_b200_mma.h)
    "otm_mma_create": (_S, [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                            ctypes.c_double, ctypes.POINTER(_P)]),
    "otm_mma_destroy": (_S, [_P]),
    "otm_mma_set_stream": (_S, [_P, _P]),
    "otm_mma_set_bound_scalar": (_S, [_P, ctypes.c_float, ctypes.c_float]),
    "otm_mma_set_bound": (_S, [_P, _P, _P]),
    "otm_mma_update": (_S, [_P, ctypes.c_int, _P, _P, _F, ctypes.POINTER(_P)]),
    "otm_mmasub_device": (_S, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _P, _P, _P, _P, ctypes.c_double, _P,
                               _P, PitchedPtr, _P, _P, ctypes.c_double, _P, _P, _P, ctypes.c_double, _P]),
    # allocation-free filter (include/opentm_b200_noalloc.h)
    "otm_oc_filter_sens_noalloc": (_S, [_P, _P, ctypes.c_size_t, _I3, ctypes.c_float, _P]),
    # serving (include/opentm_b200_server.h)
    "otm_server_config_init": (_S, [ctypes.POINTER(ServerConfig)]),
    "otm_server_create": (_S, [ctypes.POINTER(ServerConfig), _P, ctypes.POINTER(_P)]),
    "otm_server_destroy": (_S, [_P]),
    "otm_server_submit": (_S, [_P, _I3, _F, ctypes.POINTER(ctypes.c_int64)]),
    "otm_server_step": (_S, [_P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "otm_server_poll": (_S, [_P, ctypes.c_int64, _D, ctypes.POINTER(RequestInfo)]),
    "otm_server_cancel": (_S, [_P, ctypes.c_int64]),
    "otm_server_request_bytes": (ctypes.c_size_t, [_I3]),
    "otm_server_bytes_in_use": (ctypes.c_size_t, [_P]),
    "otm_server_bytes_resident": (ctypes.c_size_t, [_P]),
    # design driver (include/opentm_b200_driver.h)
    "otm_driver_config_init": (_S, [ctypes.POINTER(DriverConfig)]),
    "otm_symmetrize": (_S, [_I3, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P]),
    "otm_randtri_coeff_count": (ctypes.c_size_t, [ctypes.c_int, ctypes.c_int]),
    "otm_randtri_coefficients": (_S, [ctypes.c_uint64, ctypes.c_int, ctypes.c_int, _F]),
    "otm_randtri_field": (_S, [_I3, _P, ctypes.c_int, ctypes.c_int, _F, ctypes.c_int, _P]),
    "otm_init_density": (_S, [ctypes.POINTER(DriverConfig), _P, ctypes.c_int, _F, _P]),
    "otm_converge_checker_init": (None, [ctypes.POINTER(ConvergeChecker), ctypes.c_double]),
    "otm_converge_checker_step": (ctypes.c_int, [ctypes.POINTER(ConvergeChecker), ctypes.c_int, ctypes.c_double]),
    "otm_volume_governor_init": (None, [ctypes.POINTER(VolumeGovernor)]),
    "otm_volume_governor_check": (ctypes.c_int, [ctypes.POINTER(VolumeGovernor), ctypes.c_float, ctypes.c_float,
                                                 ctypes.c_float, ctypes.c_int]),
    "otm_volume_governor_decrease": (ctypes.c_float, [ctypes.POINTER(VolumeGovernor)]),
    "otm_run_custom": (_S, [ctypes.POINTER(DriverConfig), _F, _F, _D, ctypes.POINTER(DriverResult)]),
    "otm_write_density_binary": (_S, [ctypes.c_char_p, _I3, _F]),
    "otm_read_density_binary": (_S, [ctypes.c_char_p, _I3, _F, ctypes.c_size_t]),
    "otm_write_vectors": (_S, [ctypes.c_char_p, ctypes.c_int, ctypes.c_size_t, ctypes.POINTER(_F)]),
    "otm_read_vectors": (_S, [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(_F),
                              ctypes.c_size_t]),
    "otm_write_heat_matrix": (_S, [ctypes.c_char_p, _F, ctypes.c_int]),
}

_lib = None


def header_symbols() -> list[str]:
    """Every function the public headers declare."""
    names = []
    for h in HEADERS:
        if not os.path.exists(h):
            continue
        txt = open(h).read()
        names += re.findall(r"^OTM_API\s+[\w\s\*]+?\b(otm_\w+)\s*\(", txt, flags=re.M)
    return names


def lib() -> ctypes.CDLL:
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build the sm_100a CUDA library with `python -m opentm_b200.build` "
            "(there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def last_error() -> str:
    return lib().otm_last_error().decode()


def check(status: int, where: str, allow=(OTM_OK,)) -> int:
    if status not in allow:
        raise OtmError(status, where, last_error())
    return status


def default_config(reso=(128, 128, 128), **kw) -> Config:
    cfg = Config()
    check(lib().otm_config_init(ctypes.byref(cfg)), "otm_config_init")
    if isinstance(reso, int):
        reso = (reso, reso, reso)
    for i in range(3):
        cfg.reso[i] = int(reso[i])
    for k, v in kw.items():
        if k == "precision" and isinstance(v, str):
            v = PRECISION[v]
        if k == "solver" and isinstance(v, str):
            v = SOLVER[v]
        if k == "smoother" and isinstance(v, str):
            v = SMOOTHER[v]
        if not hasattr(cfg, k):
            raise TypeError(f"unknown config field {k}")
        setattr(cfg, k, v)
    return cfg


def i3(reso) -> ctypes.Array:
    if isinstance(reso, int):
        reso = (reso, reso, reso)
    return (ctypes.c_int * 3)(*[int(r) for r in reso])
