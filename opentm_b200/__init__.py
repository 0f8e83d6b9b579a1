"""opentm_b200 -- B200-native thermal homogenization hot path of OpenTM.

Python mirror of the reference's host interface (``Homogenization_H``, ``OCOptimizer``,
``MMAOptimizer``, the density-filter chain) over the C ABI of ``libopentm_b200.so``.
Device arrays are torch CUDA tensors (or raw device pointers); torch is used only for device
memory and streams. Every call goes to the sm_100a CUDA library; if it is not built, the
calls raise -- there is no CPU fallback.

Fields are lexicographic with x fastest: a cell of reso (nx, ny, nz) is a torch tensor of
shape (nz, ny, nx) (or (nz, ny, pitchT) for pitched fields).
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import OtmError, check, default_config, i3, lib

def launch_count() -> int:
    """Kernels launched by the CUDA library in this process (graph replays count their nodes)."""
    return int(lib().otm_launch_count())


__all__ = ["launch_count", "Server", "pinned_empty", "copy_to_device", "copy_to_host", 
    "HomoConfig", "Homogenization_H", "OCOptimizer", "MMAOptimizer", "DensityFilter", "OtmError", "lib",
    "WEIGHT_SPLINE4", "WEIGHT_LINEAR", "filter_forward", "filter_backward",
]

WEIGHT_SPLINE4 = 0
WEIGHT_LINEAR = 1


class _HostBlock:
    """Owner of one otm_host_alloc block; freed when the last array viewing it goes."""

    def __init__(self, nbytes: int):
        self.ptr = ctypes.c_void_p()
        check(lib().otm_host_alloc(ctypes.c_size_t(nbytes), ctypes.byref(self.ptr)), "otm_host_alloc")

    def __del__(self):
        try:
            if self.ptr:
                lib().otm_host_free(self.ptr)
        except Exception:
            pass


def pinned_empty(shape, dtype=np.float32) -> np.ndarray:
    """A numpy array in page-locked host memory from otm_host_alloc (cudaHostAlloc): the fast
    source and target of per-step host<->device copies (torch.from_numpy(a) is a pinned tensor)."""
    dt = np.dtype(dtype)
    count = int(np.prod(shape)) if np.ndim(shape) else int(shape)
    blk = _HostBlock(max(count * dt.itemsize, 1))
    buf = (ctypes.c_char * (count * dt.itemsize)).from_address(blk.ptr.value)
    buf._otm_block = blk  # the array keeps buf alive, buf keeps the block
    return np.frombuffer(buf, dtype=dt, count=count).reshape(shape)


def copy_to_device(dst, src: np.ndarray, stream=None) -> None:
    """Asynchronous copy of a host array (page-locked, e.g. from pinned_empty) into the CUDA
    tensor dst on the current (or given) stream."""
    if src.nbytes != dst.numel() * dst.element_size() or not src.flags.c_contiguous or not dst.is_contiguous():
        raise ValueError("copy_to_device needs contiguous arrays of the same size")
    check(lib().otm_copy_to_device(ctypes.c_void_p(_ptr(dst)), ctypes.c_void_p(src.ctypes.data),
                                   ctypes.c_size_t(src.nbytes), ctypes.c_void_p(_stream(stream))),
          "otm_copy_to_device")


def copy_to_host(dst: np.ndarray, src, stream=None) -> None:
    """Asynchronous copy of the CUDA tensor src into a host array (page-locked) on the current (or
    given) stream; synchronise before reading dst."""
    if dst.nbytes != src.numel() * src.element_size() or not dst.flags.c_contiguous or not src.is_contiguous():
        raise ValueError("copy_to_host needs contiguous arrays of the same size")
    check(lib().otm_copy_to_host(ctypes.c_void_p(dst.ctypes.data), ctypes.c_void_p(_ptr(src)),
                                 ctypes.c_size_t(dst.nbytes), ctypes.c_void_p(_stream(stream))), "otm_copy_to_host")


def _ptr(t) -> int:
    if t is None:
        return None
    if isinstance(t, int):
        return t
    if not t.is_cuda:
        raise ValueError("device arrays must be CUDA tensors")
    return t.data_ptr()


def _stream(stream=None):
    if stream is not None:
        return stream if isinstance(stream, int) else stream.cuda_stream
    import torch
    return torch.cuda.current_stream().cuda_stream


@dataclass
class HomoConfig:
    """Mirror of cfg::HomoConfig (cmdline.h:12-33) restricted to the solve, with
    init() defaults (cmdline.cpp:4-35)."""
    reso: tuple = (128, 128, 128)
    femRelThres: float = 0.01
    max_iter: int = 200
    pre_smooth: int = 1
    post_smooth: int = 1
    solver: str = "pcg"
    precision: str = "fp32"
    coarsest_max_dof: int = 64
    power_penal: float = 1.0
    warm_start: bool = True
    check_every: int = 4
    use_graphs: bool = True
    profile: bool = False
    cluster_cycle: int = 1  # 0 off, 1 automatic, 2 from 16^3, 3 from 32^3
    smoother: str = "tiled"

    def to_c(self) -> _lib.Config:
        reso = self.reso if not isinstance(self.reso, int) else (self.reso,) * 3
        return default_config(
            reso, fem_rel_thres=float(self.femRelThres), max_iter=int(self.max_iter),
            pre_smooth=int(self.pre_smooth), post_smooth=int(self.post_smooth), solver=self.solver,
            precision=self.precision, coarsest_max_dof=int(self.coarsest_max_dof),
            power_penal=float(self.power_penal), warm_start=int(bool(self.warm_start)),
            check_every=int(self.check_every), use_graphs=int(bool(self.use_graphs)),
            profile=int(bool(self.profile)), cluster_cycle=int(self.cluster_cycle),
            smoother=self.smoother)


class Homogenization_H:
    """Homogenization_H (homogenization/homogenization.h:15-30) on the B200 library."""

    def __init__(self, config: HomoConfig, stream=None):
        self.config = config
        self._h = ctypes.c_void_p()
        check(lib().otm_homo_create(ctypes.byref(config.to_c()), ctypes.byref(self._h)), "otm_homo_create")
        reso = config.reso if not isinstance(config.reso, int) else (config.reso,) * 3
        self.reso = tuple(int(r) for r in reso)
        if stream is not None:
            self.set_stream(stream)

    def close(self):
        if self._h:
            lib().otm_homo_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream):
        check(lib().otm_homo_set_stream(self._h, ctypes.c_void_p(_stream(stream))), "otm_homo_set_stream")

    def _sync_stream(self):
        self.set_stream(None)

    @property
    def n_cells(self) -> int:
        return self.reso[0] * self.reso[1] * self.reso[2]

    def set_tolerance(self, tol: float):
        check(lib().otm_homo_set_tolerance(self._h, float(tol)), "otm_homo_set_tolerance")

    def update(self, rho, pitchT: int = -1):
        """Homogenization_H::update(float* rho, int pitchT) (homogenization.cpp:76-81)."""
        self._sync_stream()
        check(lib().otm_homo_update(self._h, ctypes.c_void_p(_ptr(rho)), int(pitchT)), "otm_homo_update")

    def update_density(self, df: "DensityFilter", rho, pitchT: int = -1):
        """df.forward(rho) followed by update(k) with the conductivity import folded into the
        filter's forward pass (otm_homo_update_density): df.rho_f, df.dk and df.wsum are written as
        by df.forward, for df.backward; the conductivities go straight into this handle (df.k is
        left as it was)."""
        self._sync_stream()
        check(lib().otm_homo_update_density(self._h, i3(df.reso), ctypes.c_void_p(_ptr(rho)), int(pitchT),
                                            ctypes.c_void_p(_ptr(df.rho_f)), ctypes.c_void_p(_ptr(df.dk)),
                                            ctypes.c_void_p(_ptr(df.wsum)), df.weight, df.radius, int(df.periodic),
                                            df.p, df.k0, df.kmin), "otm_homo_update_density")

    def solve(self, allow_not_converged: bool = False) -> _lib.SolveStats:
        self._sync_stream()
        st = _lib.SolveStats()
        allow = (0, _lib.OTM_ERR_NOT_CONVERGED) if allow_not_converged else (0,)
        check(lib().otm_homo_solve(self._h, ctypes.byref(st)), "otm_homo_solve", allow)
        return st

    def heatMatrix(self, allow_not_converged: bool = False) -> np.ndarray:
        """Homogenization_H::heatMatrix(double C[3][3]) (homogenization.cu:180-252)."""
        self._sync_stream()
        C = (ctypes.c_double * 9)()
        allow = (0, _lib.OTM_ERR_NOT_CONVERGED) if allow_not_converged else (0,)
        check(lib().otm_homo_heat_matrix(self._h, C), "otm_homo_heat_matrix", allow)
        return np.array(C[:], dtype=np.float64).reshape(3, 3)

    def heatMatrix_nosolve(self) -> np.ndarray:
        self._sync_stream()
        C = (ctypes.c_double * 9)()
        check(lib().otm_homo_heat_matrix_nosolve(self._h, C), "otm_homo_heat_matrix_nosolve")
        return np.array(C[:], dtype=np.float64).reshape(3, 3)

    def Sensitivity(self, dC, sens, pitchT: int = -1, lexiOrder: bool = False):
        """Homogenization_H::Sensitivity(dC, sens, pitchT, lexiOrder) (homogenization.cu:415-479)."""
        self._sync_stream()
        d = (ctypes.c_float * 9)(*[float(v) for v in np.asarray(dC, dtype=np.float64).reshape(9)])
        check(lib().otm_homo_sensitivity(self._h, d, ctypes.c_void_p(_ptr(sens)), int(pitchT), int(bool(lexiOrder))),
              "otm_homo_sensitivity")

    def heatMatrixSensitivity(self, dC, sens, pitchT: int = -1, lexiOrder: bool = False,
                              allow_not_converged: bool = False) -> np.ndarray:
        """heatMatrix() and Sensitivity(dC, sens, pitchT, lexiOrder) in one element pass, for a dC
        that does not depend on C (a linear objective); returns C."""
        self._sync_stream()
        C = (ctypes.c_double * 9)()
        d = (ctypes.c_float * 9)(*[float(v) for v in np.asarray(dC, dtype=np.float64).reshape(9)])
        allow = (0, _lib.OTM_ERR_NOT_CONVERGED) if allow_not_converged else (0,)
        check(lib().otm_homo_heat_matrix_sensitivity(self._h, C, d, ctypes.c_void_p(_ptr(sens)), int(pitchT),
                                                     int(bool(lexiOrder))), "otm_homo_heat_matrix_sensitivity", allow)
        return np.array(C[:], dtype=np.float64).reshape(3, 3)

    def element_energy(self, out=None):
        """dK^H_ab/dk_e for the pairs 00 01 02 11 12 22 as a (6, nz, ny, nx) tensor."""
        import torch
        nx, ny, nz = self.reso
        if out is None:
            out = torch.empty((6, nz, ny, nx), dtype=torch.float32, device="cuda")
        self._sync_stream()
        check(lib().otm_homo_element_energy(self._h, ctypes.c_void_p(_ptr(out))), "otm_homo_element_energy")
        return out

    def v_cycle(self, f, u=None, pre: int = 1, post: int = 1):
        """MG_H::v_cycle (homogenization/MG.cpp:46-71): one V(pre, post) cycle of the handle's
        hierarchy on the right-hand sides f (3, nz, ny, nx) from a zero correction -> u."""
        import torch
        if u is None:
            u = torch.empty_like(f)
        self._sync_stream()
        check(lib().otm_homo_v_cycle(self._h, ctypes.c_void_p(_ptr(f)), ctypes.c_void_p(_ptr(u)), int(pre), int(post)),
              "otm_homo_v_cycle")
        return u

    def level(self, level: int) -> _lib.LevelInfo:
        """Grid_H of one level (homogenization/grid.h:104-421): sizes, stencil or matrix-free, smoother."""
        info = _lib.LevelInfo()
        check(lib().otm_homo_level(self._h, int(level), ctypes.byref(info)), "otm_homo_level")
        return info

    def solution(self, lcase: int, out=None):
        import torch
        nx, ny, nz = self.reso
        if out is None:
            out = torch.empty((nz, ny, nx), dtype=torch.float32, device="cuda")
        self._sync_stream()
        check(lib().otm_homo_get_solution(self._h, int(lcase), ctypes.c_void_p(_ptr(out))), "otm_homo_get_solution")
        return out

    def set_solution(self, lcase: int, src):
        self._sync_stream()
        check(lib().otm_homo_set_solution(self._h, int(lcase), ctypes.c_void_p(_ptr(src))), "otm_homo_set_solution")

    def reset_displacement(self):
        """MG_H::reset_displacement (homogenization/MG.cpp:73-78)."""
        self._sync_stream()
        check(lib().otm_homo_reset_displacement(self._h), "otm_homo_reset_displacement")

    def profile(self, reset: bool = True) -> _lib.Profile:
        pr = _lib.Profile()
        check(lib().otm_homo_get_profile(self._h, ctypes.byref(pr), int(bool(reset))), "otm_homo_get_profile")
        return pr

    def stats(self) -> _lib.SolveStats:
        st = _lib.SolveStats()
        check(lib().otm_homo_get_stats(self._h, ctypes.byref(st)), "otm_homo_get_stats")
        return st


def filter_forward(src, reso, radius=2.0, weight=WEIGHT_LINEAR, periodic=True, dst=None, wsum=None,
                   src_pitchT=-1, dst_pitchT=-1, stream=None):
    """conv_kernel (AutoDiff/TensorExpression.cuh:304-350)."""
    import torch
    nx, ny, nz = reso
    if dst is None:
        dst = torch.empty((nz, ny, nx), dtype=torch.float32, device="cuda")
    if wsum is None:
        wsum = torch.empty((nz, ny, nx), dtype=torch.float32, device="cuda")
    check(lib().otm_filter_forward(i3(reso), ctypes.c_void_p(_ptr(src)), int(src_pitchT), ctypes.c_void_p(_ptr(dst)),
                                   int(dst_pitchT), ctypes.c_void_p(_ptr(wsum)), int(weight), float(radius),
                                   int(bool(periodic)), ctypes.c_void_p(_stream(stream))), "otm_filter_forward")
    return dst, wsum


def filter_backward(g_dst, wsum, reso, radius=2.0, weight=WEIGHT_LINEAR, periodic=True, g_src=None, stream=None):
    """conv_backward_kernel (AutoDiff/TensorExpression.cuh:353-385)."""
    import torch
    nx, ny, nz = reso
    if g_src is None:
        g_src = torch.empty((nz, ny, nx), dtype=torch.float32, device="cuda")
    check(lib().otm_filter_backward(i3(reso), ctypes.c_void_p(_ptr(g_dst)), -1, ctypes.c_void_p(_ptr(wsum)),
                                    ctypes.c_void_p(_ptr(g_src)), -1, int(weight), float(radius), int(bool(periodic)),
                                    ctypes.c_void_p(_stream(stream))), "otm_filter_backward")
    return g_src


class DensityFilter:
    """rho -> k = (k0 - kmin) conv(rho)^p + kmin and its adjoint, as the expression
    rho.conv(ker).pow(p) * (k0 - kmin) + kmin of runCustom (Framework.cu:163)."""

    def __init__(self, reso, radius=2.0, weight=WEIGHT_LINEAR, periodic=True, p=3.0, k0=1.0, kmin=1e-3):
        import torch
        self.reso = tuple(reso)
        self.radius, self.weight, self.periodic = float(radius), int(weight), bool(periodic)
        self.p, self.k0, self.kmin = float(p), float(k0), float(kmin)
        nx, ny, nz = self.reso
        shape = (nz, ny, nx)
        self.rho_f = torch.empty(shape, dtype=torch.float32, device="cuda")
        self.k = torch.empty(shape, dtype=torch.float32, device="cuda")
        self.dk = torch.empty(shape, dtype=torch.float32, device="cuda")
        self.wsum = torch.empty(shape, dtype=torch.float32, device="cuda")

    def forward(self, rho, pitchT=-1, stream=None):
        check(lib().otm_density_forward(i3(self.reso), ctypes.c_void_p(_ptr(rho)), int(pitchT),
                                        ctypes.c_void_p(_ptr(self.rho_f)), ctypes.c_void_p(_ptr(self.k)),
                                        ctypes.c_void_p(_ptr(self.dk)), ctypes.c_void_p(_ptr(self.wsum)),
                                        self.weight, self.radius, int(self.periodic), self.p, self.k0, self.kmin,
                                        ctypes.c_void_p(_stream(stream))), "otm_density_forward")
        return self.k

    def backward(self, g_k, g_rho=None, stream=None):
        import torch
        if g_rho is None:
            g_rho = torch.empty_like(self.k)
        check(lib().otm_density_backward(i3(self.reso), ctypes.c_void_p(_ptr(g_k)), ctypes.c_void_p(_ptr(self.dk)),
                                         ctypes.c_void_p(_ptr(self.wsum)), ctypes.c_void_p(_ptr(g_rho)), -1,
                                         self.weight, self.radius, int(self.periodic),
                                         ctypes.c_void_p(_stream(stream))), "otm_density_backward")
        return g_rho


class OCOptimizer:
    """OCOptimizer (optimization/OCOptimizer.h:7-20)."""

    def __init__(self, ne: int, min_density: float = 0.001, stepLimit: float = 0.02, dampExponent: float = 0.5):
        self.ne, self.minRho, self.step_limit, self.damp = int(ne), float(min_density), float(stepLimit), float(dampExponent)
        self.last_iters = None

    def filterSens(self, sens, rho, pitchT, reso, radius: float = 2.0, stream=None):
        check(lib().otm_oc_filter_sens(ctypes.c_void_p(_ptr(sens)), ctypes.c_void_p(_ptr(rho)), int(pitchT), i3(reso),
                                       float(radius), ctypes.c_void_p(_stream(stream))), "otm_oc_filter_sens")

    def update(self, sens, rho, volratio: float, stream=None, want_iters: bool = False):
        it = ctypes.c_int(0)
        check(lib().otm_oc_update(self.ne, ctypes.c_void_p(_ptr(sens)), ctypes.c_void_p(_ptr(rho)), float(volratio),
                                  self.minRho, self.step_limit, self.damp, ctypes.c_void_p(_stream(stream)),
                                  ctypes.byref(it) if want_iters else None), "otm_oc_update")
        self.last_iters = it.value if want_iters else None
        return self.last_iters


class MMAOptimizer:
    """MMAOptimizer (optimization/mmaOptimizer.h:12-35): FP64 method of moving asymptotes on
    the device; x, dfdx and dgdx rows are float32 device arrays of n values."""

    def __init__(self, nconstrain: int, nvar: int, a0: float, a: float, c: float, d: float, stream=None):
        self.m, self.n = int(nconstrain), int(nvar)
        self._h = ctypes.c_void_p()
        check(lib().otm_mma_create(self.m, self.n, float(a0), float(a), float(c), float(d), ctypes.byref(self._h)),
              "otm_mma_create")
        if stream is not None:
            check(lib().otm_mma_set_stream(self._h, ctypes.c_void_p(_stream(stream))), "otm_mma_set_stream")

    def __del__(self):
        try:
            if self._h:
                lib().otm_mma_destroy(self._h)
        except Exception:
            pass

    def setBound(self, xmin, xmax):
        if isinstance(xmin, (int, float)):
            check(lib().otm_mma_set_bound_scalar(self._h, float(xmin), float(xmax)), "otm_mma_set_bound_scalar")
        else:
            check(lib().otm_mma_set_bound(self._h, ctypes.c_void_p(_ptr(xmin)), ctypes.c_void_p(_ptr(xmax))),
                  "otm_mma_set_bound")

    def update(self, itn: int, x, dfdx, gval, dgdx):
        check(lib().otm_mma_set_stream(self._h, ctypes.c_void_p(_stream(None))), "otm_mma_set_stream")
        g = (ctypes.c_float * self.m)(*[float(v) for v in np.asarray(gval, dtype=np.float64).reshape(self.m)])
        rows = (ctypes.c_void_p * self.m)(*[_ptr(r) for r in dgdx])
        check(lib().otm_mma_update(self._h, int(itn), ctypes.c_void_p(_ptr(x)), ctypes.c_void_p(_ptr(dfdx)), g, rows),
              "otm_mma_update")


class Server:
    """Server of independent homogenization requests (include/opentm_b200_server.h).

    submit(k) queues a solve of one cell (k: host numpy array of shape (nz, ny, nx)); step()
    retires finished requests and admits what fits the memory budget (the batched form also
    advances every running request); poll(id) returns None while the request is queued or
    running, else (K^H, info). batched=False (default) runs up to `streams` requests at once as
    resident solver handles on their own streams; batched=True advances all running requests
    with shared kernel launches.
    """

    def __init__(self, hbm_budget_bytes=150 * 10 ** 9, max_active=64, fem_rel_thres=1e-6, max_iter=200,
                 pre_smooth=2, iters_per_step=2, power_penal=1.0, stream=None, batched=False, streams=8,
                 host_stage_bytes=1 << 30):
        cfg = _lib.ServerConfig()
        check(lib().otm_server_config_init(ctypes.byref(cfg)), "otm_server_config_init")
        cfg.hbm_budget_bytes = int(hbm_budget_bytes)
        cfg.max_active = int(max_active)
        cfg.fem_rel_thres = float(fem_rel_thres)
        cfg.max_iter = int(max_iter)
        cfg.pre_smooth = int(pre_smooth)
        cfg.iters_per_step = int(iters_per_step)
        cfg.power_penal = float(power_penal)
        cfg.batched = int(bool(batched))
        cfg.streams = int(streams)
        cfg.host_stage_bytes = int(host_stage_bytes)
        self._h = ctypes.c_void_p()
        check(lib().otm_server_create(ctypes.byref(cfg), ctypes.c_void_p(_stream(stream)), ctypes.byref(self._h)),
              "otm_server_create")

    def close(self):
        if self._h:
            lib().otm_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def request_bytes(reso) -> int:
        return int(lib().otm_server_request_bytes(i3(reso)))

    def bytes_in_use(self) -> int:
        return int(lib().otm_server_bytes_in_use(self._h))

    def bytes_resident(self) -> int:
        return int(lib().otm_server_bytes_resident(self._h))

    def submit(self, k) -> int:
        k = np.ascontiguousarray(k, dtype=np.float32)
        nz, ny, nx = k.shape
        rid = ctypes.c_int64(0)
        check(lib().otm_server_submit(self._h, i3((nx, ny, nz)), k.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                      ctypes.byref(rid)), "otm_server_submit")
        return rid.value

    def step(self):
        nr, nq = ctypes.c_int(0), ctypes.c_int(0)
        check(lib().otm_server_step(self._h, ctypes.byref(nr), ctypes.byref(nq)), "otm_server_step")
        return nr.value, nq.value

    def poll(self, rid):
        C = (ctypes.c_double * 9)()
        info = _lib.RequestInfo()
        st = lib().otm_server_poll(self._h, ctypes.c_int64(rid), C, ctypes.byref(info))
        if st == _lib.OTM_ERR_NOT_READY:
            return None
        if st not in (0, _lib.OTM_ERR_NOT_CONVERGED):
            raise OtmError(st, "otm_server_poll", _lib.last_error())
        return np.array(C[:]).reshape(3, 3), info

    def state(self, rid) -> int:
        """0 queued, 1 running, 2 done, 3 cancelled, 4 failed."""
        info = _lib.RequestInfo()
        lib().otm_server_poll(self._h, ctypes.c_int64(rid), None, ctypes.byref(info))
        return int(info.state)

    def cancel(self, rid):
        check(lib().otm_server_cancel(self._h, ctypes.c_int64(rid)), "otm_server_cancel")

    def run_until_idle(self, timeout_s=600.0):
        t_end = time.monotonic() + timeout_s
        while time.monotonic() < t_end:
            nr, nq = self.step()
            if nr == 0 and nq == 0:
                return
            if nq == 0:
                time.sleep(20e-6)  # only running requests left: poll, do not spin
        raise RuntimeError("server did not drain")
