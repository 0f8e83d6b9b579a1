"""FP64 CPU oracle of OpenTM's homogenization hot path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import
this package, as the checker or as the timed CPU baseline. The product (``opentm_b200``)
never imports it.

Parity unpinned: the reference ships no golden vectors and cannot be built offline, so the
oracle is pinned by known-answer tests from the mathematics instead (see ``tests/``).

``build()`` compiles ``otm_oracle.cpp`` with the Makefile beside it; the wrappers below
accept numpy arrays and call the C functions through ctypes.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libotm_oracle.so")
_lib = None

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def build(force: bool = False) -> str:
    """Compile the oracle shared library (make -C oracle)."""
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "otm_oracle.cpp"))
    ):
        subprocess.run(["make", "-s", "-C", _HERE] + (["-B"] if force else []), check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.ora_template_matrix.argtypes = [ctypes.c_int, _D, _D, _D]
        L.ora_apply.argtypes = [_I, _D, _D, _D]
        L.ora_rhs.argtypes = [_I, _D, _D]
        L.ora_homogenize.argtypes = [_I, _D, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, _D, _D, _D, _D]
        L.ora_homogenize.restype = ctypes.c_int
        L.ora_homogenize_cases.argtypes = [_I, _D, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_int, _D, _D, _D, _D]
        L.ora_homogenize_cases.restype = ctypes.c_int
        L.ora_homogenize_warm.argtypes = [_I, _D, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, _D, _D, _D, _D, ctypes.POINTER(ctypes.c_int)]
        L.ora_homogenize_warm.restype = ctypes.c_int
        L.ora_element_energy.argtypes = [_I, _D, _D]
        L.ora_sensitivity.argtypes = [_I, _D, _D, ctypes.c_double, _D, _D]
        L.ora_conv_forward.argtypes = [_I, _D, _D, _D, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.ora_conv_backward.argtypes = [_I, _D, _D, _D, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.ora_oc_filter_sens.argtypes = [_I, _D, _D, ctypes.c_double]
        L.ora_oc_update.argtypes = [ctypes.c_longlong, _D, _D, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_double]
        L.ora_oc_update.restype = ctypes.c_int
        L.ora_mmasub.argtypes = [ctypes.c_int, ctypes.c_longlong, ctypes.c_int, _D, _D, _D, _D, _D, _D, _D, _D,
                                 _D, _D, ctypes.c_double, _D, _D, _D, ctypes.c_double]
        L.ora_num_threads.restype = ctypes.c_int
        L.ora_set_num_threads.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(_D)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _dims(shape):
    """Reso (nx, ny, nz) from a (nz, ny, nx) numpy array shape, x fastest."""
    nz, ny, nx = shape
    return (ctypes.c_int * 3)(nx, ny, nz)


def num_threads() -> int:
    return lib().ora_num_threads()


def set_num_threads(n: int) -> None:
    lib().ora_set_num_threads(int(n))


def template_matrix(reso: int):
    KE = np.zeros(64)
    fe = np.zeros(24)
    dp = np.zeros(24)
    lib().ora_template_matrix(int(reso), _dp(KE), _dp(fe), _dp(dp))
    return KE.reshape(8, 8), fe.reshape(8, 3), dp.reshape(8, 3)


def apply(k_solver: np.ndarray, x: np.ndarray) -> np.ndarray:
    k = _f64(k_solver)
    xx = _f64(x)
    y = np.zeros_like(xx)
    lib().ora_apply(_dims(k.shape), _dp(k), _dp(xx), _dp(y))
    return y


def rhs(k_solver: np.ndarray) -> np.ndarray:
    k = _f64(k_solver)
    f = np.zeros((3,) + k.shape)
    lib().ora_rhs(_dims(k.shape), _dp(k), _dp(f))
    return f


def homogenize(k: np.ndarray, power_penal: float = 1.0, tol: float = 1e-12, max_iter: int = 2000,
               precond: int = 1, coarsest_max_dof: int = 64, want_chi: bool = False, want_energy: bool = False,
               case_mask: int = 7):
    """K^H (3x3), and optionally chi (3, nz, ny, nx) and element energies (6, nz, ny, nx).

    ``k`` is the conductivity handed to the reference's ``update``; the solver adds the 1e-9
    floor. Returns a dict with keys C, chi, energy, iters, relres.
    """
    kk = _f64(k)
    C = np.zeros(9)
    chi = np.zeros((3,) + kk.shape) if want_chi else None
    en = np.zeros((6,) + kk.shape) if want_energy else None
    rr = np.zeros(3)
    it = lib().ora_homogenize_cases(_dims(kk.shape), _dp(kk), float(power_penal), float(tol), int(max_iter),
                                    int(precond), int(coarsest_max_dof), int(case_mask), _dp(C),
                                    _dp(chi) if chi is not None else None, _dp(en) if en is not None else None,
                                    _dp(rr))
    return {"C": C.reshape(3, 3), "chi": chi, "energy": en, "iters": it, "relres": rr}


def homogenize_warm(k: np.ndarray, chi: np.ndarray, power_penal: float = 1.0, tol: float = 1e-12,
                    max_iter: int = 2000, coarsest_max_dof: int = 64, want_energy: bool = False):
    """The 3 load cases solved from the initial guess ``chi`` (3, nz, ny, nx; float64, updated in
    place with the solutions), as the warm-started solve of an optimisation loop. Returns a dict
    with keys C, energy, iters (per case), relres."""
    kk = _f64(k)
    assert chi.dtype == np.float64 and chi.flags["C_CONTIGUOUS"] and chi.shape == (3,) + kk.shape
    C = np.zeros(9)
    en = np.zeros((6,) + kk.shape) if want_energy else None
    rr = np.zeros(3)
    its = (ctypes.c_int * 3)()
    lib().ora_homogenize_warm(_dims(kk.shape), _dp(kk), float(power_penal), float(tol), int(max_iter), 1,
                              int(coarsest_max_dof), _dp(chi), _dp(C), _dp(en) if en is not None else None, _dp(rr),
                              its)
    return {"C": C.reshape(3, 3), "energy": en, "iters": list(its), "relres": rr}


def element_energy(chi: np.ndarray) -> np.ndarray:
    c = _f64(chi)
    en = np.zeros((6,) + c.shape[1:])
    lib().ora_element_energy(_dims(c.shape[1:]), _dp(c), _dp(en))
    return en


def sensitivity(energy: np.ndarray, k: np.ndarray, dC, power_penal: float = 1.0) -> np.ndarray:
    en = _f64(energy)
    kk = _f64(k)
    dc = _f64(np.asarray(dC).reshape(9))
    s = np.zeros_like(kk)
    lib().ora_sensitivity(_dims(kk.shape), _dp(en), _dp(kk), float(power_penal), _dp(dc), _dp(s))
    return s


WEIGHT_SPLINE4 = 0
WEIGHT_LINEAR = 1


def conv_forward(src: np.ndarray, wtype: int, radius: float, periodic: bool):
    s = _f64(src)
    dst = np.zeros_like(s)
    ws = np.zeros_like(s)
    lib().ora_conv_forward(_dims(s.shape), _dp(s), _dp(dst), _dp(ws), int(wtype), float(radius), int(bool(periodic)))
    return dst, ws


def conv_backward(g_dst: np.ndarray, wsum: np.ndarray, wtype: int, radius: float, periodic: bool):
    g = _f64(g_dst)
    w = _f64(wsum)
    out = np.zeros_like(g)
    lib().ora_conv_backward(_dims(g.shape), _dp(g), _dp(w), _dp(out), int(wtype), float(radius),
                            int(bool(periodic)))
    return out


def oc_filter_sens(sens: np.ndarray, rho: np.ndarray, radius: float = 2.0) -> np.ndarray:
    s = _f64(sens).copy()
    r = _f64(rho)
    lib().ora_oc_filter_sens(_dims(s.shape), _dp(s), _dp(r), float(radius))
    return s


def oc_update(sens: np.ndarray, rho: np.ndarray, volratio: float, min_rho: float = 0.001,
              step_limit: float = 0.02, damp: float = 0.5):
    s = _f64(sens).ravel()
    r = _f64(rho).ravel().copy()
    it = lib().ora_oc_update(s.size, _dp(s), _dp(r), float(volratio), float(min_rho), float(step_limit),
                             float(damp))
    return r.reshape(np.shape(rho)), it


def mmasub(itn: int, xvar, xmin, xmax, xold1, xold2, df0dx, gval, dgdx, low, upp, a0, a, c, d, move=1.0):
    """One MMA step; returns updated (xvar, xold1, xold2, low, upp) as new arrays."""
    x = _f64(xvar).copy()
    o1 = _f64(xold1).copy()
    o2 = _f64(xold2).copy()
    lo = _f64(low).copy()
    up = _f64(upp).copy()
    g = _f64(dgdx)
    m = g.shape[0]
    lib().ora_mmasub(int(m), x.size, int(itn), _dp(x), _dp(_f64(xmin)), _dp(_f64(xmax)), _dp(o1), _dp(o2),
                     _dp(_f64(df0dx)), _dp(_f64(gval)), _dp(g), _dp(lo), _dp(up), float(a0), _dp(_f64(a)),
                     _dp(_f64(c)), _dp(_f64(d)), float(move))
    return x, o1, o2, lo, up
