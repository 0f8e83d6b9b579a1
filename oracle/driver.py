"""Restatement of OpenTM's design driver -- TEST INFRASTRUCTURE ONLY.

Only ``tests/`` (as the checker of ``opentm_b200.driver``) and ``bench.py``'s CPU-baseline leg of
the design workload (as the timed CPU baseline) may import this module; the product never
imports it. It restates, with numpy and the FP64 oracle in this package:

* initDensity (Framework.cu:63-145): the TPMS fields P, G, D, IWP, the sphere example, the
  thresholded noise, and randTri (homogenization/Framework.cuh:237-310) with the
  randTribase_sincos basis (Framework.cuh:106-215);
* symetrize_tensor_kernel (AutoDiff/TensorExpression.cuh:70-280), in the reference's float32
  summation order, so results compare bit for bit;
* ConvergeChecker and VolumeGovernor (Framework.cuh:312-411) with float32 members;
* runCustom (Framework.cu:147-244) for both models, in FP64 around the oracle's solver.

Parity unpinned against the reference itself (it cannot be built here and ships no fixtures);
the restatement follows the cited lines, and the random streams are this library's splitmix64
streams instead of cuRAND's.
"""
from __future__ import annotations

import numpy as np

import oracle as ora

F32 = np.float32
PI_REF = F32(3.1415926)  # Framework.cu:67

SYM_REFLECT3, SYM_REFLECT6, SYM_ROTATE3, SYM_ROTATE2, SYM_NONE = 0, 1, 2, 3, 4
INIT_RANDOM, INIT_RANDCENTER, INIT_NOISE, INIT_MANUAL, INIT_INTERP, INIT_REP_RANDCENTER = 0, 1, 2, 3, 4, 5
INIT_P, INIT_G, INIT_D, INIT_IWP, INIT_EXAMPLE = 6, 7, 8, 9, 10


def uniform(seed: int, n: int) -> np.ndarray:
    """Value i of stream `seed`: splitmix64(seed * 2^32 + i) >> 11, scaled to [0, 1)."""
    c = (np.uint64(seed) << np.uint64(32)) + np.arange(n, dtype=np.uint64)
    z = c + np.uint64(0x9E3779B97F4A7C15)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def tanproj(v, beta=20.0, tau=0.5):
    """culib/lib.cuh:1372-1379 in float32."""
    v = np.asarray(v, dtype=F32)
    beta, tau = F32(beta), F32(tau)
    tb = np.tanh(beta * tau)
    return ((tb + np.tanh(beta * (v - tau))) / (tb + np.tanh(beta * (F32(1) - tau)))).astype(F32)


def _grid(n):
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    return x, y, z


def init_closed(way: int, n: int) -> np.ndarray:
    """The closed-form initial fields of Framework.cu:86-139, before the final clamp."""
    x, y, z = _grid(n)
    p = [x.astype(F32) / F32(n), y.astype(F32) / F32(n), z.astype(F32) / F32(n)]
    w2 = F32(2) * PI_REF
    if way == INIT_P:
        val = np.cos(w2 * p[0]) + np.cos(w2 * p[1]) + np.cos(w2 * p[2])
        return np.clip(tanproj(-val), F32(0.001), F32(1))
    if way == INIT_G:
        s = [np.sin(w2 * q) for q in p]
        c = [np.cos(w2 * q) for q in p]
        val = s[0] * c[1] + s[2] * c[0] + s[1] * c[2]
        return np.clip(tanproj(val), F32(0.001), F32(1))
    if way == INIT_D:
        val = (np.cos(w2 * p[0]) * np.cos(w2 * p[1]) * np.cos(w2 * p[2]) -
               np.sin(w2 * p[0]) * np.sin(w2 * p[1]) * np.sin(w2 * p[2]))
        return np.clip(tanproj(val), F32(0.001), F32(1))
    if way == INIT_IWP:
        w4 = F32(2) * F32(2) * PI_REF
        cx, cy, cz = np.cos(w2 * p[0]), np.cos(w2 * p[1]), np.cos(w2 * p[2])
        val = F32(2) * (cx * cy + cy * cz + cz * cx) - (np.cos(w4 * p[0]) + np.cos(w4 * p[1]) + np.cos(w4 * p[2]))
        return np.clip(tanproj(val), F32(0.001), F32(1))
    if way == INIT_EXAMPLE:
        d = np.sqrt((x - n / 2 + 0.5) ** 2 + (y - n / 2 + 0.5) ** 2 + (z - n / 2 + 0.5) ** 2)
        return np.where(d < n / 6.0, 0.0, 0.3).astype(F32)
    raise ValueError(way)


# ---------------------------------------------------------------------------------------
# Symmetrisation (AutoDiff/TensorExpression.cuh:70-280)
# ---------------------------------------------------------------------------------------
def _orbit_apply(f, orbits, average_div):
    """orbits: list of (z, y, x) index-array triples in summation order, one entry per orbit
    point; every orbit gets the float32 sum in that order divided by average_div."""
    v = f[orbits[0]].astype(F32)
    for o in orbits[1:]:
        v = (v + f[o]).astype(F32)
    v = (v / F32(average_div)).astype(F32)
    for o in orbits:
        f[o] = v


def symmetrize(field: np.ndarray, sym: int, average: bool = True) -> np.ndarray:
    f = np.array(field, dtype=F32, copy=True)
    nz, ny, nx = f.shape
    if sym == SYM_NONE:
        return f
    if sym == SYM_REFLECT3:
        hx, hy, hz = nx // 2, ny // 2, nz // 2
        if hx * hy * hz == 0:
            return f
        z, y, x = np.meshgrid(np.arange(hz), np.arange(hy), np.arange(hx), indexing="ij")
        x, y, z = x.ravel(), y.ravel(), z.ravel()
        orbits = []
        for i in range(8):
            fx, fy, fz = i % 2, i // 2 % 2, i // 4
            orbits.append((nz - 1 - z if fz else z, ny - 1 - y if fy else y, nx - 1 - x if fx else x))
        if average:
            _orbit_apply(f, orbits, 8)
        else:
            v = f[orbits[0]].copy()
            for o in orbits:
                f[o] = v
        return f
    if sym == SYM_ROTATE2:
        hx = nx // 2
        z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(hx), indexing="ij")
        x, y, z = x.ravel(), y.ravel(), z.ravel()
        a, b = (z, y, x), (nz - 1 - z, ny - 1 - y, nx - 1 - x)
        v = f[a].copy()
        if average:
            v = ((v + f[b]).astype(F32) / F32(2)).astype(F32)
        f[a] = v
        f[b] = v
        return f
    n = nx
    if not (nx == ny == nz):
        raise ValueError("needs a cube")
    h = n // 2
    if sym == SYM_REFLECT6:
        reps = [(x, y, z) for z in range(h) for y in range(z + 1) for x in range(y + 1)]
        if not reps:
            return f
        r = np.array(reps)
        rx, ry, rz = r[:, 0], r[:, 1], r[:, 2]
        orbits = []
        for i in range(8):
            a = n - 1 - rx if i % 2 else rx
            b = n - 1 - ry if i // 2 % 2 else ry
            c = n - 1 - rz if i // 4 else rz
            # [a,b,c], [a,c,b], [c,a,b], [c,b,a], [b,a,c], [b,c,a] as (x, y, z)
            for px, py, pz in ((a, b, c), (a, c, b), (c, a, b), (c, b, a), (b, a, c), (b, c, a)):
                orbits.append((pz, py, px))
        _orbit_apply(f, orbits, 48)
        return f
    if sym == SYM_ROTATE3:
        if n % 2:
            raise ValueError("needs an even cube")
        reps = []
        for z in range(h):
            for y in range(z + 1):
                for x in range(z + 1):
                    key = y * (z + 1) + x
                    # one writer per orbit: skip when a cyclic rotation is an earlier representative
                    if x == z and z * (z + 1) + y < key:
                        continue
                    if y == z and x * (z + 1) + z < key:
                        continue
                    reps.append((x, y, z))
        r = np.array(reps)
        rep = [r[:, 0], r[:, 1], r[:, 2]]
        perm = [(0, 2, 1), (2, 1, 0), (1, 0, 2), (2, 0, 1), (1, 2, 0), (0, 1, 2)]
        orbits = []
        for i in range(6):
            o = [rep[perm[i][0]], rep[perm[i][1]], rep[perm[i][2]]]
            P = [h + o[0], h + o[1], h + o[2]]
            M = [h - 1 - o[0], h - 1 - o[1], h - 1 - o[2]]
            if i < 3:
                pts = [(M[0], P[1], P[2]), (P[0], M[1], P[2]), (P[0], P[1], M[2]), (M[0], M[1], M[2])]
            else:
                pts = [(P[0], P[1], P[2]), (M[0], M[1], P[2]), (P[0], M[1], M[2]), (M[0], P[1], M[2])]
            for px, py, pz in pts:
                orbits.append((pz, py, px))
        _orbit_apply(f, orbits, 24)
        return f
    raise ValueError(sym)


# ---------------------------------------------------------------------------------------
# randTri (Framework.cuh:106-215, 237-310)
# ---------------------------------------------------------------------------------------
def randtri_count(n_period: int, centered: bool) -> int:
    return 6 * n_period + 36 * n_period * n_period + (4 if centered else 0)


def randtri_coefficients(seed: int, n_period: int, centered: bool) -> np.ndarray:
    return (-1.0 + 2.0 * uniform(seed, randtri_count(n_period, centered))).astype(F32)


def quat_rotation(q) -> np.ndarray:
    w, x, y, z = (float(v) for v in q)
    nrm = np.sqrt(w * w + x * x + y * y + z * z)
    w, x, y, z = w / nrm, x / nrm, y / nrm, z / nrm
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def randtri_field(n: int, n_period: int, coeffs, centered: bool) -> np.ndarray:
    """The basis sum in FP64 at p = idx / (n - 1) (rotated about the centre when centered)."""
    c = np.asarray(coeffs, dtype=np.float64)
    npd = n_period
    x, y, z = _grid(n)
    p = np.stack([x / (n - 1.0), y / (n - 1.0), z / (n - 1.0)]).reshape(3, -1)
    if centered:
        R = quat_rotation(c[6 * npd + 36 * npd * npd:][:4])
        p = R @ (p - 0.5)
    g = np.zeros((6 * npd, p.shape[1]))
    for a in range(3):
        for fq in range(npd):
            g[a * npd + fq] = np.cos(2 * np.pi * (fq + 1) * p[a])
            g[3 * npd + a * npd + fq] = np.sin(2 * np.pi * (fq + 1) * p[a])
    s = np.zeros(p.shape[1])
    nb1 = 6 * npd
    for i in range(nb1):
        ii = i if i < 3 * npd else i - 3 * npd
        s += c[i] * g[(0 if i < 3 * npd else 3 * npd) + (ii % 3) * npd + ii // 3]
    C2 = c[nb1:nb1 + nb1 * nb1].reshape(nb1, nb1)
    s += np.einsum("jv,jk,kv->v", g, C2, g)
    return s.reshape(n, n, n)


def level_map(val, t, M, m):
    """sigmoid(val, 15, t) (M - m) + m in float32 (culib/lib.cuh:1381-1383)."""
    val = np.asarray(val, dtype=F32)
    with np.errstate(over="ignore"):  # exp overflows to inf and the sigmoid to 0, as expf does
        sig = (F32(1) / (F32(1) + np.exp(-F32(15) * (val - F32(t))))).astype(F32)
    return (sig * (F32(M) - F32(m)) + F32(m)).astype(F32)


def randtri_init(n, n_period, coeffs, centered, sym, vol):
    f = randtri_field(n, n_period, coeffs, centered).astype(F32)
    f = symmetrize(f, sym)
    volf = F32(vol)
    M, m = min(volf * F32(1.5), F32(1)), F32(0.001)
    t_u = F32(n_period * n_period * 37)
    t_l = -t_u
    t = (t_u + t_l) / F32(2)
    for _ in range(60):
        t = F32((t_u + t_l) / F32(2))
        sv = F32(np.mean(level_map(f, t, M, m).astype(np.float64)))
        if abs(sv - volf) / volf < F32(1e-3):
            break
        if sv > volf:
            t_l = t
        if sv < volf:
            t_u = t
    return level_map(f, t, M, m)


def noise_init(n, seed, sym, vol):
    f = uniform(seed, n ** 3).astype(F32).reshape(n, n, n)
    f = symmetrize(f, sym)
    r = tanproj(f)
    r = np.where(r < F32(0.5), F32(1e-9), r)
    r = np.where(r > F32(0.5), F32(1), r).astype(F32)
    s = F32(vol) / F32(np.mean(r.astype(np.float64)))
    v = (r * s).astype(F32)
    v = np.where(v < F32(0.001), F32(0.001), v)
    return np.where(v >= F32(1), F32(1), v).astype(F32)


def init_density(winit, n, sym=SYM_NONE, vol=0.3, n_period=10, seed=0, coeffs=None):
    if winit in (INIT_P, INIT_G, INIT_D, INIT_IWP, INIT_EXAMPLE):
        f = init_closed(winit, n)
    elif winit == INIT_NOISE:
        f = noise_init(n, seed, sym, vol)
    elif winit in (INIT_RANDOM, INIT_RANDCENTER, INIT_REP_RANDCENTER):
        centered = winit != INIT_RANDOM
        if coeffs is None:
            coeffs = randtri_coefficients(seed, n_period, centered)
        f = randtri_init(n, n_period, coeffs, centered, sym, vol)
    else:
        raise ValueError(winit)
    f = symmetrize(f, sym)
    return np.clip(f, F32(0.1), F32(1)).astype(F32)


# ---------------------------------------------------------------------------------------
# ConvergeChecker, VolumeGovernor (Framework.cuh:312-411)
# ---------------------------------------------------------------------------------------
class ConvergeChecker:
    def __init__(self, thres=1e-3):
        self.thres = float(thres)
        self.obj = [0.0] * 10
        self.p = 0

    def is_converge(self, it, obj):
        eid = it % 10
        self.p = eid
        self.obj[eid] = float(obj)
        if it <= 11:
            return False
        out = False
        for i in range(3):
            a, b = self.obj[(self.p - i) % 10], self.obj[(self.p - i - 1) % 10]
            out = out or abs(a - b) / abs(b) > self.thres
        return not out


class VolumeGovernor:
    """float members; arithmetic with double literals is done in double and stored as float."""

    def __init__(self):
        self.low, self.vb, self.dec, self.df = F32(0), F32(1), F32(0), F32(1)
        self.val_last, self.vib = F32(1), F32(0)
        self.vib_count = 0
        self.count = 0

    def _shrink(self):
        self.dec = F32(self.vb - self.low)
        self.vb = F32(self.vb - F32(self.df * self.dec))
        if float(self.df) > 0.05:
            self.df = F32(float(self.df) * 0.8)

    def _expand(self):
        self.vb = F32(float(self.vb) + 0.3 * float(self.dec) * float(self.df))

    def volume_check(self, value, low, volfrac, itn):
        value, low, volfrac = F32(value), F32(low), F32(volfrac)
        self.low = low
        if float(value) + 0.0001 < 1e-4 or itn == 100:
            self._shrink()
            if float(self.df) <= 0.05:
                return 1
            self.count = 0
        reach = float(abs(F32(self.vb - volfrac))) < 1e-2
        if F32(self.vib * F32(self.val_last - value)) < 0:
            self.vib_count += 1
        else:
            self.vib_count = 0
        if self.vib_count >= 8:
            if reach:
                self._expand()
                self.vib_count = 0
            else:
                self._shrink()
        self.vib = F32(self.val_last - value)
        if float(F32(self.val_last - value)) < 1e-4 and float(value) > 1e-4 and reach:
            self.count += 1
        else:
            self.count = 0
        if self.count >= 5:
            self.vb = F32(float(self.vb) + 0.3 * float(self.dec) * float(self.df))
            self.count = 0
        self.val_last = value
        return 0

    def get_current_decrease(self):
        return F32(self.df * self.dec)


# ---------------------------------------------------------------------------------------
# runCustom (Framework.cu:147-244)
# ---------------------------------------------------------------------------------------
OBJ_ENTRIES = ((0, 0), (1, 1), (2, 2), (0, 1), (2, 1), (0, 2))


def objective(K, tt):
    """Framework.cu:168-170 in float32, and dObj/dK."""
    K32 = np.asarray(K, dtype=F32).reshape(3, 3)
    v = F32(0)
    dK = np.zeros((3, 3), dtype=F32)
    for e, (i, j) in enumerate(OBJ_ENTRIES):
        r = F32(K32[i, j] - F32(tt[e]))
        v = F32(v + r * r)
        dK[i, j] = F32(2) * r
    return F32(v - F32(1e-4)), dK


def run_custom(rho0, model, heat_ratio=(1.0, 0.0), target=(0.3, 0.2, 0.1, 0.0, 0.0, 0.0), iters=3,
               finthres=5e-4, sym=SYM_NONE, tol=1e-10):
    """The design loop in FP64 from rho0; returns (rho, objective history)."""
    rho = np.asarray(rho0, dtype=np.float64).copy()
    n = rho.shape[0]
    ne = rho.size
    k0, kmin = heat_ratio
    chk = ConvergeChecker(finthres)
    gov = VolumeGovernor()
    hist = []
    state = None
    for itn in range(iters):
        rho_f, wsum = ora.conv_forward(rho, ora.WEIGHT_SPLINE4, 1.5, False)
        k = rho_f ** 3 * (k0 - kmin) + kmin
        sol = ora.homogenize(k, tol=tol, want_energy=True)
        val, dK = objective(sol["C"], target)
        hist.append(float(val))
        if model == "oc":
            gov.volume_check(val, np.mean(k), np.mean(rho), itn)
        g_k = ora.sensitivity(sol["energy"], k, dK.astype(np.float64))
        g_rho = ora.conv_backward(g_k * (3.0 * rho_f ** 2 * (k0 - kmin)), wsum, ora.WEIGHT_SPLINE4, 1.5, False)
        if model == "oc":
            if chk.is_converge(itn, val) and gov.get_current_decrease() < 1e-4:
                break
            rho = symmetrize(rho.astype(F32), sym).astype(np.float64)
            g_rho = symmetrize(g_rho.astype(F32), sym).astype(np.float64)
            g_rho = ora.oc_filter_sens(g_rho, rho, 2.0)
            rho, _ = ora.oc_update(g_rho, rho, float(gov.vb), 0.001, 0.02, 0.5)
        else:
            if chk.is_converge(itn, val):
                break
            if state is None:
                state = [np.zeros(ne) for _ in range(4)]  # xold1, xold2, low, upp start at zero
            o1, o2, lo, up = state
            x, o1, o2, lo, up = ora.mmasub(itn, rho.astype(F32).astype(np.float64).ravel(), np.full(ne, 1e-4),
                                           np.ones(ne), o1, o2, np.full(ne, F32(1.0 / ne), dtype=np.float64),
                                           np.array([float(val)]), g_rho.astype(F32).astype(np.float64).reshape(1, ne),
                                           lo, up, 1.0, np.zeros(1), np.full(1, 1e7), np.ones(1), 1.0)
            state = [o1, o2, lo, up]
            rho = x.astype(F32).astype(np.float64).reshape(rho.shape)
    return rho, np.array(hist)
