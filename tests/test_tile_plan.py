"""CPU emulation of the tile-staged fine smoother and residual (opentm_b200/csrc/otm_tile.cuh).

The kernels' index arithmetic is restated here line by line (tile origins of both tilings, the
periodic wrap of shifted tiles, the parity-split and padded shared-memory site order, the thread ->
column-segment mapping, the six-plane streaming of a pass, the right-hand-side boxes the TMA copies
deliver, the staged coarse block and the quad-wise prolongation, the write-back) and every
shared-memory and global access is checked to stay in bounds before the kernels run on a GPU.
Within a pass no thread may read the values (.xyz) of a site that another thread writes in the
same pass, and the write-back must cover each vertex once. The emulated arithmetic is then compared
with an independent block Gauss-Seidel (whole 27-point rows, colour pairs in order, halo frozen,
tiles of either tiling) and an independent residual, so the streaming algebra (which plane's
conductivities feed which coefficient) is checked too."""
import numpy as np
import pytest

TX, TY, TZ = 16, 16, 8  # interior vertices of a tile
SX, SY, SZ = TX + 2, TY + 2, TZ + 2
SHALF = SX // 2
SROW = SX + 1  # padded row pitch
SPLANE, SSITES = SROW * SY, SROW * SY * SZ
THREADS, SEG, RTHREADS = 128, 4, 256
CX, CY, CZ = TX // 2 + 2, TY // 2 + 2, TZ // 2 + 2
CSITES = CX * CY * CZ
FBX, FBY, FBZ = 8, 8, 4
FBOX = FBX * FBY * FBZ * 3
FCASE = FBX * FBY * FBZ
OP = dict(c0=0.35, c2=-0.08, c3=-0.095)  # distinct c2 / c3 so that a mix-up shows
NBR = [(-1, -1), (0, -1), (1, -1), (-1, 0), (1, 0), (-1, 1), (0, 1), (1, 1)]


def wrapm(a, n):
    assert -n <= a < 2 * n
    return a + n if a < 0 else (a - n if a >= n else a)


def tsite(lx, ly, lz):
    assert 0 <= lx < SX and 0 <= ly < SY and 0 <= lz < SZ
    return lz * SPLANE + ly * SROW + ((SHALF + (lx >> 1)) if (lx & 1) else (lx >> 1))


def rsite(lx, ly, lz):
    assert 0 <= lx < SX and 0 <= ly < SY and 0 <= lz < SZ
    return lz * SPLANE + ly * SROW + lx


def gidx(d, x, y, z):
    nx, ny, nz = d
    assert 0 <= x < nx and 0 <= y < ny and 0 <= z < nz
    return x + nx * (y + ny * z)


def tile_origin(d, b, shift):
    nx, ny, nz = d
    ntx, nty = nx // TX, ny // TY
    q = b // ntx
    return ((b - q * ntx) * TX + shift * (TX // 2), (q % nty) * TY + shift * (TY // 2),
            (q // nty) * TZ + shift * (TZ // 2))


def fpos(x, y, z):
    assert 0 <= x < TX and 0 <= y < TY and 0 <= z < TZ
    return ((x >> 3) + 2 * (y >> 3) + 4 * (z >> 2)) * FBOX + ((z & 3) * FBY + (y & 7)) * FBX + (x & 7)


def f_box(d, f, x0, y0, z0):
    """The eight TMA copies: box q = {8, 8, 4, 3} of the right-hand side at the wrapped origin
    (x0 + 8 (q & 1), y0 + 8 ((q >> 1) & 1), z0 + 4 (q >> 2), 0), landing at q * 768, x fastest."""
    nx, ny, nz = d
    nv = nx * ny * nz
    box = np.full(8 * FBOX, np.nan)
    for q in range(8):
        X, Y, Z = wrapm(x0 + FBX * (q & 1), nx), wrapm(y0 + FBY * ((q >> 1) & 1), ny), wrapm(z0 + FBZ * (q >> 2), nz)
        assert X + FBX <= nx and Y + FBY <= ny and Z + FBZ <= nz, "a box never crosses the periodic boundary"
        assert (X * 4) % 16 == 0, "TMA: the innermost coordinate times the element size is a multiple of 16 bytes"
        for c in range(3):
            for z in range(FBZ):
                for y in range(FBY):
                    for x in range(FBX):
                        box[q * FBOX + ((c * FBZ + z) * FBY + y) * FBX + x] = f[c * nv + gidx(d, X + x, Y + y, Z + z)]
    # the position function the passes use reads the values of the global array
    for c in range(3):
        for z in range(TZ):
            for y in range(TY):
                for x in range(TX):
                    g = gidx(d, wrapm(x0 + x, nx), wrapm(y0 + y, ny), wrapm(z0 + z, nz))
                    assert box[fpos(x, y, z) + c * FCASE] == f[c * nv + g]
    return box


def plane_coef(K):
    c2, c3 = OP["c2"], OP["c3"]
    return [c3 * K[0], c2 * (K[0] + K[1]), c3 * K[1], c2 * (K[0] + K[2]), c2 * (K[1] + K[3]), c3 * K[2],
            c2 * (K[2] + K[3]), c3 * K[3]]


class Smem:
    """Shared memory of one CTA with access checks."""

    def __init__(self, n):
        self.v = np.zeros((n, 4))
        self.n = n
        self.writes = {}
        self.reads = {}

    def rd(self, i, who, comp="xyzw"):
        assert 0 <= i < self.n, i
        self.reads.setdefault(i, set()).add((who, comp))
        return self.v[i]

    def wr(self, i, val, who):
        assert 0 <= i < self.n, i
        self.writes.setdefault(i, set()).add(who)
        self.v[i] = val

    def check_pass(self):
        for i, ws in self.writes.items():
            assert len(ws) == 1, f"site {i} written by {ws}"
            (w,) = ws
            for (who, comp) in self.reads.get(i, ()):
                assert who == w or comp == "w", f"site {i} written by {w}, read by {who}"
        self.writes, self.reads = {}, {}


def emulate_pass(sm, px, py, fsm, fs):
    """tile_pass<PX, PY>: 128 threads, each a column segment of 4 vertices, 6 planes streamed."""
    oL, oR = (SHALF - 1, SHALF) if px else (-SHALF, -SHALF + 1)
    for t in range(THREADS):
        i, j, seg = t & 7, (t >> 3) & 7, t >> 6
        lx, ly, lz0 = 2 * i + 1 + px, 2 * j + 1 + py, 1 + SEG * seg
        assert 1 <= lx <= TX and 1 <= ly <= TY and 1 <= lz0 and lz0 + SEG - 1 <= TZ
        # the compile-time neighbour offsets equal the site order's
        assert tsite(lx - 1, ly, 1) - tsite(lx, ly, 1) == oL and tsite(lx + 1, ly, 1) - tsite(lx, ly, 1) == oR
        fcol = fpos(lx - 1, ly - 1, lz0 - 1)
        Kp, Cp = [0.0] * 4, None
        accA, accB, accC = [0.0] * 3, [0.0] * 3, [0.0] * 3
        dA = dB = 0.0
        for s in range(SEG + 2):
            P = lz0 - 1 + s
            b = tsite(lx, ly, P)
            offs = [oL - SROW, -SROW, oR - SROW, oL, oR, oL + SROW, SROW, oR + SROW]
            for n, (ox, oy) in enumerate(NBR):
                assert b + offs[n] == tsite(lx + ox, ly + oy, P)
            nb = [sm.rd(b + o, t) for o in offs]
            kown = sm.rd(b, t, "w")[3]
            K = [nb[0][3], nb[1][3], nb[3][3], kown]
            sK = (K[0] + K[1]) + (K[2] + K[3])
            C = plane_coef(K)
            dC = 0.0
            if s < SEG:
                fv = fcol + s * (FBX * FBY)
                assert fv == fpos(lx - 1, ly - 1, lz0 - 1 + s)
                accC = [fsm[fv + c * FCASE] * fs[c] for c in range(3)]
                for n in range(8):
                    for c in range(3):
                        accC[c] -= C[n] * nb[n][c]
                dC = sK
            if 1 <= s <= SEG:
                for q, n in enumerate((0, 2, 5, 7)):
                    w = OP["c2"] * (Kp[q] + K[q])
                    for c in range(3):
                        accB[c] -= w * nb[n][c]
                dB += sK
            if s >= 2:
                for n in range(8):
                    for c in range(3):
                        accA[c] -= Cp[n] * nb[n][c]
                inv = 1.0 / (OP["c0"] * dA)
                sm.wr(tsite(lx, ly, P - 1), [accA[0] * inv, accA[1] * inv, accA[2] * inv, Kp[3]], t)
            accA, accB = accB, accC
            accC = [0.0] * 3
            dA, dB = dB, dC
            Kp, Cp = K, C
    sm.check_pass()


def prolong_site(cb, ux, uy, uz, c0x, c0y, c0z):
    ax0, ay0, az0 = (ux >> 1) - c0x, (uy >> 1) - c0y, (uz >> 1) - c0z
    ax1, ay1, az1 = ax0 + (ux & 1), ay0 + (uy & 1), az0 + (uz & 1)
    for a, n in ((ax0, CX), (ax1, CX), (ay0, CY), (ay1, CY), (az0, CZ), (az1, CZ)):
        assert 0 <= a < n
    wx1, wy1, wz1 = [0.5 if (q & 1) else 0.0 for q in (ux, uy, uz)]
    wx0, wy0, wz0 = 1 - wx1, 1 - wy1, 1 - wz1
    r00, r10 = (ay0 + CY * az0) * CX, (ay1 + CY * az0) * CX
    r01, r11 = (ay0 + CY * az1) * CX, (ay1 + CY * az1) * CX
    out = []
    for c in range(3):
        u = cb[:, c]
        out.append(wz0 * (wy0 * (wx0 * u[r00 + ax0] + wx1 * u[r00 + ax1]) +
                          wy1 * (wx0 * u[r10 + ax0] + wx1 * u[r10 + ax1])) +
                   wz1 * (wy0 * (wx0 * u[r01 + ax0] + wx1 * u[r01 + ax1]) +
                          wy1 * (wx0 * u[r11 + ax0] + wx1 * u[r11 + ax1])))
    return out


def prolong_quad(cb, xs, uy, uz, c0x, c0y, c0z):
    """The quad-wise prolongation: 3 coarse columns per coarse row, 4 fine sites."""
    assert xs % 2 == 0
    ax = (xs >> 1) - c0x
    ay0, az0 = (uy >> 1) - c0y, (uz >> 1) - c0z
    ay1, az1 = ay0 + (uy & 1), az0 + (uz & 1)
    wy1, wz1 = (0.5 if uy & 1 else 0.0), (0.5 if uz & 1 else 0.0)
    wy0, wz0 = 1 - wy1, 1 - wz1
    rows = [(ay0 + CY * az0) * CX + ax, (ay1 + CY * az0) * CX + ax, (ay0 + CY * az1) * CX + ax,
            (ay1 + CY * az1) * CX + ax]
    for r in rows:
        assert 0 <= r and r + 2 < CSITES and (r % CX) + 2 < CX
    v = [[cb[r + a] for a in range(3)] for r in rows]
    # each coarse column interpolated over (y, z), then over x: even sites take a column, odd
    # sites the mean of two
    col = [[wz0 * (wy0 * v[0][a][c] + wy1 * v[1][a][c]) + wz1 * (wy0 * v[2][a][c] + wy1 * v[3][a][c])
            for c in range(3)] for a in range(3)]
    out = [col[0], [0.5 * (col[0][c] + col[1][c]) for c in range(3)], col[1],
           [0.5 * (col[1][c] + col[2][c]) for c in range(3)]]
    # the values of the per-site prolongation, summed in another order
    for e in range(4):
        ref = prolong_site(cb, xs + e, uy, uz, c0x, c0y, c0z)
        assert all(abs(out[e][c] - ref[c]) <= 1e-6 * (1.0 + abs(ref[c])) for c in range(3))
    return out


def emulate_sweep(d, dc, ks, u_in, uc, f, start, shift, reverse, fs=(1.0, 1.0, 1.0)):
    """k_tile_sweep<start> over all tiles of tiling `shift`. start: 0 zero, 1 u_in, 2 u_in + P uc."""
    nx, ny, nz = d
    nv = nx * ny * nz
    ntiles = (nx // TX) * (ny // TY) * (nz // TZ)
    out = np.full(3 * nv, np.nan)
    written = np.zeros(nv, dtype=int)
    pos = sorted(tsite(lx, ly, lz) for lz in range(SZ) for ly in range(SY) for lx in range(SX))
    assert len(set(pos)) == SX * SY * SZ and pos[-1] < SSITES, "the site order is one-to-one and in bounds"
    for b in range(ntiles):
        x0, y0, z0 = tile_origin(d, b, shift)
        fsm = f_box(d, f, x0, y0, z0)
        sm = Smem(SSITES)
        c0x, c0y, c0z = x0 // 2 - 1, y0 // 2 - 1, z0 // 2 - 1
        cb = np.zeros((CSITES, 4))
        if start == 2:
            cnx, cny, cnz = dc
            nvc = cnx * cny * cnz
            for s in range(CSITES):
                ax, ay, az = s % CX, (s // CX) % CY, s // (CX * CY)
                g = gidx(dc, wrapm(c0x + ax, cnx), wrapm(c0y + ay, cny), wrapm(c0z + az, cnz))
                cb[s] = [uc[g], uc[nvc + g], uc[2 * nvc + g], 0.0]
        staged = {}
        for w in range(SY * SZ * (TX // 4)):
            q, row = w & 3, w >> 2
            ly, lz = row % SY, row // SY
            uy, uz = y0 - 1 + ly, z0 - 1 + lz
            g = gidx(d, wrapm(x0 + 4 * q, nx), wrapm(uy, ny), wrapm(uz, nz))
            assert g % 4 == 0 and g + 3 < nv and (g + 3) // nx == g // nx  # one aligned 4-wide vector in a row
            p = prolong_quad(cb, x0 + 4 * q, uy, uz, c0x, c0y, c0z) if start == 2 else None
            for e in range(4):
                v = [0.0, 0.0, 0.0, ks[g + e]]
                if start >= 1:
                    v = [u_in[c * nv + g + e] for c in range(3)] + [ks[g + e]]
                if start == 2:
                    v = [v[c] + p[e][c] for c in range(3)] + [ks[g + e]]
                i = tsite(1 + 4 * q + e, ly, lz)
                staged[i] = staged.get(i, 0) + 1
                sm.wr(i, v, -1)
        for w in range(SY * SZ * 2):
            side, row = w & 1, w >> 1
            ly, lz = row % SY, row // SY
            lx = SX - 1 if side else 0
            ux, uy, uz = x0 - 1 + lx, y0 - 1 + ly, z0 - 1 + lz
            g = gidx(d, wrapm(ux, nx), wrapm(uy, ny), wrapm(uz, nz))
            v = [0.0, 0.0, 0.0, ks[g]]
            if start >= 1:
                v = [u_in[c * nv + g] for c in range(3)] + [ks[g]]
            if start == 2:
                p = prolong_site(cb, ux, uy, uz, c0x, c0y, c0z)
                v = [v[c] + p[c] for c in range(3)] + [ks[g]]
            i = tsite(lx, ly, lz)
            staged[i] = staged.get(i, 0) + 1
            sm.wr(i, v, -1)
        assert len(staged) == SX * SY * SZ and set(staged.values()) == {1}, "every site staged once"
        sm.writes, sm.reads = {}, {}
        for p in ((3, 2, 1, 0) if reverse else (0, 1, 2, 3)):
            emulate_pass(sm, p & 1, p >> 1, fsm, fs)
        for w in range(TX * TY * TZ // 4):
            q, row = w & 3, w >> 2
            ly, lz = 1 + row % TY, 1 + row // TY
            g = gidx(d, wrapm(x0 + 4 * q, nx), wrapm(y0 + ly - 1, ny), wrapm(z0 + lz - 1, nz))
            assert g % 4 == 0
            for e in range(4):
                o = sm.v[tsite(1 + 4 * q + e, ly, lz)]
                written[g + e] += 1
                for c in range(3):
                    out[c * nv + g + e] = o[c]
    assert (written == 1).all()
    return out


def emulate_resid(d, ks, u, f, fs=(1.0, 1.0, 1.0)):
    """k_tile_resid over all tiles of tiling 0: 256 threads, one column each, 10 planes streamed."""
    nx, ny, nz = d
    nv = nx * ny * nz
    r = np.full(3 * nv, np.nan)
    written = np.zeros(nv, dtype=int)
    for b in range((nx // TX) * (ny // TY) * (nz // TZ)):
        x0, y0, z0 = tile_origin(d, b, 0)
        fsm = f_box(d, f, x0, y0, z0)
        sm = np.full((SSITES, 4), np.nan)
        for w in range(SY * SZ * (TX // 4)):
            q, row = w & 3, w >> 2
            ly, lz = row % SY, row // SY
            g = gidx(d, wrapm(x0 + 4 * q, nx), wrapm(y0 - 1 + ly, ny), wrapm(z0 - 1 + lz, nz))
            for e in range(4):
                sm[rsite(1 + 4 * q + e, ly, lz)] = [u[g + e], u[nv + g + e], u[2 * nv + g + e], ks[g + e]]
        for w in range(SY * SZ * 2):
            side, row = w & 1, w >> 1
            ly, lz = row % SY, row // SY
            lx = SX - 1 if side else 0
            g = gidx(d, wrapm(x0 - 1 + lx, nx), wrapm(y0 - 1 + ly, ny), wrapm(z0 - 1 + lz, nz))
            sm[rsite(lx, ly, lz)] = [u[g], u[nv + g], u[2 * nv + g], ks[g]]
        for t in range(RTHREADS):
            lx, ly = 1 + (t & 15), 1 + (t >> 4)
            col = gidx(d, x0 + lx - 1, y0 + ly - 1, 0)
            pl = nx * ny
            Kp, Cp = [0.0] * 4, None
            accA, accB, accC = [0.0] * 3, [0.0] * 3, [0.0] * 3
            dA = dB = 0.0
            uA, uB = [0.0] * 3, [0.0] * 3
            for P in range(SZ):
                b0 = rsite(lx, ly, P)
                offs = [-SROW - 1, -SROW, -SROW + 1, -1, 1, SROW - 1, SROW, SROW + 1]
                for n, (ox, oy) in enumerate(NBR):
                    assert b0 + offs[n] == rsite(lx + ox, ly + oy, P)
                nb = [sm[b0 + o] for o in offs]
                own = sm[b0]
                assert not np.isnan(own).any() and not any(np.isnan(x).any() for x in nb), "read a staged site"
                K = [nb[0][3], nb[1][3], nb[3][3], own[3]]
                sK = (K[0] + K[1]) + (K[2] + K[3])
                C = plane_coef(K)
                dC = 0.0
                if P + 1 <= TZ:
                    fv = fpos(lx - 1, ly - 1, P)
                    accC = [fsm[fv + c * FCASE] * fs[c] for c in range(3)]
                    for n in range(8):
                        for c in range(3):
                            accC[c] -= C[n] * nb[n][c]
                    dC = sK
                if 1 <= P <= TZ:
                    for q, n in enumerate((0, 2, 5, 7)):
                        w = OP["c2"] * (Kp[q] + K[q])
                        for c in range(3):
                            accB[c] -= w * nb[n][c]
                    dB += sK
                    uB = list(own[:3])
                if P >= 2:
                    for n in range(8):
                        for c in range(3):
                            accA[c] -= Cp[n] * nb[n][c]
                    diag = OP["c0"] * dA
                    g = col + (z0 + P - 2) * pl
                    assert 0 <= g < nv
                    written[g] += 1
                    for c in range(3):
                        r[c * nv + g] = accA[c] - diag * uA[c]
                accA, accB, accC = accB, accC, [0.0] * 3
                uA = uB
                dA, dB = dB, dC
                Kp, Cp = K, C
    assert (written == 1).all()
    return r


# ---- independent restatements: whole 27-point rows ----------------------------------------
def row_coefs(d, ks, x, y, z):
    """A(v, v+o) for the 27 offsets of vertex (x,y,z) with c1 = 0."""
    nx, ny, nz = d
    k8 = {}
    for bz in (0, 1):
        for by in (0, 1):
            for bx in (0, 1):
                k8[(bx, by, bz)] = ks[gidx(d, (x - 1 + bx) % nx, (y - 1 + by) % ny, (z - 1 + bz) % nz)]
    c = {0: OP["c0"], 1: 0.0, 2: OP["c2"], 3: OP["c3"]}
    out = {}
    for oz in (-1, 0, 1):
        for oy in (-1, 0, 1):
            for ox in (-1, 0, 1):
                nzc = (ox != 0) + (oy != 0) + (oz != 0)
                ssum = 0.0
                for (bx, by, bz), kv in k8.items():
                    ok = all((o > 0 and b == 1) or (o < 0 and b == 0) or o == 0
                             for o, b in ((ox, bx), (oy, by), (oz, bz)))
                    if ok:
                        ssum += kv
                out[(ox, oy, oz)] = c[nzc] * ssum
    return out


def block_gs(d, ks, u0, f, order, shift):
    """One colour-pair Gauss-Seidel sweep per 16 x 16 x 8 block of tiling `shift` (blocks shifted by
    half a block along every axis for shift 1, wrapping periodically), the halo (every neighbour
    outside the block, periodic images of the block's own vertices included) frozen at u0."""
    nx, ny, nz = d
    nv = nx * ny * nz
    sx, sy, sz = shift * TX // 2, shift * TY // 2, shift * TZ // 2
    out = u0.copy()
    for z0 in range(sz, nz + sz, TZ):
        for y0 in range(sy, ny + sy, TY):
            for x0 in range(sx, nx + sx, TX):
                loc = u0.copy()
                for p in order:
                    px, py = p & 1, p >> 1
                    for z in range(z0, z0 + TZ):
                        for y in range(y0 + py, y0 + TY, 2):
                            for x in range(x0 + px, x0 + TX, 2):
                                A = row_coefs(d, ks, x % nx, y % ny, z % nz)
                                v = gidx(d, x % nx, y % ny, z % nz)
                                for c in range(3):
                                    s = f[c * nv + v]
                                    for (ox, oy, oz), a in A.items():
                                        if (ox, oy, oz) == (0, 0, 0):
                                            continue
                                        inside = (x0 <= x + ox < x0 + TX and y0 <= y + oy < y0 + TY
                                                  and z0 <= z + oz < z0 + TZ)
                                        src = loc if inside else u0  # the halo stays at u0
                                        s -= a * src[c * nv + gidx(d, (x + ox) % nx, (y + oy) % ny, (z + oz) % nz)]
                                    loc[c * nv + v] = s / A[(0, 0, 0)]
                for z in range(z0, z0 + TZ):
                    for y in range(y0, y0 + TY):
                        for x in range(x0, x0 + TX):
                            v = gidx(d, x % nx, y % ny, z % nz)
                            for c in range(3):
                                out[c * nv + v] = loc[c * nv + v]
    return out


def residual(d, ks, u, f):
    nx, ny, nz = d
    nv = nx * ny * nz
    r = np.zeros(3 * nv)
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                A = row_coefs(d, ks, x, y, z)
                v = gidx(d, x, y, z)
                for c in range(3):
                    s = f[c * nv + v]
                    for (ox, oy, oz), a in A.items():
                        s -= a * u[c * nv + gidx(d, (x + ox) % nx, (y + oy) % ny, (z + oz) % nz)]
                    r[c * nv + v] = s
    return r


def prolong(d, dc, uc):
    nx, ny, nz = d
    cnx, cny, cnz = dc
    nv, nvc = nx * ny * nz, cnx * cny * cnz
    out = np.zeros(3 * nv)
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                v = gidx(d, x, y, z)
                for c in range(3):
                    a = 0.0
                    for (X, wx) in ((x // 2, 1.0),) if x % 2 == 0 else ((x // 2, 0.5), ((x // 2 + 1) % cnx, 0.5)):
                        for (Y, wy) in ((y // 2, 1.0),) if y % 2 == 0 else ((y // 2, 0.5), ((y // 2 + 1) % cny, 0.5)):
                            for (Z, wz) in ((z // 2, 1.0),) if z % 2 == 0 else ((z // 2, 0.5), ((z // 2 + 1) % cnz, 0.5)):
                                a += wx * wy * wz * uc[c * nvc + gidx(dc, X, Y, Z)]
                    out[c * nv + v] = a
    return out


@pytest.fixture(scope="module")
def fields():
    rng = np.random.default_rng(7)
    d = (32, 16, 16)  # two tiles along x and z: halos cross tile faces, shifted tiles wrap
    dc = (16, 8, 8)
    nv, nvc = 32 * 16 * 16, 16 * 8 * 8
    ks = 0.001 + rng.random(nv)
    f = rng.standard_normal(3 * nv)
    u_in = rng.standard_normal(3 * nv)
    uc = rng.standard_normal(3 * nvc)
    return d, dc, ks, f, u_in, uc


def test_sweep_from_zero_forward_tiling0(fields):
    d, dc, ks, f, u_in, uc = fields
    got = emulate_sweep(d, dc, ks, None, None, f, start=0, shift=0, reverse=False)
    ref = block_gs(d, ks, np.zeros_like(f), f, (0, 1, 2, 3), 0)
    assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()


def test_sweep_from_u_forward_shifted_tiling(fields):
    d, dc, ks, f, u_in, uc = fields
    got = emulate_sweep(d, dc, ks, u_in, None, f, start=1, shift=1, reverse=False)
    ref = block_gs(d, ks, u_in, f, (0, 1, 2, 3), 1)
    assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()


def test_sweep_with_prolongation_reverse_shifted_tiling(fields):
    d, dc, ks, f, u_in, uc = fields
    got = emulate_sweep(d, dc, ks, u_in, uc, f, start=2, shift=1, reverse=True)
    ref = block_gs(d, ks, u_in + prolong(d, dc, uc), f, (3, 2, 1, 0), 1)
    assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()


def test_residual_indices_and_values(fields):
    d, dc, ks, f, u_in, uc = fields
    got = emulate_resid(d, ks, u_in, f)
    ref = residual(d, ks, u_in, f)
    assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()


# ---- coarse levels: otm_ctile.cuh -----------------------------------------------------------
CTX, CTY, CTZ = 16, 8, 8
CSX, CSY, CSZ = CTX + 2, CTY + 2, CTZ + 2
CSHALF, CSROW = CSX // 2, CSX + 1
CSPLANE, CSSITES = CSROW * CSY, CSROW * CSY * CSZ
CTHREADS = (CTX // 2) * (CTY // 2) * (CTZ // 2)
CCX, CCY, CCZ = CTX // 2 + 2, CTY // 2 + 2, CTZ // 2 + 2
CCSITES = CCX * CCY * CCZ


def csite(lx, ly, lz):
    assert 0 <= lx < CSX and 0 <= ly < CSY and 0 <= lz < CSZ
    return lz * CSPLANE + ly * CSROW + ((CSHALF + (lx >> 1)) if (lx & 1) else (lx >> 1))


def ctile_origin(d, b, shift):
    nx, ny, nz = d
    ntx, nty = nx // CTX, ny // CTY
    q = b // ntx
    return ((b - q * ntx) * CTX + shift * (CTX // 2), (q % nty) * CTY + shift * (CTY // 2),
            (q // nty) * CTZ + shift * (CTZ // 2))


def cb_index(d, x, y, z):
    nx, ny, nz = d
    hx, hy = nx // 2, ny // 2
    colour = (x & 1) + 2 * (y & 1) + 4 * (z & 1)
    return colour * (nx * ny * nz // 8) + (x >> 1) + hx * ((y >> 1) + hy * (z >> 1))


def cprolong_site(cb, ux, uy, uz, c0x, c0y, c0z):
    ax0, ay0, az0 = (ux >> 1) - c0x, (uy >> 1) - c0y, (uz >> 1) - c0z
    ax1, ay1, az1 = ax0 + (ux & 1), ay0 + (uy & 1), az0 + (uz & 1)
    for a, n in ((ax0, CCX), (ax1, CCX), (ay0, CCY), (ay1, CCY), (az0, CCZ), (az1, CCZ)):
        assert 0 <= a < n
    wx1, wy1, wz1 = [0.5 if (q & 1) else 0.0 for q in (ux, uy, uz)]
    wx0, wy0, wz0 = 1 - wx1, 1 - wy1, 1 - wz1
    r = lambda ay, az: (ay + CCY * az) * CCX
    out = []
    for c in range(3):
        u = cb[:, c]
        out.append(wz0 * (wy0 * (wx0 * u[r(ay0, az0) + ax0] + wx1 * u[r(ay0, az0) + ax1]) +
                          wy1 * (wx0 * u[r(ay1, az0) + ax0] + wx1 * u[r(ay1, az0) + ax1])) +
                   wz1 * (wy0 * (wx0 * u[r(ay0, az1) + ax0] + wx1 * u[r(ay0, az1) + ax1]) +
                          wy1 * (wx0 * u[r(ay1, az1) + ax0] + wx1 * u[r(ay1, az1) + ax1])))
    return out


def emulate_csweep(d, dc, st, u_in, uc, f, start, shift, reverse):
    """k_ctile_sweep<start> over all coarse tiles of tiling `shift`."""
    nx, ny, nz = d
    nv = nx * ny * nz
    out = np.full(3 * nv, np.nan)
    written = np.zeros(nv, dtype=int)
    pos = [csite(lx, ly, lz) for lz in range(CSZ) for ly in range(CSY) for lx in range(CSX)]
    assert len(set(pos)) == len(pos) and max(pos) < CSSITES
    for b in range((nx // CTX) * (ny // CTY) * (nz // CTZ)):
        x0, y0, z0 = ctile_origin(d, b, shift)
        c0x, c0y, c0z = x0 // 2 - 1, y0 // 2 - 1, z0 // 2 - 1
        cb = np.zeros((CCSITES, 4))
        if start == 2:
            cnx, cny, cnz = dc
            nvc = cnx * cny * cnz
            for q in range(CCSITES):
                ax, ay, az = q % CCX, (q // CCX) % CCY, q // (CCX * CCY)
                g = gidx(dc, wrapm(c0x + ax, cnx), wrapm(c0y + ay, cny), wrapm(c0z + az, cnz))
                cb[q] = [uc[g], uc[nvc + g], uc[2 * nvc + g], 0.0]
        sm = Smem(CSSITES)
        for q in range(CSX * CSY * CSZ):
            lx, ly, lz = q % CSX, (q // CSX) % CSY, q // (CSX * CSY)
            ux, uy, uz = x0 - 1 + lx, y0 - 1 + ly, z0 - 1 + lz
            v = [0.0, 0.0, 0.0, 0.0]
            if start >= 1:
                g = gidx(d, wrapm(ux, nx), wrapm(uy, ny), wrapm(uz, nz))
                v = [u_in[c * nv + g] for c in range(3)] + [0.0]
                if start == 2:
                    p = cprolong_site(cb, ux, uy, uz, c0x, c0y, c0z)
                    v = [v[c] + p[c] for c in range(3)] + [0.0]
            sm.wr(csite(lx, ly, lz), v, -1)
        sm.writes, sm.reads = {}, {}
        order = list(range(8))[::-1] if reverse else list(range(8))
        for col in order:
            cx, cy, cz = col & 1, (col >> 1) & 1, col >> 2
            oL, oR = (-CSHALF, -CSHALF + 1) if cx == 0 else (CSHALF - 1, CSHALF)
            for t in range(CTHREADS):
                i, j, k = t & 7, (t >> 3) & 3, t >> 5
                lx, ly, lz = 1 + 2 * i + cx, 1 + 2 * j + cy, 1 + 2 * k + cz
                X, Y, Z = wrapm(x0 + lx - 1, nx), wrapm(y0 + ly - 1, ny), wrapm(z0 + lz - 1, nz)
                v = gidx(d, X, Y, Z)
                sb = cb_index(d, X, Y, Z)
                assert 0 <= sb < nv
                s = [st[o * nv + sb] for o in range(27)]
                acc = [f[c * nv + v] for c in range(3)]
                base = csite(lx, ly, lz)
                for o in range(27):
                    if o == 13:
                        continue
                    ox, oy, oz = o % 3 - 1, (o // 3) % 3 - 1, o // 9 - 1
                    off = (oL if ox < 0 else (oR if ox > 0 else 0)) + oy * CSROW + oz * CSPLANE
                    assert base + off == csite(lx + ox, ly + oy, lz + oz)
                    n = sm.rd(base + off, t)
                    for c in range(3):
                        acc[c] -= s[o] * n[c]
                sm.wr(base, [acc[c] / s[13] for c in range(3)] + [0.0], t)
            sm.check_pass()
        for q in range(CTX * CTY * CTZ):
            lx, ly, lz = 1 + q % CTX, 1 + (q // CTX) % CTY, 1 + q // (CTX * CTY)
            g = gidx(d, wrapm(x0 + lx - 1, nx), wrapm(y0 + ly - 1, ny), wrapm(z0 + lz - 1, nz))
            written[g] += 1
            o = sm.v[csite(lx, ly, lz)]
            for c in range(3):
                out[c * nv + g] = o[c]
    assert (written == 1).all()
    return out


def block_gs_stencil(d, st, u0, f, order, shift):
    """Colour Gauss-Seidel with 27-point stencils per 16 x 8 x 8 block of tiling `shift`, halo frozen."""
    nx, ny, nz = d
    nv = nx * ny * nz
    sx, sy, sz = shift * CTX // 2, shift * CTY // 2, shift * CTZ // 2
    out = u0.copy()
    for z0 in range(sz, nz + sz, CTZ):
        for y0 in range(sy, ny + sy, CTY):
            for x0 in range(sx, nx + sx, CTX):
                loc = u0.copy()
                for col in order:
                    cx, cy, cz = col & 1, (col >> 1) & 1, col >> 2
                    for z in range(z0 + cz, z0 + CTZ, 2):
                        for y in range(y0 + cy, y0 + CTY, 2):
                            for x in range(x0 + cx, x0 + CTX, 2):
                                X, Y, Z = x % nx, y % ny, z % nz
                                v, sb = gidx(d, X, Y, Z), cb_index(d, X, Y, Z)
                                for c in range(3):
                                    s = f[c * nv + v]
                                    for o in range(27):
                                        if o == 13:
                                            continue
                                        ox, oy, oz = o % 3 - 1, (o // 3) % 3 - 1, o // 9 - 1
                                        inside = (x0 <= x + ox < x0 + CTX and y0 <= y + oy < y0 + CTY
                                                  and z0 <= z + oz < z0 + CTZ)
                                        src = loc if inside else u0
                                        s -= st[o * nv + sb] * src[c * nv + gidx(d, (x + ox) % nx, (y + oy) % ny,
                                                                                   (z + oz) % nz)]
                                    loc[c * nv + v] = s / st[13 * nv + sb]
                for z in range(z0, z0 + CTZ):
                    for y in range(y0, y0 + CTY):
                        for x in range(x0, x0 + CTX):
                            v = gidx(d, x % nx, y % ny, z % nz)
                            for c in range(3):
                                out[c * nv + v] = loc[c * nv + v]
    return out


@pytest.fixture(scope="module")
def cfields():
    rng = np.random.default_rng(11)
    d, dc = (32, 16, 16), (16, 8, 8)
    nv, nvc = 32 * 16 * 16, 16 * 8 * 8
    st = rng.random(27 * nv) - 0.5
    st[13 * nv:14 * nv] = 20.0 + rng.random(nv)  # a dominant diagonal
    f = rng.standard_normal(3 * nv)
    u_in = rng.standard_normal(3 * nv)
    uc = rng.standard_normal(3 * nvc)
    return d, dc, st, f, u_in, uc


def test_coarse_sweep_from_zero_tiling0(cfields):
    d, dc, st, f, u_in, uc = cfields
    got = emulate_csweep(d, dc, st, None, None, f, start=0, shift=0, reverse=False)
    ref = block_gs_stencil(d, st, np.zeros_like(f), f, list(range(8)), 0)
    assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()


def test_coarse_sweep_with_prolongation_reverse_shifted(cfields):
    d, dc, st, f, u_in, uc = cfields
    got = emulate_csweep(d, dc, st, u_in, uc, f, start=2, shift=1, reverse=True)
    ref = block_gs_stencil(d, st, u_in + prolong(d, dc, uc), f, list(range(8))[::-1], 1)
    assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()
