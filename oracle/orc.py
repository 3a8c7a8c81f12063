"""ORACLE driver -- TEST INFRASTRUCTURE ONLY.

Python side of the CPU oracle: the drivers of CHarm's point synthesis and
analysis restated around the C kernels in orc.c (liborc_d.so, liborc_q.so).
Only tests/, the smoke check and the CPU-baseline leg of bench.py import this
module; the product path never does.

Restated reference drivers (CHarm 0.4.9):
  shs_point        src/shs/shs_point.c:26-129, shs_point_grd.c:97-1076,
                   shs_point_sctr.c:86-728, shs_point_gradn.c:32-165
  sha_point        src/sha/sha_point.c:124-1125
  shs_cell         src/shs/shs_cell.c:22-121, shs_cell_grd.c:42-884,
                   shs_cell_sctr.c, shs_grd_fft_lc.c:73-118, shs_grd_lr.c:68-99
  sha_cell         src/sha/sha_cell.c:37-1487
  gl, dh1, dh2     src/crd/crd_point_gl_chunk.c, crd_point_dh_chunk.c
The longitude sums use numpy's FFT (the role FFTW plays in CHarm) on grids
where CHarm uses FFT, and direct sums elsewhere.
"""
import ctypes as ct
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

SCATTERED, GRID, GL, DH1, DH2 = 1, 2, 3, 4, 5
EPS = np.finfo(np.float64).eps
THRESHOLD = 100.0 * EPS          # src/glob/glob.c:16
THRESHOLD2 = 100000.0 * EPS      # src/glob/glob.c:17
PI = 3.14159265358979323846
PI_2 = 1.57079632679489661923

_libs = {}


def build():
    """Compiles liborc_d.so and liborc_q.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib(prec="d"):
    if prec not in _libs:
        path = os.path.join(HERE, "liborc_%s.so" % prec)
        if not os.path.exists(path):
            build()
        L = ct.CDLL(path)
        p = ct.c_void_p
        ul, sz, i = ct.c_ulong, ct.c_size_t, ct.c_int
        fn = getattr(L, "orc_%s_shs_lumped" % prec)
        fn.argtypes = [ul, ul, p, p, sz, p, p, p, p, i, i, i, i, p, p, p, p]
        fn.restype = None
        fn = getattr(L, "orc_%s_sha_contract" % prec)
        fn.argtypes = [ul, sz, p, p, p, p, p, p, p]
        fn.restype = None
        fn = getattr(L, "orc_%s_cell_lumped" % prec)
        fn.argtypes = [ul, ul, p, p, sz, p, p, p, p, p, ct.c_double, p, p,
                       p, p]
        fn.restype = None
        fn = getattr(L, "orc_%s_cell_contract" % prec)
        fn.argtypes = [ul, sz, p, p, p, p, p, p, ct.c_double, p, p]
        fn.restype = None
        fn = getattr(L, "orc_%s_gl" % prec)
        fn.argtypes = [ul, p, p]
        fn.restype = i
        fn = getattr(L, "orc_%s_dh" % prec)
        fn.argtypes = [ul, p, p]
        fn.restype = None
        if prec == "q":
            L.orc_q_from_dd.argtypes = [p, p, p, sz]
            L.orc_q_to_dd.argtypes = [p, p, p, sz]
            L.orc_q_lonsum.argtypes = [sz, sz, p, p, sz, p, p, p]
            L.orc_q_sin.argtypes = [p, p, sz]
            L.orc_q_cos.argtypes = [p, p, sz]
            L.orc_q_arith.argtypes = [i, p, p, p, sz, i]
            L.orc_q_from_double.argtypes = [p, p, sz]
            # the real-valued scalar argument of lonsum is passed by pointer
            # through a one-element buffer; see lonsum() below
        _libs[prec] = L
    return _libs[prec]


def _ptr(a):
    return a.ctypes.data_as(ct.c_void_p)


def nearly_equal(a, b, eps):
    """src/misc/misc_is_nearly_equal.c:20-31"""
    aa, ba, d = abs(a), abs(b), abs(a - b)
    if a == b:
        return True
    if a == 0.0 or b == 0.0:
        return d <= eps
    if aa + ba == aa or aa + ba == ba:
        return d <= eps
    return d / max(aa, ba) <= eps


def arr_chck_symm(arr, center, eps):
    """src/misc/misc_arr_chck_symm.c; 0 if symmetric."""
    size = len(arr)
    middle = size // 2
    for i in range(middle):
        if not nearly_equal(arr[i] - center, center - arr[size - 1 - i], eps):
            return 1
    if size % 2 == 1 and not nearly_equal(center, arr[middle], eps):
        return 2
    return 0


# ---------------------------------------------------------------------------
# Data containers mirroring charm_shc / charm_point (src/shc/shc.h.in:139-381,
# src/crd/crd.h.in:125-332)
# ---------------------------------------------------------------------------
class Shc:
    """Coefficient triangle, order-major: c[m][n - m] at col0[m] + n - m."""

    def __init__(self, nmax, mu, r, c=None, s=None):
        self.nmax = int(nmax)
        self.mu = float(mu)
        self.r = float(r)
        T = (self.nmax + 1) * (self.nmax + 2) // 2
        self.c = np.zeros(T) if c is None else np.ascontiguousarray(c, np.float64)
        self.s = np.zeros(T) if s is None else np.ascontiguousarray(s, np.float64)

    def idx(self, n, m):
        return tri_index(self.nmax, n, m)


def tri_col0(nmax):
    m = np.arange(nmax + 1)
    return (m * (2 * nmax + 3 - m)) // 2


def tri_index(nmax, n, m):
    return m * (2 * nmax + 3 - m) // 2 + n - m


class Point:
    def __init__(self, ptype, lat, lon, r, w=None):
        self.type = ptype
        self.lat = np.ascontiguousarray(lat, np.float64)
        self.lon = np.ascontiguousarray(lon, np.float64)
        self.r = np.ascontiguousarray(r, np.float64)
        self.w = None if w is None else np.ascontiguousarray(w, np.float64)

    @property
    def nlat(self):
        return len(self.lat)

    @property
    def nlon(self):
        return len(self.lon)

    @property
    def npoint(self):
        if self.type == SCATTERED:
            return self.nlat
        return self.nlat * self.nlon


# ---------------------------------------------------------------------------
# Grids (src/crd)
# ---------------------------------------------------------------------------
def gl_shape(nmax):
    return nmax + 1, 2 * (nmax + 1)


def dh1_shape(nmax):
    return 2 * (nmax + 1), 2 * (nmax + 1)


def dh2_shape(nmax):
    return 2 * (nmax + 1), 4 * (nmax + 1)


def gl(nmax, r, prec="d"):
    """crd_point_gl (src/crd/crd_point_gl_chunk.c:122-190)."""
    nlat, nlon = gl_shape(nmax)
    if prec == "q":
        lat = np.zeros((nlat, 2))
        w = np.zeros((nlat, 2))
        if lib("q").orc_q_gl(nmax, _ptr(lat), _ptr(w)):
            raise RuntimeError("GL iterations did not converge")
        return lat, w
    lat = np.zeros(nlat)
    w = np.zeros(nlat)
    if lib("d").orc_d_gl(nmax, _ptr(lat), _ptr(w)):
        raise RuntimeError("GL iterations did not converge")
    c = PI / float(nmax + 1)
    lon = c * np.arange(nlon, dtype=np.float64)
    return Point(GL, lat, lon, np.full(nlat, float(r)), w)


def dh(nmax, r, kind, prec="d"):
    """crd_point_dh1/dh2 (src/crd/crd_point_dh_chunk.c, *_lat_w_chunk.c)."""
    nlat, nlon = dh1_shape(nmax) if kind == DH1 else dh2_shape(nmax)
    if prec == "q":
        lat = np.zeros((nlat, 2))
        w = np.zeros((nlat, 2))
        lib("q").orc_q_dh(nmax, _ptr(lat), _ptr(w))
        return lat, w
    lat = np.zeros(nlat)
    w = np.zeros(nlat)
    lib("d").orc_d_dh(nmax, _ptr(lat), _ptr(w))
    L = nmax + 1
    c = PI / float(L) if kind == DH1 else PI / float(2 * L)
    lon = c * np.arange(nlon, dtype=np.float64)
    return Point(kind, lat, lon, np.full(nlat, float(r)), w)


def generate_point(ptype, nlat, nlon, r, lat_rng, lon_rng):
    """tests/generate_point.c: the custom grids and scattered points used by
    CHarm's synthesis tests."""
    nlat2 = nlat - 1 if (ptype == GRID and nlat > 1) else nlat
    lat = np.array([PI_2 - (float(l) / float(nlat2)) * lat_rng
                    for l in range(nlat)])
    lon = np.array([(float(l) / float(nlon)) * lon_rng for l in range(nlon)])
    return Point(ptype, lat, lon, np.full(nlat, float(r)))


# ---------------------------------------------------------------------------
# Synthesis
# ---------------------------------------------------------------------------
def mode_of(kind):
    """kind: "pot", "grad1", "grad2" or (dr, dlat, dlon).
    Returns kgrad, dr, dlat, dlon, dorder, npar (shs_get_mur_dorder_npar.c)."""
    if kind == "pot":
        return 0, 0, 0, 0, 0, 1
    if kind == "grad1":
        return 1, 1, 1, 1, 1, 3
    if kind == "grad2":
        return 2, 2, 2, 2, 2, 6
    dr, dlat, dlon = kind
    if min(dr, dlat, dlon) < 0 or dr + dlat + dlon > 2:
        raise ValueError("dr + dlat + dlon must be in [0, 2]")
    return 0, dr, dlat, dlon, dr + dlat + dlon, 1


def mur_of(shc, dorder):
    rpow = shc.r
    for _ in range(dorder):
        rpow *= shc.r
    return shc.mu / rpow


def reorder(kgrad, f):
    """Output pointer reordering, src/shs/shs_point_gradn.c:133-165."""
    if kgrad == 1:
        return [f[2], f[0], f[1]]
    if kgrad == 2:
        return [f[5], f[2], f[4], f[0], f[1], f[3]]
    return f


def grid_rows(pnt):
    """Evaluated rows, mirror rows and symmetry flags of a grid, restating
    shs_point_grd.c:113-197 and crd_grd_check_symm.c:21-72."""
    nlat = pnt.nlat
    is_dh = pnt.type in (DH1, DH2)
    is_quad = pnt.type in (GL, DH1, DH2)
    pnt_nlat = nlat + 1 if is_dh else nlat
    even = (pnt_nlat % 2) == 0
    if pnt_nlat == 1:
        symm = False
    elif is_quad:
        symm = True
    else:
        symm = arr_chck_symm(pnt.lat, 0.0, THRESHOLD2) == 0
    if is_quad:
        nmax_grd = nlat - 1 if pnt.type == GL else (nlat - 2) // 2
        if pnt.type == GL and nmax_grd % 2:
            equator = None
        else:
            equator = nlat // 2
    nlatdo = (pnt_nlat + 1 - int(even)) // 2 if symm else pnt_nlat
    rows, mirrors, flags = [], [], []
    for ipv in range(nlatdo):
        if is_quad:
            if is_dh and ipv == 0:
                s = 0
            elif equator is None or ipv < equator:
                s = 1
            else:
                s = 0
        else:
            if not symm:
                s = 0
            elif (not even) and ipv == nlatdo - 1:
                s = 0
            else:
                s = 1
        rows.append(ipv)
        mirrors.append(pnt_nlat - ipv - 1 if s else -1)
        flags.append(s)
    return np.array(rows), np.array(mirrors), np.array(flags, dtype=np.int32)


def fft_applicable(pnt, nmax):
    """shs_grd_point_fft_check.c:30-55 (after the linear-step check)."""
    nlon = pnt.nlon
    if nlon < 1:
        return False
    dlon = pnt.lon[1] - pnt.lon[0] if nlon > 1 else 0.0
    return ((nlon - 1) // 2 >= nmax
            and nearly_equal(pnt.lon[0], 0.0, THRESHOLD)
            and nearly_equal(pnt.lon[-1] + dlon, 2.0 * PI, THRESHOLD))


def lumped(shc, nmax, lat, rr, rr2, symm, kind):
    kgrad, dr, dlat, dlon, dorder, npar = mode_of(kind)
    nrow = len(lat)
    L = nmax + 1
    out = [np.zeros((npar, nrow, L)) for _ in range(4)]
    lib("d").orc_d_shs_lumped(
        nmax, shc.nmax, _ptr(shc.c), _ptr(shc.s), nrow,
        _ptr(np.ascontiguousarray(lat, np.float64)),
        _ptr(np.ascontiguousarray(rr, np.float64)),
        _ptr(np.ascontiguousarray(rr2, np.float64)),
        _ptr(np.ascontiguousarray(symm, np.int32)),
        kgrad, dr, dlat, dlon, *[_ptr(o) for o in out])
    return out


def lon_synthesis_fft(a, b, nlon, mur):
    """Inverse real DFT along the parallels as CHarm packs it for FFTW
    (shs_grd_fft_lc.c:54-175, shs_grd_fft.c:23-136)."""
    L = a.shape[-1]
    nfc = nlon // 2 + 1
    fc = np.zeros(a.shape[:-1] + (nfc,), dtype=np.complex128)
    c = np.full(L, 0.5)
    c[0] = 1.0
    fc[..., :L] = (a * c) - 1j * (b * c)
    return mur * (np.fft.irfft(fc, n=nlon, axis=-1) * nlon)


def lon_synthesis_direct(a, b, lon, mur):
    """Sum over orders at arbitrary longitudes (shs_grd_lr.c, PSLR)."""
    L = a.shape[-1]
    ml = np.outer(np.arange(L, dtype=np.float64), lon)
    return mur * (a @ np.cos(ml) + b @ np.sin(ml))


def shs_point(pnt, shc, nmax, kind="pot"):
    """Synthesis; returns the list of output components in CHarm's final
    order (one for "pot" and single derivatives, 3 for grad1, 6 for grad2)."""
    if nmax > shc.nmax:
        raise ValueError("nmax > shcs->nmax")
    kgrad, dr, dlat, dlon, dorder, npar = mode_of(kind)
    mur = mur_of(shc, dorder)
    if pnt.npoint == 0:
        return [np.zeros(0) for _ in range(npar)]
    r_eq = all(nearly_equal(x, shc.r, THRESHOLD) for x in pnt.r)
    if pnt.type == SCATTERED:
        if pnt.nlat != pnt.nlon:
            raise ValueError("nlat != nlon for scattered points")
        rr = np.ones(pnt.nlat) if r_eq else shc.r / pnt.r
        a, b, _, _ = lumped(shc, nmax, pnt.lat, rr, rr,
                            np.zeros(pnt.nlat, np.int32), kind)
        # shs_point_sctr.c:599-641: cos/sin of m * lon in working precision
        out = []
        mvec = np.arange(nmax + 1, dtype=np.float64)
        for p in range(npar):
            ml = mvec[None, :] * pnt.lon[:, None]
            fp = np.sum(a[p] * np.cos(ml) + b[p] * np.sin(ml), axis=1)
            out.append(mur * fp)
        return reorder(kgrad, out)

    rows, mirrors, flags = grid_rows(pnt)
    nlat, nlon = pnt.nlat, pnt.nlon
    lat = pnt.lat[rows]
    if r_eq:
        rr = np.ones(len(rows))
        rr2 = np.ones(len(rows))
    else:
        rr = shc.r / pnt.r[rows]
        rr2 = np.array([shc.r / pnt.r[mm] if mm >= 0 else 1.0
                        for mm in mirrors])
    a, b, a2, b2 = lumped(shc, nmax, lat, rr, rr2, flags, kind)
    use_fft = fft_applicable(pnt, nmax)
    out = []
    for p in range(npar):
        f = np.zeros((nlat, nlon))
        if use_fft:
            fn = lon_synthesis_fft(a[p], b[p], nlon, mur)
            fs = lon_synthesis_fft(a2[p], b2[p], nlon, mur)
        else:
            fn = lon_synthesis_direct(a[p], b[p], pnt.lon, mur)
            fs = lon_synthesis_direct(a2[p], b2[p], pnt.lon, mur)
        for k, (i, mi) in enumerate(zip(rows, mirrors)):
            if i < nlat:
                f[i] = fn[k]
            if mi >= 0 and mi < nlat:
                f[mi] = fs[k]
        out.append(f.reshape(-1))
    return reorder(kgrad, out)


# ---------------------------------------------------------------------------
# Analysis
# ---------------------------------------------------------------------------
def sha_point(pnt, f, nmax, mu, r, shc_nmax=None):
    """charm_sha_point restated (src/sha/sha_point.c:124-1125); returns an
    Shc of degree shc_nmax (default nmax)."""
    if pnt.type not in (GL, DH1, DH2):
        raise ValueError("unsupported point type for analysis")
    shc_nmax = nmax if shc_nmax is None else shc_nmax
    out = Shc(shc_nmax, mu, r)
    if nmax > shc_nmax:
        raise ValueError("nmax > shcs->nmax")
    r0 = pnt.r[0]
    for x in pnt.r[1:]:
        if not nearly_equal(x, r0, THRESHOLD):
            raise ValueError("all radii must be equal")
    nlat, nlon = pnt.nlat, pnt.nlon
    nmax_grd = nlat - 1 if pnt.type == GL else (nlat - 2) // 2
    if nmax > nmax_grd:
        raise ValueError("grid degree too low")
    if pnt.type in (GL, DH1):
        c = PI / float(nmax_grd + 1)
    else:
        c = PI / float(2 * nmax_grd + 2)
    c *= 1.0 / (4.0 * PI) * (r0 / mu)
    rows, mirrors, flags = grid_rows(pnt)
    f2 = np.asarray(f, np.float64).reshape(nlat, nlon)
    F = np.fft.rfft(f2, axis=1)
    L = nmax + 1
    nrow = len(rows)
    a = np.zeros((nrow, L))
    b = np.zeros((nrow, L))
    a2 = np.zeros((nrow, L))
    b2 = np.zeros((nrow, L))
    for k, (i, mi) in enumerate(zip(rows, mirrors)):
        cw = c * pnt.w[i]
        a[k] = cw * F[i, :L].real
        b[k] = -cw * F[i, :L].imag
        if mi >= 0:
            cw2 = c * pnt.w[mi]
            a2[k] = cw2 * F[mi, :L].real
            b2[k] = -cw2 * F[mi, :L].imag
    sy = flags[:, None].astype(np.float64)
    amp = np.ascontiguousarray(a + sy * a2)
    amm = np.ascontiguousarray(a - sy * a2)
    bmp = np.ascontiguousarray(b + sy * b2)
    bmm = np.ascontiguousarray(b - sy * b2)
    T = L * (L + 1) // 2
    cc = np.zeros(T)
    ss = np.zeros(T)
    lib("d").orc_d_sha_contract(nmax, nrow, _ptr(np.ascontiguousarray(
        pnt.lat[rows])), _ptr(amp), _ptr(amm), _ptr(bmp), _ptr(bmm),
        _ptr(cc), _ptr(ss))
    # copy the degree-nmax triangle into the shc_nmax triangle
    col_src = tri_col0(nmax)
    col_dst = tri_col0(shc_nmax)
    for m in range(L):
        out.c[col_dst[m]:col_dst[m] + L - m] = cc[col_src[m]:col_src[m] + L - m]
        out.s[col_dst[m]:col_dst[m] + L - m] = ss[col_src[m]:col_src[m] + L - m]
    if not nearly_equal(r, r0, THRESHOLD):
        # shc_rescale (src/shc/shc_rescale.c) from r0 to r
        r_ratio = r0 / r
        tmp = np.empty(shc_nmax + 1)
        tmp[0] = 1.0
        tmp2 = r_ratio
        for n in range(1, shc_nmax + 1):
            tmp[n] = tmp2
            tmp2 *= r_ratio
        for m in range(shc_nmax + 1):
            sl = slice(col_dst[m], col_dst[m] + shc_nmax + 1 - m)
            out.c[sl] *= tmp[m:]
            out.s[sl] *= tmp[m:]
    return out


# ---------------------------------------------------------------------------
# Quadruple-precision helpers (the binary128 build)
# ---------------------------------------------------------------------------
def q_from_dd(hi, lo=None):
    hi = np.ascontiguousarray(hi, np.float64).reshape(-1)
    lo = np.zeros_like(hi) if lo is None else np.ascontiguousarray(
        lo, np.float64).reshape(-1)
    out = np.zeros((hi.size, 2))
    lib("q").orc_q_from_dd(_ptr(hi), _ptr(lo), _ptr(out), hi.size)
    return out


def q_to_dd(q):
    q = np.ascontiguousarray(q).reshape(-1, 2)
    hi = np.zeros(q.shape[0])
    lo = np.zeros(q.shape[0])
    lib("q").orc_q_to_dd(_ptr(q), _ptr(hi), _ptr(lo), q.shape[0])
    return hi, lo


def q_arith(op, a, b):
    a = np.ascontiguousarray(a).reshape(-1, 2)
    b = np.ascontiguousarray(b).reshape(-1, 2)
    out = np.zeros_like(a)
    ops = {"+": 0, "-": 1, "*": 2, "/": 3}
    lib("q").orc_q_arith(ops[op], _ptr(a), _ptr(b), _ptr(out), a.shape[0],
                         int(b.shape[0] == 1 and a.shape[0] != 1))
    return out


def shs_point_quad_grid(ptype, nmax, shc_nmax, mu_q, r_q, c_q, s_q, rgrid_q,
                        nlon_override=None, lat_shift=None):
    """Potential synthesis on a GL/DH grid entirely in binary128.  Inputs are
    (n, 2) binary128 buffers; returns the grid values as (hi, lo) float64.
    nlon_override / lat_shift restate the "dsun" tests of
    tests/check_shs_point_all.c:767-907 (first meridian only, first latitude
    moved by lat_shift, which breaks the symmetry)."""
    if ptype == GL:
        lat, w = gl(nmax, 0.0, prec="q")
        nlat, nlon = gl_shape(nmax)
        lonc = PI / float(nmax + 1)
    else:
        lat, w = dh(nmax, 0.0, ptype, prec="q")
        nlat, nlon = dh1_shape(nmax) if ptype == DH1 else dh2_shape(nmax)
        lonc = None
    L = nmax + 1
    # longitudes in quad: c * i with c = PI / L (or PI / 2L)
    piq = q_from_dd(np.array([math.pi]), np.array([1.2246467991473532e-16]))
    if ptype == DH2:
        cq = q_arith("/", piq, q_from_dd(np.array([2.0 * L])))
    else:
        cq = q_arith("/", piq, q_from_dd(np.array([float(L)])))
    if nlon_override is not None:
        nlon = nlon_override
    lon = q_arith("*", q_from_dd(np.arange(nlon, dtype=np.float64)), cq)
    if lat_shift is not None:
        # the grid keeps its GL/DH type, so CHarm still pairs the moved first
        # latitude with the last row (shs_point_grd.c:150-163)
        lat = lat.copy()
        lat[0:1] = q_arith("-", lat[0:1], lat_shift)
    hi_lat, _ = q_to_dd(lat)
    pnt = Point(ptype, hi_lat, np.zeros(nlon), np.ones(nlat))
    rows, mirrors, flags = grid_rows(pnt)
    nrow = len(rows)
    latr = np.ascontiguousarray(lat[rows])
    # r == R in all the quad golden cases handled here except dr1 (r = R+1000)
    rr_hi, _ = q_to_dd(rgrid_q)
    R_hi, _ = q_to_dd(r_q)
    if nearly_equal(rr_hi[0], R_hi[0], THRESHOLD):
        rr = q_from_dd(np.ones(nrow))
    else:
        rr = q_arith("/", np.repeat(r_q, nrow, axis=0),
                     np.repeat(rgrid_q, nrow, axis=0))
    rr2 = rr.copy()
    out = [np.zeros((nrow * L, 2)) for _ in range(4)]
    lib("q").orc_q_shs_lumped(nmax, shc_nmax, _ptr(c_q), _ptr(s_q), nrow,
                              _ptr(latr), _ptr(rr), _ptr(rr2),
                              _ptr(np.ascontiguousarray(flags, np.int32)),
                              0, 0, 0, 0, *[_ptr(o) for o in out])
    mur = q_arith("/", mu_q, r_q)
    fn = np.zeros((nrow * nlon, 2))
    fs = np.zeros((nrow * nlon, 2))
    lib("q").orc_q_lonsum(nrow, L, _ptr(out[0]), _ptr(out[1]), nlon,
                          _ptr(lon), _ptr(mur), _ptr(fn))
    lib("q").orc_q_lonsum(nrow, L, _ptr(out[2]), _ptr(out[3]), nlon,
                          _ptr(lon), _ptr(mur), _ptr(fs))
    f = np.zeros((nlat * nlon, 2))
    for k, (i, mi) in enumerate(zip(rows, mirrors)):
        if i < nlat:
            f[i * nlon:(i + 1) * nlon] = fn[k * nlon:(k + 1) * nlon]
        if mi >= 0 and mi < nlat:
            f[mi * nlon:(mi + 1) * nlon] = fs[k * nlon:(k + 1) * nlon]
    return q_to_dd(f)


# ---------------------------------------------------------------------------
# Block-mean values in cells (charm_cell, src/crd/crd.h.in:339-409)
# ---------------------------------------------------------------------------
CELL_GRID, CELL_SCATTERED = -2, -1
SHA_CELL_AQ = 0
POLAR_OFF = -1.0


class Cell:
    def __init__(self, ctype, latmin, latmax, lonmin, lonmax, r):
        self.type = ctype
        self.latmin = np.ascontiguousarray(latmin, np.float64).reshape(-1)
        self.latmax = np.ascontiguousarray(latmax, np.float64).reshape(-1)
        self.lonmin = np.ascontiguousarray(lonmin, np.float64).reshape(-1)
        self.lonmax = np.ascontiguousarray(lonmax, np.float64).reshape(-1)
        self.r = np.ascontiguousarray(r, np.float64).reshape(-1)

    @property
    def nlat(self):
        return self.latmin.size

    @property
    def nlon(self):
        return self.lonmin.size

    @property
    def ncell(self):
        return self.nlat if self.type == CELL_SCATTERED else self.nlat * self.nlon


def generate_cell(ctype, nlat, nlon, r, lat_rng, lon_rng):
    """tests/generate_cell.c:18-56: cells of equal size from the north pole
    down lat_rng and from longitude 0 east lon_rng."""
    l = np.arange(nlat, dtype=np.float64)
    latmin = PI_2 - ((l + 1.0) / float(nlat)) * lat_rng
    latmax = PI_2 - (l / float(nlat)) * lat_rng
    k = np.arange(nlon, dtype=np.float64)
    lonmin = (k / float(nlon)) * lon_rng
    lonmax = ((k + 1.0) / float(nlon)) * lon_rng
    return Cell(ctype, latmin, latmax, lonmin, lonmax, np.full(nlat, r))


def arr_chck_lin_incr(arr, eps):
    """src/misc/misc_arr_chck_lin_incr.c with first = 0, every_nth = 1:
    0 if the array increases with a constant step."""
    n = len(arr)
    if n < 2:
        return 0
    if not nearly_equal(arr[0], float(np.min(arr)), eps):
        return 1
    step = arr[1] - arr[0]
    if step <= 0.0:
        return 1
    for j in range(1, n):
        if not nearly_equal(step, arr[j] - arr[j - 1], eps):
            return 1
    return 0


def cell_check_grd_lons(cell):
    """src/shs/shs_cell_check_grd_lons.c:14-85; returns deltalon."""
    if cell.nlon > 1:
        if arr_chck_lin_incr(cell.lonmin, THRESHOLD2):
            raise ValueError("lonmin is not linearly increasing")
        if arr_chck_lin_incr(cell.lonmax, THRESHOLD2):
            raise ValueError("lonmax is not linearly increasing")
        if not nearly_equal(cell.lonmin[1] - cell.lonmin[0],
                            cell.lonmax[1] - cell.lonmax[0], THRESHOLD2):
            raise ValueError("lonmin and lonmax steps differ")
        return cell.lonmin[1] - cell.lonmin[0]
    return cell.lonmax[0] - cell.lonmin[0]


def crd_check_cells(cell):
    """src/crd/crd_check_cells.c:14-40"""
    if np.any(cell.latmax <= cell.latmin):
        raise ValueError("latmin must be smaller than latmax")
    if np.any(cell.lonmin >= cell.lonmax):
        raise ValueError("lonmin must be smaller than lonmax")


def cell_fft_applicable(cell, nmax):
    """src/shs/shs_grd_cell_fft_check.c:17-60"""
    if cell.nlon <= 1:
        return False
    return ((cell.nlon - 1) // 2 >= nmax
            and nearly_equal(cell.lonmin[0], 0.0, THRESHOLD)
            and nearly_equal(cell.lonmax[-1], 2.0 * PI, THRESHOLD)
            and nearly_equal(cell.lonmin[1], cell.lonmax[0], THRESHOLD))


def cell_grid_rows(cell):
    """Rows, mirrors and symmetry flags of a cell grid:
    shs_cell_grd.c:52-110 with crd_grd_check_symm.c for cell grids."""
    nlat = cell.nlat
    even = nlat % 2 == 0
    symm = nlat > 1
    for i in range(nlat):
        if not nearly_equal(cell.latmin[i], -cell.latmax[nlat - i - 1],
                            THRESHOLD2):
            symm = False
            break
    nlatdo = (nlat + 1 - int(even)) // 2 if symm else nlat
    rows, mirrors, flags = [], [], []
    for ipv in range(nlatdo):
        s = 1 if symm and not ((not even) and ipv == nlatdo - 1) else 0
        rows.append(ipv)
        mirrors.append(nlat - ipv - 1 if s else -1)
        flags.append(s)
    return np.array(rows), np.array(mirrors), np.array(flags, np.int32)


def cell_lumped(shc, nmax, latmin, latmax, rr, rr2, symm, polar_thr=POLAR_OFF,
                prec="d"):
    nrow = len(latmin)
    L = nmax + 1
    out = [np.zeros((nrow, L)) for _ in range(4)]
    getattr(lib(prec), "orc_%s_cell_lumped" % prec)(
        nmax, shc.nmax, _ptr(shc.c), _ptr(shc.s), nrow,
        _ptr(np.ascontiguousarray(latmin, np.float64)),
        _ptr(np.ascontiguousarray(latmax, np.float64)),
        _ptr(np.ascontiguousarray(rr, np.float64)),
        _ptr(np.ascontiguousarray(rr2, np.float64)),
        _ptr(np.ascontiguousarray(symm, np.int32)), float(polar_thr),
        *[_ptr(o) for o in out])
    return out


def cell_lon_factors(nmax, dlon):
    """(sm, cm) of shs_grd_fft_lc.c:79-97: the longitude integrals of one
    cell of width dlon starting at its lonmin."""
    L = nmax + 1
    sm = np.empty(L)
    cm = np.empty(L)
    sm[0], cm[0] = dlon, 0.0
    for m in range(1, L):
        mr = float(m)
        cm[m] = (math.cos(mr * dlon) - 1.0) / mr
        sm[m] = math.sin(mr * dlon) / mr
    return sm, cm


def cell_m2sm2dl(nmax, dlon):
    """(2 / m) sin(dlon / (2 / m)), m2sm2dl of shs_grd_lr.c:76-84 and
    shs_cell_sctr.c (dlon at m = 0)."""
    L = nmax + 1
    out = np.empty(L)
    out[0] = dlon
    for m in range(1, L):
        m2 = 2.0 / float(m)
        out[m] = m2 * math.sin(dlon / m2)
    return out


def shs_cell(cell, shc, nmax, polar_thr=POLAR_OFF):
    """charm_shs_cell restated; returns the block means (ncell,)."""
    if nmax > shc.nmax:
        raise ValueError("nmax > shcs->nmax")
    if cell.ncell == 0:
        return np.zeros(0)
    mur = shc.mu / shc.r
    L = nmax + 1
    if cell.type == CELL_SCATTERED:
        if cell.nlat != cell.nlon:
            raise ValueError("nlat != nlon for scattered cells")
        crd_check_cells(cell)
        n = cell.nlat
        rr = shc.r / cell.r
        a, b, _, _ = cell_lumped(shc, nmax, cell.latmin, cell.latmax, rr,
                                 rr, np.zeros(n, np.int32), polar_thr)
        f = np.zeros(n)
        for i in range(n):
            dl = cell.lonmax[i] - cell.lonmin[i]
            w = cell_m2sm2dl(nmax, dl)
            ml = (np.arange(L, dtype=np.float64) / 2.0) * (cell.lonmin[i] +
                                                          cell.lonmax[i])
            fi = np.sum((a[i] * w) * np.cos(ml) + (b[i] * w) * np.sin(ml))
            dsigma = (math.sin(cell.latmax[i]) - math.sin(cell.latmin[i])) * dl
            f[i] = mur * (fi / dsigma)
        return f
    if cell.type != CELL_GRID:
        raise ValueError("unsupported cell type")
    rows, mirrors, flags = cell_grid_rows(cell)
    dlon = cell_check_grd_lons(cell)
    use_fft = cell_fft_applicable(cell, nmax)
    crd_check_cells(cell)
    rr = shc.r / cell.r[rows]
    rr2 = np.array([shc.r / cell.r[mm] if mm >= 0 else 0.0 for mm in mirrors])
    a, b, a2, b2 = cell_lumped(shc, nmax, cell.latmin[rows],
                               cell.latmax[rows], rr, rr2, flags, polar_thr)
    nlat, nlon = cell.nlat, cell.nlon
    if use_fft:
        sm, cm = cell_lon_factors(nmax, dlon)
        c = np.full(L, 0.5)
        c[0] = 1.0

        def lon_sum(a_, b_):
            nfc = nlon // 2 + 1
            fc = np.zeros((a_.shape[0], nfc), dtype=np.complex128)
            fc[:, :L] = ((a_ * sm - b_ * cm) * c) - 1j * ((a_ * cm + b_ * sm) * c)
            return np.fft.irfft(fc, n=nlon, axis=-1) * nlon
    else:
        w = cell_m2sm2dl(nmax, dlon)
        lon0 = (cell.lonmin[0] + cell.lonmax[0]) / 2.0
        lons = lon0 + np.arange(nlon) * dlon

        def lon_sum(a_, b_):
            return lon_synthesis_direct(a_ * w, b_ * w, lons, 1.0)
    fn = lon_sum(a, b)
    fs = lon_sum(a2, b2)
    f = np.zeros((nlat, nlon))
    for k, (i, mi) in enumerate(zip(rows, mirrors)):
        dsigma = (math.sin(cell.latmax[i]) - math.sin(cell.latmin[i])) * dlon
        cc = mur / dsigma
        f[i] = cc * fn[k]
        if mi >= 0:
            f[mi] = cc * fs[k]
    return f.reshape(-1)


def sha_cell(cell, f, nmax, mu, r, shc_nmax=None, polar_thr=POLAR_OFF):
    """charm_sha_cell with CHARM_SHA_CELL_AQ restated
    (src/sha/sha_cell.c:37-1487); returns an Shc of degree shc_nmax."""
    shc_nmax = nmax if shc_nmax is None else shc_nmax
    out = Shc(shc_nmax, mu, r)
    if cell.type != CELL_GRID:
        raise ValueError("unsupported cell type for analysis")
    if nmax > shc_nmax:
        raise ValueError("nmax > shcs->nmax")
    if cell.ncell == 0:
        return out
    r0 = cell.r[0]
    for x in cell.r[1:]:
        if not nearly_equal(x, r0, THRESHOLD):
            raise ValueError("all radii must be equal")
    nlat, nlon = cell.nlat, cell.nlon
    if not nearly_equal(cell.latmax[0], PI_2, THRESHOLD):
        raise ValueError("latmax[0] must be pi/2")
    if nlat < nmax + 1:
        raise ValueError("not enough latitudes")
    if not nearly_equal(cell.latmin[-1], -PI_2, THRESHOLD):
        raise ValueError("latmin[-1] must be -pi/2")
    for i in range(nlat - 1):
        if not nearly_equal(cell.latmin[i], cell.latmax[i + 1], THRESHOLD):
            raise ValueError("cells not aligned in latitude")
    even = nlat % 2 == 0
    symm = nlat > 1
    for i in range(nlat):
        if not nearly_equal(cell.latmin[i], -cell.latmax[nlat - i - 1],
                            THRESHOLD2):
            symm = False
            break
    if nlon < 2 * nmax + 1:
        raise ValueError("not enough longitudes")
    if not nearly_equal(cell.lonmin[0], 0.0, THRESHOLD):
        raise ValueError("lonmin[0] must be 0")
    if not nearly_equal(cell.lonmax[-1], 2.0 * PI, THRESHOLD):
        raise ValueError("lonmax[-1] must be 2 pi")
    dlon = cell_check_grd_lons(cell)
    if nlon > 1 and not nearly_equal(cell.lonmin[1], cell.lonmax[0],
                                     THRESHOLD):
        raise ValueError("cells not aligned in longitude")
    crd_check_cells(cell)
    nlatdo = ((nlat // 2) if even else (nlat + 1) // 2) if symm else nlat
    rows = np.arange(nlatdo)
    flags = np.array([1 if symm and not ((not even) and i == nlatdo - 1)
                      else 0 for i in rows], np.int32)
    mirrors = np.where(flags == 1, nlat - 1 - rows, -1)
    L = nmax + 1
    F = np.fft.rfft(np.asarray(f, np.float64).reshape(nlat, nlon), axis=1)
    a = F[rows, :L].real
    b = -F[rows, :L].imag
    a2 = np.zeros_like(a)
    b2 = np.zeros_like(b)
    for k, mi in enumerate(mirrors):
        if mi >= 0:
            a2[k] = F[mi, :L].real
            b2[k] = -F[mi, :L].imag
    sy = flags[:, None].astype(np.float64)
    sm, cm = cell_lon_factors(nmax, dlon)
    ap, am_ = a + sy * a2, a - sy * a2
    bp, bm_ = b + sy * b2, b - sy * b2
    amp = np.ascontiguousarray(ap * sm + bp * cm)
    amm = np.ascontiguousarray(am_ * sm + bm_ * cm)
    bmp = np.ascontiguousarray(bp * sm - ap * cm)
    bmm = np.ascontiguousarray(bm_ * sm - am_ * cm)
    # m = 0: (a +- a2) dlon (sha_cell.c:797-803)
    amp[:, 0] = ap[:, 0] * dlon
    amm[:, 0] = am_[:, 0] * dlon
    bmp[:, 0] = 0.0
    bmm[:, 0] = 0.0
    T = L * (L + 1) // 2
    cc = np.zeros(T)
    ss = np.zeros(T)
    lib("d").orc_d_cell_contract(
        nmax, nlatdo, _ptr(np.ascontiguousarray(cell.latmin[rows])),
        _ptr(np.ascontiguousarray(cell.latmax[rows])), _ptr(amp), _ptr(amm),
        _ptr(bmp), _ptr(bmm), float(polar_thr), _ptr(cc), _ptr(ss))
    c2 = 1.0 / (4.0 * PI) * (r0 / mu)
    col_src = tri_col0(nmax)
    col_dst = tri_col0(shc_nmax)
    for m in range(L):
        out.c[col_dst[m]:col_dst[m] + L - m] = c2 * cc[col_src[m]:col_src[m] + L - m]
        out.s[col_dst[m]:col_dst[m] + L - m] = c2 * ss[col_src[m]:col_src[m] + L - m]
    if not nearly_equal(r, r0, THRESHOLD):
        r_ratio = r0 / r
        tmp = np.empty(shc_nmax + 1)
        tmp[0] = 1.0
        tmp2 = r_ratio
        for n in range(1, shc_nmax + 1):
            tmp[n] = tmp2
            tmp2 *= r_ratio
        for m in range(shc_nmax + 1):
            sl = slice(col_dst[m], col_dst[m] + shc_nmax + 1 - m)
            out.c[sl] *= tmp[m:]
            out.s[sl] *= tmp[m:]
    return out


# ---------------------------------------------------------------------------
# Spectral gravity forward modelling, global variant
# (src/gfm/gfm_sgfm.c with SGFM_GLOBAL, gfm_global_density_*.c)
# ---------------------------------------------------------------------------
def global_vnmc(nmax, p, i, c):
    """gfm_sgfm.c global_vnmc: c * binomial-type factor of degree n."""
    out = np.zeros(nmax + 1)
    pr = float(p)
    for n in range(nmax + 1):
        npip3 = float(n + i + 3)
        snpi = npip3 / pr
        for pt in range(1, p):
            snpi *= (npip3 - float(pt)) / (pr - float(pt))
        snpi *= 2.0 / ((2.0 * float(n) + 1.0) * npip3)
        out[n] = c * snpi
    return out


def gfm_global(shape, shape_nmax, R, density, density_nmax, G, mass, pmin,
               pmax, nmax_pot, const_density=None):
    """The potential coefficients of charm_gfm_global_density_3d (density:
    list of Shc, density_nmax: list), _lateral (one density) or _const
    (const_density, density None).  Returns an Shc of degree nmax_pot with
    mu = G mass and r = R."""
    out = Shc(nmax_pot, G * mass, R)
    if const_density is None:
        imax = len(density) - 1
        # get_max_nmax(density_nmax, density_order): the first
        # density_order entries (gfm_sgfm.c)
        dmax = density_nmax[0]
        for k in range(1, imax):
            dmax = max(dmax, density_nmax[k])
    else:
        imax = 0
        dmax = 0
    c = (2.0 * PI * R ** 3) / mass
    if const_density is not None:
        c *= const_density
    col_pot = tri_col0(nmax_pot)
    for p in range(pmin, pmax + 1):
        nmaxp = p * shape_nmax + dmax
        thr = min(nmaxp, nmax_pot)
        g = gl(nmaxp, 1.0)
        fshape = shs_point(g, shape, shape_nmax)[0] - R
        Ri = 1.0
        for i in range(imax + 1):
            s_ij = fshape / R
            sp = s_ij.copy()
            for _ in range(2, p + 1):
                sp = sp * s_ij
            if const_density is None:
                rho = shs_point(g, density[i], density_nmax[i])[0]
                rho = rho * (sp * Ri)
                Ri *= R
            else:
                rho = sp
            a = sha_point(g, rho.reshape(g.nlat, g.nlon), thr, 1.0, 1.0)
            v = global_vnmc(thr, p, i, c)
            col = tri_col0(thr)
            for m in range(thr + 1):
                sl = slice(col[m], col[m] + thr + 1 - m)
                dl = slice(col_pot[m], col_pot[m] + thr + 1 - m)
                out.c[dl] += a.c[sl] * v[m:]
                out.s[dl] += a.s[sl] * v[m:]
    return out


def shc_da(shc, nmax):
    """src/shc/shc_da.c: degree amplitudes sqrt(sum_m C_nm^2 + S_nm^2)."""
    col = tri_col0(shc.nmax)
    out = np.zeros(nmax + 1)
    for n in range(nmax + 1):
        v = 0.0
        for m in range(n + 1):
            i = col[m] + n - m
            v += shc.c[i] * shc.c[i] + shc.s[i] * shc.s[i]
        out[n] = math.sqrt(v)
    return out
