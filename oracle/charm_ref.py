"""ORACLE -- TEST INFRASTRUCTURE ONLY.

ctypes access to CHarm 0.4.9 itself, built from its own sources by
oracle/build_ref.py into oracle/_ref/ (double with AVX-512 or AVX2, float,
and quad).  Only tests/, the smoke check and bench.py's CPU legs use it, as
the checker and as the timed reference CPU implementation; nothing in the
charm_b200 package imports it.

The structures mirror CHarm's public, non-MPI layouts (src/crd/crd.h.in
`charm_point`, src/shc/shc.h.in `charm_shc`, src/err/err.h.in `charm_err`),
the same ones PyHarm hard-codes (wrap/pyharm/crd.py:48-56, shc.py:68-75,
_err.py:29-35).  Quad-precision arrays cross the boundary as binary128
buffers filled from / read into double-double pairs by the oracle's
orc_q_from_dd / orc_q_to_dd (liborc_q.so).
"""
import ctypes as ct
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, "_ref")

GL, DH1, DH2 = 3, 4, 5
GRID, SCATTERED = 2, 1

_libs = {}


def cpu_has_avx512():
    """True when the host CPU reports the AVX-512 F and DQ extensions that
    the AVX-512 build of CHarm is compiled for."""
    try:
        flags = set()
        for line in open("/proc/cpuinfo"):
            if line.startswith("flags"):
                flags.update(line.split(":", 1)[1].split())
                break
        return {"avx512f", "avx512dq"} <= flags
    except OSError:
        return False


def lib_path(prec="d"):
    if prec == "d":
        name = "libcharm_d_avx512.so" if cpu_has_avx512() else "libcharm_d_avx2.so"
    elif prec == "q":
        name = "libcharmq.so"
    elif prec == "f":
        name = "libcharmf.so"
    else:
        raise ValueError(prec)
    return os.path.join(REF, name)


def available(prec="d"):
    return os.path.exists(lib_path(prec))


class _F128(ct.Structure):
    """The 16 bytes of one IEEE binary128 value.  ctypes cannot pass
    __float128 by value (it travels in SSE registers), so the quad build is
    only called through pointers: its coefficient structure is filled in
    here, the way charmq_shc_init fills it (src/shc/shc_init_chunk.c)."""
    _fields_ = [("b", ct.c_ubyte * 16)]


def _structs(flt):
    class Err(ct.Structure):
        _fields_ = [("level", ct.c_size_t),
                    ("file", ct.POINTER(ct.POINTER(ct.c_char))),
                    ("line", ct.POINTER(ct.c_size_t)),
                    ("func", ct.POINTER(ct.POINTER(ct.c_char))),
                    ("code", ct.c_int),
                    ("msg", ct.POINTER(ct.c_char)),
                    ("saturated", ct.c_bool),
                    ("distributed", ct.c_bool)]

    class Point(ct.Structure):
        _fields_ = [("type", ct.c_int), ("nlat", ct.c_size_t),
                    ("nlon", ct.c_size_t), ("npoint", ct.c_size_t),
                    ("lat", ct.POINTER(flt)), ("lon", ct.POINTER(flt)),
                    ("r", ct.POINTER(flt)), ("w", ct.POINTER(flt)),
                    ("owner", ct.c_bool), ("distributed", ct.c_bool)]

    # __float128 members are 16-byte aligned; _F128 is a byte array, so
    # the quad layout spells out the padding before `mu`
    pad = [("_pad", ct.c_ubyte * 8)] if flt is _F128 else []

    class Shc(ct.Structure):
        _fields_ = [("nmax", ct.c_ulong)] + pad + [
                    ("mu", flt), ("r", flt),
                    ("nc", ct.c_size_t), ("ns", ct.c_size_t),
                    ("c", ct.POINTER(ct.POINTER(flt))),
                    ("s", ct.POINTER(ct.POINTER(flt))),
                    ("owner", ct.c_bool), ("distributed", ct.c_bool)]

    class Cell(ct.Structure):
        _fields_ = [("type", ct.c_int), ("nlat", ct.c_size_t),
                    ("nlon", ct.c_size_t), ("ncell", ct.c_size_t),
                    ("latmin", ct.POINTER(flt)), ("latmax", ct.POINTER(flt)),
                    ("lonmin", ct.POINTER(flt)), ("lonmax", ct.POINTER(flt)),
                    ("r", ct.POINTER(flt)), ("owner", ct.c_bool)]
    return Err, Point, Shc, Cell


class Charm:
    """One CHarm build: prefix '' (double), 'f' (float) or 'q' (quad)."""

    def __init__(self, prec="d"):
        path = lib_path(prec)
        if not os.path.exists(path):
            raise FileNotFoundError(
                "%s is missing; build it with `python oracle/build_ref.py "
                "--reference <CHarm source tree>`" % path)
        self.prec = prec
        self.path = path
        self.L = ct.CDLL(path)
        pre = {"d": "charm_", "f": "charmf_", "q": "charmq_"}[prec]
        self.pre = pre
        flt = {"d": ct.c_double, "f": ct.c_float, "q": _F128}[prec]
        self.flt = flt
        self.Err, self.Point, self.Shc, self.Cell = _structs(flt)
        P, UL, SZ = ct.POINTER, ct.c_ulong, ct.c_size_t
        sig = {
            "err_init": ([], P(self.Err)),
            "err_reset": ([P(self.Err)], None),
            "err_free": ([P(self.Err)], None),
            "err_isempty": ([P(self.Err)], ct.c_bool),
            "crd_point_init": ([ct.c_int, SZ, SZ, P(flt), P(flt), P(flt)],
                               P(self.Point)),
            "crd_point_free": ([P(self.Point)], None),
            "shc_free": ([P(self.Shc)], None),
            "shs_point": ([P(self.Point), P(self.Shc), UL, P(flt),
                           P(self.Err)], None),
            "shs_point_grad1": ([P(self.Point), P(self.Shc), UL, P(P(flt)),
                                 P(self.Err)], None),
            "shs_point_grad2": ([P(self.Point), P(self.Shc), UL, P(P(flt)),
                                 P(self.Err)], None),
            "shs_point_guru": ([P(self.Point), P(self.Shc), UL, ct.c_uint,
                                ct.c_uint, ct.c_uint, P(flt), P(self.Err)],
                               None),
            "sha_point": ([P(self.Point), P(flt), UL, P(self.Shc),
                           P(self.Err)], None),
            "crd_cell_init": ([ct.c_int, SZ, SZ, P(flt), P(flt), P(flt),
                               P(flt), P(flt)], P(self.Cell)),
            "crd_cell_free": ([P(self.Cell)], None),
            "shs_cell": ([P(self.Cell), P(self.Shc), UL, P(flt),
                          P(self.Err)], None),
            "sha_cell": ([P(self.Cell), P(flt), UL, ct.c_int, P(self.Shc),
                          P(self.Err)], None),
        }
        if prec != "q":
            sig["shc_init"] = ([UL, flt, flt, P(flt), P(flt)], P(self.Shc))
            sig["crd_point_gl"] = ([UL, flt], P(self.Point))
            sig["crd_point_dh1"] = ([UL, flt], P(self.Point))
            sig["crd_point_dh2"] = ([UL, flt], P(self.Point))
        for name, (args, res) in sig.items():
            fn = getattr(self.L, pre + name)
            fn.argtypes = args
            fn.restype = res
        # CHarm's error handler prints to stderr; check() raises instead
        self.err = self.fn("err_init")()

    def fn(self, name):
        return getattr(self.L, self.pre + name)

    def check(self):
        if not self.fn("err_isempty")(self.err):
            msg = ct.string_at(self.err.contents.msg).decode(errors="replace")
            raise RuntimeError("CHarm (%s): %s" % (self.path, msg))

    # -- double / float ------------------------------------------------
    def _np(self):
        return np.float64 if self.prec == "d" else np.float32

    def _ptr(self, a):
        return a.ctypes.data_as(ct.POINTER(self.flt))

    def grid(self, kind, nmax, r):
        """CHarm's own GL / DH1 / DH2 grid; returns (point, lat, lon, w) with
        numpy views of the point's arrays (valid while `point` lives;
        point.ptr.contents is the charm_point itself)."""
        name = {GL: "crd_point_gl", DH1: "crd_point_dh1", DH2: "crd_point_dh2"}[kind]
        p = self.fn(name)(nmax, r)
        if not p:
            raise RuntimeError("CHarm %s(%d) failed" % (name, nmax))
        pt = p.contents
        lat = np.ctypeslib.as_array(pt.lat, (pt.nlat,))
        lon = np.ctypeslib.as_array(pt.lon, (pt.nlon,))
        w = np.ctypeslib.as_array(pt.w, (pt.nlat,))
        return _Owned(p, (), self.fn("crd_point_free")), lat, lon, w

    def point(self, kind, lat, lon, r):
        """charm_crd_point_init over caller arrays (kept alive on the
        returned object)."""
        t = self._np()
        lat = np.ascontiguousarray(lat, t)
        lon = np.ascontiguousarray(lon, t)
        r = np.ascontiguousarray(r, t)
        p = self.fn("crd_point_init")(kind, lat.size, lon.size, self._ptr(lat),
                                      self._ptr(lon), self._ptr(r))
        if not p:
            raise RuntimeError("CHarm crd_point_init failed")
        return _Owned(p, (lat, lon, r), self.fn("crd_point_free"))

    def shc(self, nmax, mu, r, c, s):
        t = self._np()
        c = np.ascontiguousarray(c, t)
        s = np.ascontiguousarray(s, t)
        h = self.fn("shc_init")(nmax, mu, r, self._ptr(c), self._ptr(s))
        if not h:
            raise RuntimeError("CHarm shc_init failed")
        return _Owned(h, (c, s), self.fn("shc_free"))

    def shs_point(self, pnt, shcs, nmax, npoint):
        f = np.empty(npoint, self._np())
        self.fn("shs_point")(_p(pnt), _p(shcs), nmax, self._ptr(f), self.err)
        self.check()
        return f

    def shs_point_grad(self, pnt, shcs, nmax, npoint, order):
        npar = 3 if order == 1 else 6
        fs = [np.empty(npoint, self._np()) for _ in range(npar)]
        arr = (ct.POINTER(self.flt) * npar)(*[self._ptr(x) for x in fs])
        self.fn("shs_point_grad%d" % order)(_p(pnt), _p(shcs), nmax, arr,
                                            self.err)
        self.check()
        # CHarm reorders the caller's pointers (src/shs/shs_point_gradn.c:
        # 133-165): component i is where arr[i] points after the call
        by_addr = {x.ctypes.data: x for x in fs}
        return [by_addr[ct.cast(arr[i], ct.c_void_p).value] for i in range(npar)]

    def shs_point_guru(self, pnt, shcs, nmax, npoint, dr, dlat, dlon):
        f = np.empty(npoint, self._np())
        self.fn("shs_point_guru")(_p(pnt), _p(shcs), nmax, dr, dlat, dlon,
                                  self._ptr(f), self.err)
        self.check()
        return f

    def sha_point(self, pnt, f, nmax, mu, r):
        """Analysis into a fresh triangle of degree nmax; returns (c, s)."""
        T = (nmax + 1) * (nmax + 2) // 2
        c = np.zeros(T, self._np())
        s = np.zeros(T, self._np())
        out = self.shc(nmax, mu, r, c, s)
        f = np.ascontiguousarray(f, self._np())
        self.fn("sha_point")(_p(pnt), self._ptr(f), nmax, out.ptr, self.err)
        self.check()
        return out.keep[0].copy(), out.keep[1].copy()

    def cell(self, ctype, latmin, latmax, lonmin, lonmax, r):
        """charm_crd_cell_init over caller arrays (kept alive on the
        returned object)."""
        t = self._np()
        arrs = [np.ascontiguousarray(a, t) for a in
                (latmin, latmax, lonmin, lonmax, r)]
        c = self.fn("crd_cell_init")(ctype, arrs[0].size, arrs[2].size,
                                     *[self._ptr(a) for a in arrs])
        if not c:
            raise RuntimeError("CHarm crd_cell_init failed")
        return _Owned(c, tuple(arrs), self.fn("crd_cell_free"))

    def shs_cell(self, cell, shcs, nmax, ncell):
        f = np.empty(ncell, self._np())
        self.fn("shs_cell")(_p(cell), _p(shcs), nmax, self._ptr(f), self.err)
        self.check()
        return f

    def sha_cell(self, cell, f, nmax, mu, r):
        """Approximate-quadrature analysis (CHARM_SHA_CELL_AQ) into a fresh
        triangle of degree nmax; returns (c, s)."""
        T = (nmax + 1) * (nmax + 2) // 2
        out = self.shc(nmax, mu, r, np.zeros(T), np.zeros(T))
        f = np.ascontiguousarray(f, self._np())
        self.fn("sha_cell")(_p(cell), self._ptr(f), nmax, 0, out.ptr,
                            self.err)
        self.check()
        return out.keep[0].copy(), out.keep[1].copy()


def _p(x):
    return x.ptr if isinstance(x, (_Owned, _Held)) else x


class _Held:
    """A structure built here: nothing to free in CHarm."""
    def __init__(self, ptr, keep):
        self.ptr = ptr
        self.keep = keep


class _Owned:
    def __init__(self, ptr, keep, free):
        self.ptr = ptr
        self.keep = keep
        self._free = free

    def __del__(self):
        try:
            self._free(self.ptr)
        except Exception:
            pass


# -- quad ------------------------------------------------------------------
class CharmQ(Charm):
    """CHarm's quad build.  Values go in and come out as double-double
    (hi, lo) pairs, converted by the oracle's liborc_q.so."""

    def __init__(self):
        super().__init__("q")
        from oracle import orc
        self.Q = orc.lib("q")
        for name in ("orc_q_from_dd", "orc_q_to_dd"):
            getattr(self.Q, name).argtypes = [ct.c_void_p] * 3 + [ct.c_size_t]
            getattr(self.Q, name).restype = None

    def qbuf(self, hi, lo=None):
        hi = np.ascontiguousarray(hi, np.float64).ravel()
        lo = np.zeros_like(hi) if lo is None else np.ascontiguousarray(lo, np.float64).ravel()
        buf = (_F128 * max(hi.size, 1))()
        self.Q.orc_q_from_dd(hi.ctypes.data, lo.ctypes.data, ct.addressof(buf),
                             hi.size)
        return buf

    def to_dd(self, buf, n):
        hi = np.empty(n)
        lo = np.empty(n)
        self.Q.orc_q_to_dd(ct.addressof(buf), hi.ctypes.data, lo.ctypes.data, n)
        return hi, lo

    def scalar(self, x_hi, x_lo=0.0):
        return self.qbuf(np.array([x_hi]), np.array([x_lo]))[0]

    def point(self, kind, lat, lon, r, lat_lo=None, lon_lo=None, r_lo=None):
        qlat = self.qbuf(lat, lat_lo)
        qlon = self.qbuf(lon, lon_lo)
        qr = self.qbuf(r, r_lo)
        F = ct.POINTER(_F128)
        p = self.fn("crd_point_init")(kind, len(np.ravel(lat)), len(np.ravel(lon)),
                                      ct.cast(qlat, F), ct.cast(qlon, F),
                                      ct.cast(qr, F))
        if not p:
            raise RuntimeError("CHarm quad crd_point_init failed")
        return _Owned(p, (qlat, qlon, qr), self.fn("crd_point_free"))

    def point_raw(self, kind, latq, lonq, rq):
        """charmq_crd_point_init over binary128 arrays given as the oracle's
        raw (n, 2) float64 buffers (oracle.orc.q_from_dd / q_arith), for
        coordinates that must be exact in binary128, e.g. longitudes
        j pi / L that CHarm checks for a linear increase within its quad
        threshold."""
        keep = [np.ascontiguousarray(a) for a in (latq, lonq, rq)]
        F = ct.POINTER(_F128)
        p = self.fn("crd_point_init")(kind, keep[0].shape[0], keep[1].shape[0],
                                      ct.cast(keep[0].ctypes.data, F),
                                      ct.cast(keep[1].ctypes.data, F),
                                      ct.cast(keep[2].ctypes.data, F))
        if not p:
            raise RuntimeError("CHarm quad crd_point_init failed")
        return _Owned(p, tuple(keep), self.fn("crd_point_free"))

    def shc(self, nmax, mu, r, c, s, c_lo=None, s_lo=None):
        """A charmq_shc over binary128 copies of (c, s), with the column
        pointers c[m] = base + m (2 nmax + 3 - m) / 2 that charmq_shc_init
        sets (src/shc/shc_init_chunk.c:135-147)."""
        qc = self.qbuf(c, c_lo)
        qs = self.qbuf(s, s_lo)
        F = ct.POINTER(_F128)
        cp = (F * (nmax + 1))()
        sp = (F * (nmax + 1))()
        base_c, base_s = ct.addressof(qc), ct.addressof(qs)
        for m in range(nmax + 1):
            off = 16 * (m * (2 * nmax + 3 - m) // 2)
            cp[m] = ct.cast(base_c + off, F)
            sp[m] = ct.cast(base_s + off, F)
        h = self.Shc()
        h.nmax = nmax
        h.mu = self.scalar(mu)
        h.r = self.scalar(r)
        h.nc = h.ns = (nmax + 1) * (nmax + 2) // 2
        h.c = ct.cast(cp, ct.POINTER(F))
        h.s = ct.cast(sp, ct.POINTER(F))
        h.owner = False
        h.distributed = False
        return _Held(ct.pointer(h), (qc, qs, cp, sp, h))

    def shs_point(self, pnt, shcs, nmax, npoint):
        """Returns the synthesis as (hi, lo) double-double arrays."""
        f = (_F128 * npoint)()
        self.fn("shs_point")(_p(pnt), _p(shcs), nmax,
                             ct.cast(f, ct.POINTER(_F128)), self.err)
        self.check()
        return self.to_dd(f, npoint)
