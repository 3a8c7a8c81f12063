"""PyHarm-style Python interface over libcharm.so.

Mirrors the names, argument meaning and error behaviour of CHarm's PyHarm
modules for the point path (wrap/pyharm/shs.py:27-190, sha.py:36-103,
crd.py, shc.py): ``Shc``, ``PointGridGL``, ``PointGridDH1``,
``PointGridDH2``, ``PointGrid``, ``PointSctr``, ``shs_point``,
``shs_point_grad1``, ``shs_point_grad2``, ``shs_point_guru`` and
``sha_point``; for block means in cells ``CellGrid``, ``CellSctr``,
``shs_cell`` and ``sha_cell`` (wrap/pyharm/crd.py cell classes, shs.py
shs_cell, sha.py sha_cell).  Arrays are numpy float64 and stay owned by Python; the C
structures point into them.  Errors reported through charm_err raise
CHarmError.
"""
import ctypes as ct

import numpy as np

from ._lib import _libcharm, _Cell, _Err, _Point, _Shc

SCATTERED, GRID, GRID_GL, GRID_DH1, GRID_DH2 = 1, 2, 3, 4, 5
CELL_GRID, CELL_SCATTERED = -2, -1
SHA_CELL_AQ = 0
MU = 1.0
R = 1.0


class CHarmError(Exception):
    pass


def _dptr(a):
    return a.ctypes.data_as(ct.POINTER(ct.c_double))


class _ErrGuard:
    """charm_err_init / handler / free around one call (wrap/pyharm/_err.py)."""

    def __enter__(self):
        self.err = _libcharm.charm_err_init()
        if not self.err:
            raise MemoryError("charm_err_init failed")
        return self.err

    def __exit__(self, *exc):
        try:
            if exc[0] is None and not _libcharm.charm_err_isempty(self.err):
                e = self.err.contents
                msg = ct.string_at(e.msg).decode(errors="replace")
                code = e.code
                raise CHarmError("CHarm error %d: %s" % (code, msg))
        finally:
            _libcharm.charm_err_free(self.err)
        return False


# ---------------------------------------------------------------------------
# Coefficients (wrap/pyharm/shc.py)
# ---------------------------------------------------------------------------
class Shc:
    """Spherical harmonic coefficients of degree nmax, scaling mu and
    reference radius r.  c, s are order-major triangles (C_nm at
    m (2 nmax + 3 - m) / 2 + n - m)."""

    def __init__(self, nmax, mu, r, c=None, s=None):
        self.nmax = int(nmax)
        T = (self.nmax + 1) * (self.nmax + 2) // 2
        self.c = np.zeros(T) if c is None else np.ascontiguousarray(c, np.float64)
        self.s = np.zeros(T) if s is None else np.ascontiguousarray(s, np.float64)
        if self.c.size != T or self.s.size != T:
            raise ValueError("coefficient arrays must hold %d values" % T)
        self._Shc = _libcharm.charm_shc_init(self.nmax, float(mu), float(r),
                                             _dptr(self.c), _dptr(self.s))
        if not self._Shc:
            raise CHarmError("charm_shc_init failed (is r positive?)")

    @classmethod
    def from_zeros(cls, nmax, mu=MU, r=R):
        return cls(nmax, mu, r)

    @classmethod
    def from_garbage(cls, nmax, mu=MU, r=R):
        T = (int(nmax) + 1) * (int(nmax) + 2) // 2
        return cls(nmax, mu, r, np.empty(T), np.empty(T))

    @property
    def mu(self):
        return self._Shc.contents.mu

    @property
    def r(self):
        return self._Shc.contents.r

    def idx(self, n, m):
        return m * (2 * self.nmax + 3 - m) // 2 + n - m

    def __del__(self):
        if getattr(self, "_Shc", None):
            _libcharm.charm_shc_free(self._Shc)
            self._Shc = None


# ---------------------------------------------------------------------------
# Points (wrap/pyharm/crd.py)
# ---------------------------------------------------------------------------
class _PointBase:
    def _from_struct(self, ptr):
        if not ptr:
            raise CHarmError("point construction failed")
        self._Point = ptr
        p = ptr.contents
        self.type = p.type
        nlat, nlon = p.nlat, p.nlon
        self.lat = np.ctypeslib.as_array(p.lat, shape=(nlat,)) if nlat else np.zeros(0)
        self.lon = np.ctypeslib.as_array(p.lon, shape=(nlon,)) if nlon else np.zeros(0)
        self.r = np.ctypeslib.as_array(p.r, shape=(nlat,)) if nlat else np.zeros(0)
        if p.w:
            self.w = np.ctypeslib.as_array(p.w, shape=(nlat,))

    def _from_arrays(self, ptype, lat, lon, r):
        self.lat = np.ascontiguousarray(lat, np.float64)
        self.lon = np.ascontiguousarray(lon, np.float64)
        self.r = np.ascontiguousarray(r, np.float64)
        self.type = ptype
        ptr = _libcharm.charm_crd_point_init(ptype, self.lat.size,
                                             self.lon.size, _dptr(self.lat),
                                             _dptr(self.lon), _dptr(self.r))
        if not ptr:
            raise CHarmError("charm_crd_point_init failed")
        self._Point = ptr

    @property
    def npoint(self):
        return self._Point.contents.npoint

    def __del__(self):
        if getattr(self, "_Point", None):
            _libcharm.charm_crd_point_free(self._Point)
            self._Point = None


class PointGridGL(_PointBase):
    """Gauss--Legendre grid for degree nmax on the sphere of radius r."""

    def __init__(self, nmax, r=R):
        self.nmax = int(nmax)
        self._from_struct(_libcharm.charm_crd_point_gl(self.nmax, float(r)))


class PointGridDH1(_PointBase):
    def __init__(self, nmax, r=R):
        self.nmax = int(nmax)
        self._from_struct(_libcharm.charm_crd_point_dh1(self.nmax, float(r)))


class PointGridDH2(_PointBase):
    def __init__(self, nmax, r=R):
        self.nmax = int(nmax)
        self._from_struct(_libcharm.charm_crd_point_dh2(self.nmax, float(r)))


class PointGrid(_PointBase):
    """User-defined grid of latitudes x longitudes (radii per latitude)."""

    def __init__(self, lat, lon, r, ptype=GRID):
        self._from_arrays(ptype, lat, lon, r)


class PointSctr(_PointBase):
    """Scattered points (lat[i], lon[i], r[i])."""

    def __init__(self, lat, lon, r):
        self._from_arrays(SCATTERED, lat, lon, r)


def _out_shape(pnt):
    if pnt.type == SCATTERED:
        return (pnt.lat.size,)
    return (pnt.lat.size, pnt.lon.size)


# ---------------------------------------------------------------------------
# Synthesis and analysis (wrap/pyharm/shs.py, sha.py)
# ---------------------------------------------------------------------------
def shs_point(pnt, shcs, nmax):
    f = np.zeros(_out_shape(pnt))
    with _ErrGuard() as err:
        _libcharm.charm_shs_point(pnt._Point, shcs._Shc, int(nmax), _dptr(f),
                                  err)
    return f


def _shs_gradn(fn, npar, pnt, shcs, nmax):
    bufs = [np.zeros(_out_shape(pnt)) for _ in range(npar)]
    arr = (ct.POINTER(ct.c_double) * npar)(*[_dptr(b) for b in bufs])
    with _ErrGuard() as err:
        fn(pnt._Point, shcs._Shc, int(nmax), arr, err)
    # CHarm reorders the pointer array (shs_point_gradn.c:133-165); follow it
    addr = {b.ctypes.data: b for b in bufs}
    return [addr[ct.cast(arr[i], ct.c_void_p).value] for i in range(npar)]


def shs_point_grad1(pnt, shcs, nmax):
    return _shs_gradn(_libcharm.charm_shs_point_grad1, 3, pnt, shcs, nmax)


def shs_point_grad2(pnt, shcs, nmax):
    return _shs_gradn(_libcharm.charm_shs_point_grad2, 6, pnt, shcs, nmax)


def shs_point_guru(pnt, shcs, nmax, dr, dlat, dlon):
    f = np.zeros(_out_shape(pnt))
    with _ErrGuard() as err:
        _libcharm.charm_shs_point_guru(pnt._Point, shcs._Shc, int(nmax),
                                       int(dr), int(dlat), int(dlon),
                                       _dptr(f), err)
    return f


def sha_point(pnt, f, nmax, mu=MU, r=R):
    shcs = Shc(nmax, mu, r)
    f = np.ascontiguousarray(f, np.float64)
    with _ErrGuard() as err:
        _libcharm.charm_sha_point(pnt._Point, _dptr(f), int(nmax), shcs._Shc,
                                  err)
    return shcs


# ---------------------------------------------------------------------------
# Cells (wrap/pyharm/crd.py CellGrid / CellSctr, shs.py shs_cell, sha.py
# sha_cell)
# ---------------------------------------------------------------------------
class _CellBase:
    def _from_arrays(self, ctype, latmin, latmax, lonmin, lonmax, r):
        self.type = ctype
        self.latmin = np.ascontiguousarray(latmin, np.float64)
        self.latmax = np.ascontiguousarray(latmax, np.float64)
        self.lonmin = np.ascontiguousarray(lonmin, np.float64)
        self.lonmax = np.ascontiguousarray(lonmax, np.float64)
        self.r = np.ascontiguousarray(r, np.float64)
        ptr = _libcharm.charm_crd_cell_init(
            ctype, self.latmin.size, self.lonmin.size, _dptr(self.latmin),
            _dptr(self.latmax), _dptr(self.lonmin), _dptr(self.lonmax),
            _dptr(self.r))
        if not ptr:
            raise CHarmError("charm_crd_cell_init failed")
        self._Cell = ptr

    @property
    def ncell(self):
        return self._Cell.contents.ncell

    def __del__(self):
        if getattr(self, "_Cell", None):
            _libcharm.charm_crd_cell_free(self._Cell)
            self._Cell = None


class CellGrid(_CellBase):
    """Grid of cells: latitude bands [latmin[i], latmax[i]] at radius r[i]
    times longitude bands [lonmin[j], lonmax[j]]."""

    def __init__(self, latmin, latmax, lonmin, lonmax, r):
        self._from_arrays(CELL_GRID, latmin, latmax, lonmin, lonmax, r)


class CellSctr(_CellBase):
    """Scattered cells: cell i is [latmin[i], latmax[i]] x [lonmin[i],
    lonmax[i]] at radius r[i]."""

    def __init__(self, latmin, latmax, lonmin, lonmax, r):
        self._from_arrays(CELL_SCATTERED, latmin, latmax, lonmin, lonmax, r)


def shs_cell(cell, shcs, nmax):
    if cell.type == CELL_SCATTERED:
        f = np.zeros(cell.latmin.size)
    else:
        f = np.zeros((cell.latmin.size, cell.lonmin.size))
    with _ErrGuard() as err:
        _libcharm.charm_shs_cell(cell._Cell, shcs._Shc, int(nmax), _dptr(f),
                                 err)
    return f


def sha_cell(cell, f, nmax, method=SHA_CELL_AQ, mu=MU, r=R):
    shcs = Shc(nmax, mu, r)
    f = np.ascontiguousarray(f, np.float64)
    with _ErrGuard() as err:
        _libcharm.charm_sha_cell(cell._Cell, _dptr(f), int(nmax), int(method),
                                 shcs._Shc, err)
    return shcs


# ---------------------------------------------------------------------------
# Global spectral gravity forward modelling (wrap/pyharm/gfm.py
# global_density_3d, global_density_lateral, global_density_const)
# ---------------------------------------------------------------------------
def _enc(x):
    return None if x is None else str(x).encode()


def gfm_global_density_3d(shape_shcs, shape_nmax, shape_radius_ref,
                          density_shcs, density_nmax, density_order,
                          grav_const, mass, shape_power_min, shape_power_max,
                          potential_shcs_nmax, shape_density_shcs_path=None,
                          potential_shcs_path=None, shcs_file_format="bin"):
    pot = Shc(potential_shcs_nmax, 1.0, 1.0)
    n = int(density_order) + 1
    arr = (ct.POINTER(_Shc) * n)(*[d._Shc for d in density_shcs[:n]])
    nm = (ct.c_ulong * n)(*[int(x) for x in density_nmax[:n]])
    with _ErrGuard() as err:
        _libcharm.charm_gfm_global_density_3d(
            shape_shcs._Shc, int(shape_nmax), float(shape_radius_ref), arr,
            nm, int(density_order), float(grav_const), float(mass),
            int(shape_power_min), int(shape_power_max),
            int(potential_shcs_nmax), _enc(shape_density_shcs_path),
            _enc(potential_shcs_path), _enc(shcs_file_format), pot._Shc, err)
    return pot


def gfm_global_density_lateral(shape_shcs, shape_nmax, shape_radius_ref,
                               density_shcs, density_nmax, grav_const, mass,
                               shape_power_min, shape_power_max,
                               potential_shcs_nmax,
                               shape_density_shcs_path=None,
                               potential_shcs_path=None,
                               shcs_file_format="bin"):
    pot = Shc(potential_shcs_nmax, 1.0, 1.0)
    with _ErrGuard() as err:
        _libcharm.charm_gfm_global_density_lateral(
            shape_shcs._Shc, int(shape_nmax), float(shape_radius_ref),
            density_shcs._Shc, int(density_nmax), float(grav_const),
            float(mass), int(shape_power_min), int(shape_power_max),
            int(potential_shcs_nmax), _enc(shape_density_shcs_path),
            _enc(potential_shcs_path), _enc(shcs_file_format), pot._Shc, err)
    return pot


def gfm_global_density_const(shape_shcs, shape_nmax, shape_radius_ref,
                             density, grav_const, mass, shape_power_min,
                             shape_power_max, potential_shcs_nmax,
                             shape_shcs_path=None, potential_shcs_path=None,
                             shcs_file_format="bin"):
    pot = Shc(potential_shcs_nmax, 1.0, 1.0)
    with _ErrGuard() as err:
        _libcharm.charm_gfm_global_density_const(
            shape_shcs._Shc, int(shape_nmax), float(shape_radius_ref),
            float(density), float(grav_const), float(mass),
            int(shape_power_min), int(shape_power_max),
            int(potential_shcs_nmax), _enc(shape_shcs_path),
            _enc(potential_shcs_path), _enc(shcs_file_format), pot._Shc, err)
    return pot
