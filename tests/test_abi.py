"""The C ABI without a GPU: libcharm.so loads, exports every symbol that
include/charm_b200.h declares, its struct layouts are CHarm's (the layouts
PyHarm hard-codes), and argument errors are reported through charm_err
exactly as CHarm reports them, before any device work."""
import ctypes as ct
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "charm_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    funcs = re.findall(r"CHARM_EXTERN[^;(]*?\b(charmf?_\w+)\s*\(", text)
    data = re.findall(r"CHARM_EXTERN\s+extern\s+[\w ]+?\b(charmf?_\w+)\s*;",
                      text)
    return sorted(set(funcs)), sorted(set(data))


def test_exports_everything_declared():
    from charm_b200 import LIB_PATH
    lib = ct.CDLL(LIB_PATH)
    funcs, data = declared_symbols()
    assert len(funcs) >= 24
    glob = {"glob_threshold", "glob_threshold2",
            "glob_polar_optimization_a1", "glob_polar_optimization_a2"}
    assert set(data) == {p + g for p in ("charm_", "charmf_") for g in glob}
    # the float build's entry points (CHarm src/prec.h:84-86, @P@ = f)
    for name in ("shs_point", "shs_point_grad1", "shs_point_grad2",
                 "shs_point_guru", "sha_point", "shc_init", "shc_malloc",
                 "shc_calloc", "shc_free", "crd_point_gl", "crd_point_dh1",
                 "crd_point_dh2", "crd_point_init", "crd_point_free",
                 "err_init", "err_free", "err_isempty"):
        assert "charmf_" + name in funcs, name
    for name in funcs + data:
        assert hasattr(lib, name), name


def test_globals_default_values():
    from charm_b200._lib import _libcharm
    eps = np.finfo(np.float64).eps
    assert ct.c_double.in_dll(_libcharm, "charm_glob_threshold").value == 100 * eps
    assert ct.c_double.in_dll(_libcharm, "charm_glob_threshold2").value == 1e5 * eps
    assert ct.c_ulong.in_dll(_libcharm,
                             "charm_glob_polar_optimization_a1").value == 100
    assert ct.c_double.in_dll(_libcharm,
                              "charm_glob_polar_optimization_a2").value == -1.0


def test_float_globals_and_layouts():
    """charmf_glob_* hold the float build's defaults (src/glob/glob.c with
    EPS = FLT_EPSILON), and charmf_point / charmf_shc have CHarm's float
    layouts (RDT = float)."""
    from charm_b200._lib import _libcharm
    feps = np.finfo(np.float32).eps
    assert ct.c_float.in_dll(_libcharm, "charmf_glob_threshold").value == \
        np.float32(100 * feps)
    assert ct.c_float.in_dll(_libcharm, "charmf_glob_threshold2").value == \
        np.float32(1e5 * feps)

    class PointF(ct.Structure):
        _fields_ = [("type", ct.c_int), ("nlat", ct.c_size_t),
                    ("nlon", ct.c_size_t), ("npoint", ct.c_size_t),
                    ("lat", ct.POINTER(ct.c_float)),
                    ("lon", ct.POINTER(ct.c_float)),
                    ("r", ct.POINTER(ct.c_float)),
                    ("w", ct.POINTER(ct.c_float)),
                    ("owner", ct.c_bool), ("distributed", ct.c_bool)]

    class ShcF(ct.Structure):
        _fields_ = [("nmax", ct.c_ulong), ("mu", ct.c_float),
                    ("r", ct.c_float), ("nc", ct.c_size_t),
                    ("ns", ct.c_size_t),
                    ("c", ct.POINTER(ct.POINTER(ct.c_float))),
                    ("s", ct.POINTER(ct.POINTER(ct.c_float))),
                    ("owner", ct.c_bool), ("distributed", ct.c_bool)]
    L = _libcharm
    L.charmf_shc_calloc.restype = ct.POINTER(ShcF)
    L.charmf_shc_calloc.argtypes = [ct.c_ulong, ct.c_float, ct.c_float]
    L.charmf_shc_free.argtypes = [ct.POINTER(ShcF)]
    h = L.charmf_shc_calloc(10, 3.5, 2.0)
    assert h.contents.nmax == 10 and h.contents.mu == 3.5 and \
        h.contents.r == 2.0 and h.contents.nc == 66 and h.contents.owner
    # column m starts m (2 nmax + 3 - m) / 2 floats into the triangle
    base = ct.cast(h.contents.c[0], ct.c_void_p).value
    assert ct.cast(h.contents.c[3], ct.c_void_p).value - base == 4 * 30
    L.charmf_shc_free(h)
    L.charmf_crd_point_calloc.restype = ct.POINTER(PointF)
    L.charmf_crd_point_calloc.argtypes = [ct.c_int, ct.c_size_t, ct.c_size_t]
    L.charmf_crd_point_free.argtypes = [ct.POINTER(PointF)]
    p = L.charmf_crd_point_calloc(3, 5, 12)     # GL type: weights too
    assert p.contents.npoint == 60 and bool(p.contents.w)
    L.charmf_crd_point_free(p)


def test_struct_layouts():
    """Field offsets of charm_point / charm_shc / charm_err match the
    non-MPI CHarm layout mirrored by PyHarm (crd.py:48-56, shc.py:68-75,
    _err.py:29-35)."""
    from charm_b200._lib import _Err, _Point, _Shc
    assert [f[0] for f in _Point._fields_][:9] == [
        "type", "nlat", "nlon", "npoint", "lat", "lon", "r", "w", "owner"]
    assert _Point.owner.offset == 64 and _Point.lat.offset == 32
    assert _Shc.c.offset == 40 and _Shc.owner.offset == 56
    assert _Err.code.offset == 32 and _Err.saturated.offset == 48


def test_shc_and_point_constructors():
    import charm_b200 as cb
    from charm_b200._lib import _libcharm
    h = _libcharm.charm_shc_calloc(5, 2.0, 3.0)
    assert h and h.contents.nmax == 5 and h.contents.nc == 21
    # columns point into one contiguous block (shc_init_chunk.c:126-145)
    base = ct.cast(h.contents.c[0], ct.c_void_p).value
    for m in range(6):
        col = ct.cast(h.contents.c[m], ct.c_void_p).value
        assert col == base + 8 * sum(6 - k for k in range(m))
    _libcharm.charm_shc_free(h)
    assert not _libcharm.charm_shc_calloc(5, 1.0, -1.0)      # r must be > 0
    p = _libcharm.charm_crd_point_calloc(cb.SCATTERED, 3, 3)
    assert p and p.contents.npoint == 3 and p.contents.owner
    _libcharm.charm_crd_point_free(p)
    assert not _libcharm.charm_crd_point_calloc(cb.SCATTERED, 3, 4)
    q = _libcharm.charm_crd_point_calloc(cb.GRID_GL, 3, 6)
    assert q and q.contents.npoint == 18 and q.contents.w
    _libcharm.charm_crd_point_free(q)
    nlat, nlon = ct.c_size_t(), ct.c_size_t()
    _libcharm.charm_crd_point_dh2_shape(10, ct.byref(nlat), ct.byref(nlon))
    assert (nlat.value, nlon.value) == (22, 44)


def test_argument_errors_without_gpu():
    import charm_b200 as cb
    shc = cb.Shc(4, 1.0, 1.0)
    p = cb.PointSctr([0.1, 0.2], [0.3, 0.4], [1.0, 1.0])
    with pytest.raises(cb.CHarmError, match="cannot be larger"):
        cb.shs_point(p, shc, 5)
    with pytest.raises(cb.CHarmError, match="dr \\+ dlat \\+ dlon"):
        cb.shs_point_guru(p, shc, 4, 2, 1, 0)
    with pytest.raises(cb.CHarmError, match="Unsupported"):
        cb.sha_point(p, np.zeros(2), 2)
    # zero points is a valid no-op (shs_point.c:79-80)
    z = cb.PointSctr(np.zeros(0), np.zeros(0), np.zeros(0))
    assert cb.shs_point(z, shc, 4).size == 0


def test_cell_constructors_and_errors_without_gpu():
    """charm_cell layout and constructors (src/crd/crd.h.in:339-409,
    crd_cell_alloc.c, crd_cell_init.c) and the argument checks that
    charm_shs_cell / charm_sha_cell make before any GPU work
    (src/shs/shs_cell.c:22-121, src/sha/sha_cell.c:37-100)."""
    import charm_b200 as cb
    from charm_b200._lib import _Cell, _libcharm
    assert _Cell.latmin.offset == 32 and _Cell.r.offset == 64
    assert _Cell.owner.offset == 72
    c = _libcharm.charm_crd_cell_calloc(cb.CELL_GRID, 3, 5)
    assert c and c.contents.ncell == 15 and c.contents.owner
    _libcharm.charm_crd_cell_free(c)
    c = _libcharm.charm_crd_cell_malloc(cb.CELL_SCATTERED, 4, 4)
    assert c and c.contents.ncell == 4
    _libcharm.charm_crd_cell_free(c)
    assert not _libcharm.charm_crd_cell_calloc(cb.CELL_SCATTERED, 3, 4)
    assert not _libcharm.charm_crd_cell_calloc(cb.GRID, 3, 4)
    shc = cb.Shc(4, 1.0, 1.0)
    cg = cb.CellGrid([0.1], [0.2], [0.0], [1.0], [1.0])
    with pytest.raises(cb.CHarmError, match="cannot be larger"):
        cb.shs_cell(cg, shc, 5)
    with pytest.raises(cb.CHarmError, match="Unsupported .method."):
        cb.sha_cell(cg, np.zeros(1), 2, method=7)
    cs = cb.CellSctr([0.1], [0.2], [0.0], [1.0], [1.0])
    with pytest.raises(cb.CHarmError, match="Unsupported .cell->type."):
        cb.sha_cell(cs, np.zeros(1), 2)
    # zero cells are a valid no-op (shs_cell.c:63-64)
    z = cb.CellSctr(np.zeros(0), np.zeros(0), np.zeros(0), np.zeros(0),
                    np.zeros(0))
    assert cb.shs_cell(z, shc, 4).size == 0


def test_err_object_lifecycle():
    from charm_b200._lib import _libcharm
    e = _libcharm.charm_err_init()
    assert e and _libcharm.charm_err_isempty(e)
    assert e.contents.level == 0 and e.contents.code == 0
    _libcharm.charm_err_reset(e)
    _libcharm.charm_err_handler(e, False)       # empty: no-op
    _libcharm.charm_err_free(e)
