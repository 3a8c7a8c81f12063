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
    funcs = re.findall(r"CHARM_EXTERN[^;(]*?\b(charm_\w+)\s*\(", text)
    data = re.findall(r"CHARM_EXTERN\s+extern\s+[\w ]+?\b(charm_\w+)\s*;", text)
    return sorted(set(funcs)), sorted(set(data))


def test_exports_everything_declared():
    from charm_b200 import LIB_PATH
    lib = ct.CDLL(LIB_PATH)
    funcs, data = declared_symbols()
    assert len(funcs) >= 24
    assert set(data) == {"charm_glob_threshold", "charm_glob_threshold2",
                         "charm_glob_polar_optimization_a1",
                         "charm_glob_polar_optimization_a2"}
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


def test_err_object_lifecycle():
    from charm_b200._lib import _libcharm
    e = _libcharm.charm_err_init()
    assert e and _libcharm.charm_err_isempty(e)
    assert e.contents.level == 0 and e.contents.code == 0
    _libcharm.charm_err_reset(e)
    _libcharm.charm_err_handler(e, False)       # empty: no-op
    _libcharm.charm_err_free(e)
