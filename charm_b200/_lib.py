"""Loads libcharm.so (this package's CUDA build of CHarm's point synthesis
and analysis) and mirrors the ctypes layouts PyHarm uses for it
(wrap/pyharm/_err.py:29-35, crd.py:48-56, shc.py:68-75 of CHarm 0.4.9;
the cell layout of src/crd/crd.h.in:339-409).

There is no CPU fallback: if the library is missing, importing fails with
an error that says how to build it.
"""
import ctypes as ct
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcharm.so")

_ct_flt = ct.c_double
_ct_ulong = ct.c_ulong
_ct_size_t = ct.c_size_t
_ct_int = ct.c_int


class _Err(ct.Structure):
    _fields_ = [("level", _ct_size_t),
                ("file", ct.POINTER(ct.POINTER(ct.c_char))),
                ("line", ct.POINTER(_ct_size_t)),
                ("func", ct.POINTER(ct.POINTER(ct.c_char))),
                ("code", _ct_int),
                ("msg", ct.POINTER(ct.c_char)),
                ("saturated", ct.c_bool),
                ("distributed", ct.c_bool)]


class _Point(ct.Structure):
    _fields_ = [("type", _ct_int),
                ("nlat", _ct_size_t),
                ("nlon", _ct_size_t),
                ("npoint", _ct_size_t),
                ("lat", ct.POINTER(_ct_flt)),
                ("lon", ct.POINTER(_ct_flt)),
                ("r", ct.POINTER(_ct_flt)),
                ("w", ct.POINTER(_ct_flt)),
                ("owner", ct.c_bool),
                ("distributed", ct.c_bool)]


class _Shc(ct.Structure):
    _fields_ = [("nmax", _ct_ulong),
                ("mu", _ct_flt),
                ("r", _ct_flt),
                ("nc", _ct_size_t),
                ("ns", _ct_size_t),
                ("c", ct.POINTER(ct.POINTER(_ct_flt))),
                ("s", ct.POINTER(ct.POINTER(_ct_flt))),
                ("owner", ct.c_bool),
                ("distributed", ct.c_bool)]


class _Cell(ct.Structure):
    _fields_ = [("type", _ct_int),
                ("nlat", _ct_size_t),
                ("nlon", _ct_size_t),
                ("ncell", _ct_size_t),
                ("latmin", ct.POINTER(_ct_flt)),
                ("latmax", ct.POINTER(_ct_flt)),
                ("lonmin", ct.POINTER(_ct_flt)),
                ("lonmax", ct.POINTER(_ct_flt)),
                ("r", ct.POINTER(_ct_flt)),
                ("owner", ct.c_bool)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            "charm_b200: %s is missing; build it with "
            "`python charm_b200/build.py` (needs nvcc with sm_100a)" % LIB_PATH)
    lib = ct.CDLL(LIB_PATH)
    P, D, UL, SZ = ct.POINTER, _ct_flt, _ct_ulong, _ct_size_t
    sig = {
        "charm_err_init": ([], P(_Err)),
        "charm_err_free": ([P(_Err)], None),
        "charm_err_reset": ([P(_Err)], None),
        "charm_err_handler": ([P(_Err), ct.c_bool], None),
        "charm_err_isempty": ([P(_Err)], ct.c_bool),
        "charm_crd_point_malloc": ([_ct_int, SZ, SZ], P(_Point)),
        "charm_crd_point_calloc": ([_ct_int, SZ, SZ], P(_Point)),
        "charm_crd_point_init": ([_ct_int, SZ, SZ, P(D), P(D), P(D)],
                                 P(_Point)),
        "charm_crd_point_free": ([P(_Point)], None),
        "charm_crd_point_gl": ([UL, D], P(_Point)),
        "charm_crd_point_dh1": ([UL, D], P(_Point)),
        "charm_crd_point_dh2": ([UL, D], P(_Point)),
        "charm_crd_point_gl_shape": ([UL, P(SZ), P(SZ)], None),
        "charm_crd_point_dh1_shape": ([UL, P(SZ), P(SZ)], None),
        "charm_crd_point_dh2_shape": ([UL, P(SZ), P(SZ)], None),
        "charm_shc_malloc": ([UL, D, D], P(_Shc)),
        "charm_shc_calloc": ([UL, D, D], P(_Shc)),
        "charm_shc_init": ([UL, D, D, P(D), P(D)], P(_Shc)),
        "charm_shc_free": ([P(_Shc)], None),
        "charm_shs_point": ([P(_Point), P(_Shc), UL, P(D), P(_Err)], None),
        "charm_shs_point_grad1": ([P(_Point), P(_Shc), UL, P(P(D)), P(_Err)],
                                  None),
        "charm_shs_point_grad2": ([P(_Point), P(_Shc), UL, P(P(D)), P(_Err)],
                                  None),
        "charm_shs_point_guru": ([P(_Point), P(_Shc), UL, ct.c_uint,
                                  ct.c_uint, ct.c_uint, P(D), P(_Err)], None),
        "charm_sha_point": ([P(_Point), P(D), UL, P(_Shc), P(_Err)], None),
        "charm_crd_cell_malloc": ([_ct_int, SZ, SZ], P(_Cell)),
        "charm_crd_cell_calloc": ([_ct_int, SZ, SZ], P(_Cell)),
        "charm_crd_cell_init": ([_ct_int, SZ, SZ, P(D), P(D), P(D), P(D),
                                 P(D)], P(_Cell)),
        "charm_crd_cell_free": ([P(_Cell)], None),
        "charm_shs_cell": ([P(_Cell), P(_Shc), UL, P(D), P(_Err)], None),
        "charm_sha_cell": ([P(_Cell), P(D), UL, _ct_int, P(_Shc), P(_Err)],
                           None),
        "charm_gfm_global_density_3d": (
            [P(_Shc), UL, D, P(P(_Shc)), P(UL), ct.c_uint, D, D, ct.c_uint,
             ct.c_uint, UL, ct.c_char_p, ct.c_char_p, ct.c_char_p, P(_Shc),
             P(_Err)], None),
        "charm_gfm_global_density_lateral": (
            [P(_Shc), UL, D, P(_Shc), UL, D, D, ct.c_uint, ct.c_uint, UL,
             ct.c_char_p, ct.c_char_p, ct.c_char_p, P(_Shc), P(_Err)], None),
        "charm_gfm_global_density_const": (
            [P(_Shc), UL, D, D, D, D, ct.c_uint, ct.c_uint, UL, ct.c_char_p,
             ct.c_char_p, ct.c_char_p, P(_Shc), P(_Err)], None),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


_libcharm = _load()
