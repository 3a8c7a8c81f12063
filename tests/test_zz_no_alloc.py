"""charm_b200_sha_point_dev_static, the analysis entry point that allocates
nothing, against charm_b200_sha_point_dev on the same device-resident grid.

Both run the same kernels with the same work split, so the coefficients
must be identical, for two calls in a row (the second reuses the tables the
first left in the static scratch).  The device's free memory must not move
across a call after the first.  The file is named to be collected last, so
that it also runs after every other GPU test in one session."""
import ctypes as ct

import numpy as np
import pytest

from charm_b200.workloads import GM, R_EARTH, kaula

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    import charm_b200 as cb
    from charm_b200._lib import _libcharm as L
    args = [ct.c_void_p, ct.c_void_p, ct.c_ulong, ct.c_double, ct.c_double,
            ct.c_ulong, ct.c_void_p, ct.c_void_p, ct.c_void_p]
    L.charm_b200_sha_point_dev.argtypes = args
    L.charm_b200_sha_point_dev_static.argtypes = args
    L.charm_b200_shs_point_dev.argtypes = [
        ct.c_void_p, ct.c_ulong, ct.c_double, ct.c_double, ct.c_void_p,
        ct.c_void_p, ct.c_ulong, ct.c_int, ct.c_uint, ct.c_uint, ct.c_uint,
        ct.c_void_p, ct.c_void_p]
    err = L.charm_err_init()
    yield torch, cb, L, err
    L.charm_err_free(err)


def _message(L, err):
    if L.charm_err_isempty(err):
        return None
    msg = ct.string_at(err.contents.msg).decode()
    L.charm_err_reset(err)
    return msg


def _analyse(env, fn_name, pnt, d_f, nmax, r, shc_nmax):
    torch, cb, L, err = env
    T = (shc_nmax + 1) * (shc_nmax + 2) // 2
    dev = d_f.device
    d_c = torch.full((T,), np.nan, dtype=torch.float64, device=dev)
    d_s = torch.full((T,), np.nan, dtype=torch.float64, device=dev)
    getattr(L, fn_name)(ct.cast(pnt._Point, ct.c_void_p), d_f.data_ptr(),
                        nmax, GM, r, shc_nmax, d_c.data_ptr(), d_s.data_ptr(),
                        ct.cast(err, ct.c_void_p))
    msg = _message(L, err)
    assert msg is None, msg
    return d_c.cpu().numpy(), d_s.cpu().numpy()


@pytest.mark.parametrize("grid,nmax,shc_nmax,r", [
    ("GL", 360, 360, R_EARTH),          # Bluestein rows (H = 361)
    ("DH2", 200, 210, R_EARTH + 5e4),   # rescaled, zero tail above nmax
    ("GL", 511, 511, R_EARTH),          # the largest degree served
])
def test_static_matches_dev_twice(env, grid, nmax, shc_nmax, r):
    torch, cb, L, err = env
    ctor = {"GL": cb.PointGridGL, "DH2": cb.PointGridDH2}[grid]
    c, s = kaula(nmax, 9000 + nmax)
    pnt = ctor(nmax, R_EARTH)
    f = cb.shs_point(pnt, cb.Shc(nmax, GM, R_EARTH, c, s), nmax)
    d_f = torch.from_numpy(np.ascontiguousarray(f).ravel()).to("cuda:0")
    ref = _analyse(env, "charm_b200_sha_point_dev", pnt, d_f, nmax, r,
                   shc_nmax)
    for _ in range(2):
        got = _analyse(env, "charm_b200_sha_point_dev_static", pnt, d_f,
                       nmax, r, shc_nmax)
        assert np.array_equal(got[0], ref[0])
        assert np.array_equal(got[1], ref[1])


def test_static_second_call_allocates_nothing(env):
    torch, cb, L, err = env
    nmax = 300
    c, s = kaula(nmax, 77)
    pnt = cb.PointGridGL(nmax, R_EARTH)
    f = cb.shs_point(pnt, cb.Shc(nmax, GM, R_EARTH, c, s), nmax)
    d_f = torch.from_numpy(np.ascontiguousarray(f).ravel()).to("cuda:0")
    T = (nmax + 1) * (nmax + 2) // 2
    d_c = torch.empty(T, dtype=torch.float64, device="cuda:0")
    d_s = torch.empty(T, dtype=torch.float64, device="cuda:0")

    def call():
        L.charm_b200_sha_point_dev_static(
            ct.cast(pnt._Point, ct.c_void_p), d_f.data_ptr(), nmax, GM,
            R_EARTH, nmax, d_c.data_ptr(), d_s.data_ptr(),
            ct.cast(err, ct.c_void_p))
        msg = _message(L, err)
        assert msg is None, msg

    call()                      # set-up on this device
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    call()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_static_rejects_oversize(env):
    torch, cb, L, err = env
    nmax = 600
    pnt = cb.PointGridGL(nmax, R_EARTH)
    d_f = torch.zeros(pnt.lat.size * pnt.lon.size, dtype=torch.float64,
                      device="cuda:0")
    T = (nmax + 1) * (nmax + 2) // 2
    d_c = torch.empty(T, dtype=torch.float64, device="cuda:0")
    d_s = torch.empty(T, dtype=torch.float64, device="cuda:0")
    L.charm_b200_sha_point_dev_static(
        ct.cast(pnt._Point, ct.c_void_p), d_f.data_ptr(), nmax, GM, R_EARTH,
        nmax, d_c.data_ptr(), d_s.data_ptr(), ct.cast(err, ct.c_void_p))
    msg = _message(L, err)
    assert msg is not None and "exceeds the static scratch limit of 511" in msg
