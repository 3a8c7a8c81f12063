"""Host-array entry points with page-locked host arrays, the grid copied in
bands: charm_shs_point
copies the rows of each band of latitude tiles to the host while the next
band is synthesised, charm_sha_point copies band b while band b - 1 is
transformed and analysed, and copies the coefficients to the host in bands
of orders while the last band is analysed.  Synthesis work items compute the
same sums as in one launch, so the grids equal those of the device-array
entry point bit for bit.  The analysis of a host grid adds its partial sums
in groups of single latitude tiles (the device-array entry point in larger
groups), so its coefficients agree to rounding: 1e-14 relative RMS.
(Pageable host arrays take the ring of page-locked buffers instead:
tests/test_gpu_pageable.py.)"""
import ctypes as ct

import numpy as np
import pytest

from charm_b200.workloads import GM, R_EARTH, coef_rel_rms, kaula

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    import charm_b200 as cb
    from charm_b200._lib import _libcharm as L
    P = ct.c_void_p
    L.charm_b200_shs_point_dev.argtypes = [
        P, ct.c_ulong, ct.c_double, ct.c_double, P, P, ct.c_ulong, ct.c_int,
        ct.c_uint, ct.c_uint, ct.c_uint, P, P]
    L.charm_b200_sha_point_dev.argtypes = [
        P, P, ct.c_ulong, ct.c_double, ct.c_double, ct.c_ulong, P, P, P]
    return torch, cb, L


def device_shs(env, p, c, s, N):
    torch, cb, L = env
    dc = torch.from_numpy(c).cuda()
    ds = torch.from_numpy(s).cuda()
    f = torch.empty(p.lat.size * p.lon.size, dtype=torch.float64,
                    device="cuda")
    err = L.charm_err_init()
    L.charm_b200_shs_point_dev(ct.cast(p._Point, ct.c_void_p), N, GM,
                               R_EARTH, dc.data_ptr(), ds.data_ptr(), N, 0, 0,
                               0, 0, f.data_ptr(), ct.cast(err, ct.c_void_p))
    assert L.charm_err_isempty(err)
    L.charm_err_free(err)
    return f.cpu().numpy().reshape(p.lat.size, p.lon.size)


def device_sha(env, p, f, N):
    torch, cb, L = env
    df = torch.from_numpy(np.ascontiguousarray(f).ravel()).cuda()
    T = (N + 1) * (N + 2) // 2
    oc = torch.empty(T, dtype=torch.float64, device="cuda")
    os_ = torch.empty(T, dtype=torch.float64, device="cuda")
    err = L.charm_err_init()
    L.charm_b200_sha_point_dev(ct.cast(p._Point, ct.c_void_p), df.data_ptr(),
                               N, GM, R_EARTH, N, oc.data_ptr(),
                               os_.data_ptr(), ct.cast(err, ct.c_void_p))
    assert L.charm_err_isempty(err)
    L.charm_err_free(err)
    return oc.cpu().numpy(), os_.cpu().numpy()


def pinned_round_trip(env, p, c, s, N, analyse):
    """charm_shs_point (and charm_sha_point of its grid) with page-locked
    host arrays: the banded paths."""
    torch, cb, L = env
    P = ct.POINTER(ct.c_double)
    T = (N + 1) * (N + 2) // 2
    hc = torch.from_numpy(c).pin_memory()
    hs = torch.from_numpy(s).pin_memory()
    hf = torch.empty(p.lat.size * p.lon.size, dtype=torch.float64).pin_memory()
    oc = torch.zeros(T, dtype=torch.float64).pin_memory()
    os_ = torch.zeros(T, dtype=torch.float64).pin_memory()
    shc_in = L.charm_shc_init(N, GM, R_EARTH, ct.cast(hc.data_ptr(), P),
                              ct.cast(hs.data_ptr(), P))
    shc_out = L.charm_shc_init(N, GM, R_EARTH, ct.cast(oc.data_ptr(), P),
                               ct.cast(os_.data_ptr(), P))
    err = L.charm_err_init()
    L.charm_shs_point(p._Point, shc_in, N, ct.cast(hf.data_ptr(), P), err)
    assert L.charm_err_isempty(err)
    if analyse:
        L.charm_sha_point(p._Point, ct.cast(hf.data_ptr(), P), N, shc_out,
                          err)
        assert L.charm_err_isempty(err)
    L.charm_err_free(err)
    L.charm_shc_free(shc_in)
    L.charm_shc_free(shc_out)
    return (hf.numpy().reshape(p.lat.size, p.lon.size).copy(),
            oc.numpy().copy(), os_.numpy().copy())


@pytest.mark.parametrize("grid,N,h", [("GL", 2190, 0.0), ("GL", 601, 0.0),
                                      ("DH1", 800, 0.0), ("DH2", 700, 3e4)])
def test_host_paths_equal_device_paths(env, grid, N, h):
    torch, cb, L = env
    ctor = {"GL": cb.PointGridGL, "DH1": cb.PointGridDH1,
            "DH2": cb.PointGridDH2}[grid]
    p = ctor(N, R_EARTH + h)
    c, s = kaula(N, 880 + N)
    f_host, hc, hs = pinned_round_trip(env, p, c, s, N, h == 0.0)
    f_dev = device_shs(env, p, c, s, N)
    assert np.array_equal(f_host, f_dev)
    if h == 0.0:
        oc, os_ = device_sha(env, p, f_host, N)
        assert coef_rel_rms(hc, hs, oc, os_) <= 1e-14
        # every coefficient, not only the RMS
        scale = np.max(np.abs(np.concatenate([oc, os_])))
        assert np.max(np.abs(hc - oc)) <= 1e-13 * scale
        assert np.max(np.abs(hs - os_)) <= 1e-13 * scale


class ScatteredShc:
    """A charm_shc whose columns C[m], S[m] are separate arrays (allowed by
    CHarm's layout: one pointer per order), so that the copies go column by
    column."""

    def __init__(self, N, c, s):
        from charm_b200._lib import _Shc
        P = ct.POINTER(ct.c_double)
        idx = [m * (2 * N + 3 - m) // 2 for m in range(N + 2)]
        self.cc = [np.array(c[idx[m]:idx[m + 1]]) for m in range(N + 1)]
        self.cs = [np.array(s[idx[m]:idx[m + 1]]) for m in range(N + 1)]
        self.pc = (P * (N + 1))(*[a.ctypes.data_as(P) for a in self.cc])
        self.ps = (P * (N + 1))(*[a.ctypes.data_as(P) for a in self.cs])
        T = (N + 1) * (N + 2) // 2
        self.st = _Shc(nmax=N, mu=GM, r=R_EARTH, nc=T, ns=T,
                       c=ct.cast(self.pc, ct.POINTER(P)),
                       s=ct.cast(self.ps, ct.POINTER(P)), owner=False,
                       distributed=False)
        self.ptr = ct.pointer(self.st)

    def gather(self):
        return np.concatenate(self.cc), np.concatenate(self.cs)


def test_repeated_calls_and_scattered_columns(env):
    """The second host call of a shape copies the coefficients in bands of
    orders (the first one also runs the synthesis autotuner); a charm_shc
    with one array per order is copied column by column.  Grids equal the
    device-array path's bit for bit, coefficients agree to rounding."""
    torch, cb, L = env
    N = 600
    p = cb.PointGridGL(N, R_EARTH)
    c, s = kaula(N, 777)
    f_dev = device_shs(env, p, c, s, N)
    for _ in range(3):
        assert np.array_equal(pinned_round_trip(env, p, c, s, N, False)[0],
                              f_dev)
    sc = ScatteredShc(N, c, s)
    # page-locked grids (the banded paths), coefficient columns in
    # pageable arrays of their own
    f = torch.empty(p.lat.size * p.lon.size,
                    dtype=torch.float64).pin_memory().numpy()
    P = ct.POINTER(ct.c_double)
    oc, os_ = device_sha(env, p, f_dev, N)
    out = ScatteredShc(N, np.zeros_like(c), np.zeros_like(s))
    fd = torch.from_numpy(np.ascontiguousarray(f_dev).ravel()).pin_memory()
    fd = fd.numpy()
    for _ in range(2):
        err = L.charm_err_init()
        L.charm_shs_point(p._Point, sc.ptr, N, f.ctypes.data_as(P), err)
        assert L.charm_err_isempty(err)
        L.charm_sha_point(p._Point, fd.ctypes.data_as(P), N, out.ptr, err)
        assert L.charm_err_isempty(err)
        L.charm_err_free(err)
        assert np.array_equal(f.reshape(p.lat.size, p.lon.size), f_dev)
        gc, gs = out.gather()
        assert coef_rel_rms(gc, gs, oc, os_) <= 1e-14
