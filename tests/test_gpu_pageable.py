"""Host-array entry points with pageable host memory (numpy arrays, as
PyHarm passes them): charm_shs_point / _grad1 and charm_sha_point copy such
arrays through a ring of page-locked buffers (host threads copy one chunk
while the copy engine moves the previous one) and run the transform on
device arrays.  Grids equal those of the page-locked (banded) and device
paths bit for bit; the analysis equals the device path bit for bit and the
banded one to rounding.  Sizes span several 8 MB chunks of the ring; mixed
cases (pageable grid, page-locked coefficients and the reverse) and an
output array that starts off a 16-byte boundary are covered."""
import ctypes as ct

import numpy as np
import pytest

from charm_b200.workloads import GM, R_EARTH, coef_rel_rms, kaula

pytestmark = pytest.mark.gpu

P = ct.POINTER(ct.c_double)


@pytest.fixture(scope="module")
def env():
    import torch
    import charm_b200 as cb
    from charm_b200._lib import _libcharm as L
    return torch, cb, L


def shc(L, N, c, s):
    return L.charm_shc_init(N, GM, R_EARTH, c.ctypes.data_as(P),
                            s.ctypes.data_as(P))


def pinned(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()


def pinned_empty(torch, n):
    return torch.empty(n, dtype=torch.float64).pin_memory().numpy()


def call(L, fn, *args):
    err = L.charm_err_init()
    fn(*args, err)
    ok = L.charm_err_isempty(err)
    L.charm_err_free(err)
    assert ok


def test_grid_round_trip_pageable_vs_pinned(env):
    torch, cb, L = env
    N = 1500                        # grid 36 MB, triangles 9 MB each
    p = cb.PointGridGL(N, R_EARTH)
    npt = p.lat.size * p.lon.size
    T = (N + 1) * (N + 2) // 2
    c, s = kaula(N, 4242)
    cp, sp = np.array(c), np.array(s)                  # pageable
    cl, sl = pinned(torch, c), pinned(torch, s)        # page-locked
    shc_p, shc_l = shc(L, N, cp, sp), shc(L, N, cl, sl)

    f_p = np.empty(npt)
    f_l = pinned_empty(torch, npt)
    call(L, L.charm_shs_point, p._Point, shc_p, N, f_p.ctypes.data_as(P))
    call(L, L.charm_shs_point, p._Point, shc_l, N, f_l.ctypes.data_as(P))
    assert np.array_equal(f_p, f_l)
    # mixed: page-locked coefficients, pageable grid, and the reverse
    f_m = np.empty(npt)
    call(L, L.charm_shs_point, p._Point, shc_l, N, f_m.ctypes.data_as(P))
    assert np.array_equal(f_m, f_l)
    f_m2 = pinned_empty(torch, npt)
    call(L, L.charm_shs_point, p._Point, shc_p, N, f_m2.ctypes.data_as(P))
    assert np.array_equal(f_m2, f_l)

    # analysis: pageable grid and outputs against the device path
    oc_p, os_p = np.zeros(T), np.zeros(T)
    out_p = shc(L, N, oc_p, os_p)
    call(L, L.charm_sha_point, p._Point, f_p.ctypes.data_as(P), N, out_p)
    dc = torch.empty(T, dtype=torch.float64, device="cuda")
    ds = torch.empty(T, dtype=torch.float64, device="cuda")
    df = torch.from_numpy(f_p).cuda()
    L.charm_b200_sha_point_dev.argtypes = [ct.c_void_p] * 2 + [
        ct.c_ulong, ct.c_double, ct.c_double, ct.c_ulong] + [ct.c_void_p] * 3
    err = L.charm_err_init()
    L.charm_b200_sha_point_dev(ct.cast(p._Point, ct.c_void_p), df.data_ptr(),
                               N, GM, R_EARTH, N, dc.data_ptr(), ds.data_ptr(),
                               ct.cast(err, ct.c_void_p))
    assert L.charm_err_isempty(err)
    L.charm_err_free(err)
    assert np.array_equal(oc_p, dc.cpu().numpy())
    assert np.array_equal(os_p, ds.cpu().numpy())
    # the page-locked (banded) analysis to rounding, and the truth
    oc_l, os_l = pinned_empty(torch, T), pinned_empty(torch, T)
    out_l = shc(L, N, oc_l, os_l)
    call(L, L.charm_sha_point, p._Point, f_l.ctypes.data_as(P), N, out_l)
    assert coef_rel_rms(oc_p, os_p, oc_l, os_l) <= 1e-14
    assert coef_rel_rms(oc_p, os_p, c, s) <= 1e-12
    # mixed: pageable grid, page-locked coefficients
    oc_m, os_m = pinned_empty(torch, T), pinned_empty(torch, T)
    out_m = shc(L, N, oc_m, os_m)
    call(L, L.charm_sha_point, p._Point, f_p.ctypes.data_as(P), N, out_m)
    assert np.array_equal(oc_m, oc_p) and np.array_equal(os_m, os_p)
    for h in (shc_p, shc_l, out_p, out_l, out_m):
        L.charm_shc_free(h)


def test_grad1_and_scattered_pageable_vs_pinned(env):
    torch, cb, L = env
    N = 700
    p = cb.PointGridDH1(N, R_EARTH + 5e3)
    npt = p.lat.size * p.lon.size
    c, s = kaula(N, 4343)
    # the charm_shc structures point into these arrays: keep them alive
    keep = (np.array(c), np.array(s), pinned(torch, c), pinned(torch, s))
    h_p = shc(L, N, keep[0], keep[1])
    h_l = shc(L, N, keep[2], keep[3])
    # three components; the pageable ones start off a 16-byte boundary
    buf = np.empty(3 * npt + 1)
    f_p = [buf[1 + k * npt:1 + (k + 1) * npt] for k in range(3)]
    f_l = [pinned_empty(torch, npt) for _ in range(3)]
    arr_p = (P * 3)(*[a.ctypes.data_as(P) for a in f_p])
    arr_l = (P * 3)(*[a.ctypes.data_as(P) for a in f_l])
    call(L, L.charm_shs_point_grad1, p._Point, h_p, N, arr_p)
    call(L, L.charm_shs_point_grad1, p._Point, h_l, N, arr_l)
    for a, b in zip(f_p, f_l):
        assert np.array_equal(a, b)
    # scattered points
    rng = np.random.default_rng(4444)
    n = 3_000_000                   # 24 MB per array
    q = cb.PointSctr(np.arcsin(rng.uniform(-1, 1, n)),
                     rng.uniform(0, 2 * np.pi, n),
                     R_EARTH + rng.uniform(0, 9e3, n))
    g_p = np.empty(n)
    g_l = pinned_empty(torch, n)
    call(L, L.charm_shs_point, q._Point, h_p, 200, g_p.ctypes.data_as(P))
    call(L, L.charm_shs_point, q._Point, h_l, 200, g_l.ctypes.data_as(P))
    assert np.array_equal(g_p, g_l)
    L.charm_shc_free(h_p)
    L.charm_shc_free(h_l)
