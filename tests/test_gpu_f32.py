"""Single-precision mode (charm_b200_shs_point_dev_f32 /
charm_b200_sha_point_dev_f32) against the FP64 path on the same inputs.

FP32 keeps about 7 significant digits per value; over thousands of degrees
the recurrence and the sums lose one to two more, so the fields agree with
the FP64 path to a relative RMS of a few 1e-6 and the round trip returns
the coefficients to a few 1e-5 (tolerances below leave a factor of ten)."""
import ctypes as ct

import numpy as np
import pytest

from charm_b200.workloads import GM, R_EARTH, coef_rel_rms, kaula, rel_rms

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    import charm_b200 as cb
    from charm_b200._lib import _libcharm as L
    P = ct.c_void_p
    L.charm_b200_shs_point_dev_f32.argtypes = [
        P, ct.c_ulong, ct.c_double, ct.c_double, P, P, ct.c_ulong, P, P]
    L.charm_b200_sha_point_dev_f32.argtypes = [
        P, P, ct.c_ulong, ct.c_double, ct.c_double, ct.c_ulong, P, P, P]
    return torch, cb, L


def _err(L):
    return L.charm_err_init()


def _check(L, err):
    if L.charm_err_isempty(err):
        return None
    msg = ct.string_at(err.contents.msg).decode()
    L.charm_err_reset(err)
    return msg


def shs32(env, pnt, c, s, N, R=R_EARTH):
    torch, cb, L = env
    d_c = torch.from_numpy(c.astype(np.float32)).cuda()
    d_s = torch.from_numpy(s.astype(np.float32)).cuda()
    f = torch.empty(pnt.lat.size * pnt.lon.size, dtype=torch.float32,
                    device="cuda")
    err = _err(L)
    L.charm_b200_shs_point_dev_f32(ct.cast(pnt._Point, ct.c_void_p), N, GM, R,
                                   d_c.data_ptr(), d_s.data_ptr(), N,
                                   f.data_ptr(), ct.cast(err, ct.c_void_p))
    msg = _check(L, err)
    L.charm_err_free(err)
    return f, msg


def sha32(env, pnt, f, N, R=R_EARTH):
    torch, cb, L = env
    T = (N + 1) * (N + 2) // 2
    oc = torch.empty(T, dtype=torch.float32, device="cuda")
    os_ = torch.empty(T, dtype=torch.float32, device="cuda")
    err = _err(L)
    L.charm_b200_sha_point_dev_f32(ct.cast(pnt._Point, ct.c_void_p),
                                   f.data_ptr(), N, GM, R, N, oc.data_ptr(),
                                   os_.data_ptr(), ct.cast(err, ct.c_void_p))
    msg = _check(L, err)
    L.charm_err_free(err)
    return oc.cpu().numpy().astype(np.float64), os_.cpu().numpy().astype(
        np.float64), msg


@pytest.mark.parametrize("grid,N", [("GL", 360), ("DH1", 200), ("DH2", 300),
                                    ("GL", 2190)])
def test_f32_against_f64(env, grid, N):
    torch, cb, L = env
    ctor = {"GL": cb.PointGridGL, "DH1": cb.PointGridDH1,
            "DH2": cb.PointGridDH2}[grid]
    c, s = kaula(N, 700 + N)
    p = ctor(N, R_EARTH)
    # the FP64 path on the float-rounded coefficients
    c32 = c.astype(np.float32).astype(np.float64)
    s32 = s.astype(np.float32).astype(np.float64)
    ref = cb.shs_point(p, cb.Shc(N, GM, R_EARTH, c32, s32), N)
    f, msg = shs32(env, p, c, s, N)
    assert msg is None, msg
    f64 = f.cpu().numpy().astype(np.float64).reshape(ref.shape)
    e_shs = rel_rms(f64, ref)
    # and of the disturbing part (without the degree-0 term)
    e_dist = rel_rms(f64 - GM / R_EARTH, ref - GM / R_EARTH)
    oc, os_, msg = sha32(env, p, f, N)
    assert msg is None, msg
    e_rt = coef_rel_rms(oc, os_, c32, s32)
    print("%s %d: shs %.2e (disturbing %.2e), round trip %.2e"
          % (grid, N, e_shs, e_dist, e_rt))
    assert e_shs <= 1e-6
    assert e_dist <= 5e-2
    assert e_rt <= 1e-4


def test_f32_rejects_unsupported(env):
    torch, cb, L = env
    N = 30
    c, s = kaula(N, 5)
    lat = np.linspace(1.0, -1.0, 16)
    lon = np.arange(62) * (2 * np.pi / 62)
    p = cb.PointGrid(lat, lon, np.full(16, R_EARTH + 1000.0))
    f, msg = shs32(env, p, c, s, N)
    assert msg is not None and "r = R" in msg
    q = cb.PointSctr(lat, lon[:16], np.full(16, R_EARTH))
    f, msg = shs32(env, q, c, s, N)
    assert msg is not None and "grids only" in msg


def test_f32_and_f64_against_quad_oracle_nmax2190(env):
    """nmax 2190 (Kaula, seed 2000, r = R) at 16 GL latitudes x 128 GL
    longitudes against CHarm's quad-precision build (fixture made by
    tests/golden/make_quad_n2190.py): the FP64 path to a relative RMS of
    1e-14 of the whole potential; the single-precision mode to 1e-6 of the
    whole potential (measured: a few 1e-8) -- its degree-0 term alone
    (GM / R = 6.25e7) sets the scale of the float rounding."""
    import os
    torch, cb, L = env
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)),
                             "golden", "shs_gl2190_quad16.npz"))
    N = int(z["nmax"])
    ref = z["f_hi"] + z["f_lo"]
    idx = z["lon_idx"]
    c, s = kaula(N, int(z["seed"]))
    nlon = 2 * (N + 1)
    lon = np.arange(nlon) * (np.pi / (N + 1))
    p = cb.PointGrid(z["lat"], lon, np.full(z["lat"].size, R_EARTH))
    f64 = cb.shs_point(p, cb.Shc(N, GM, R_EARTH, c, s), N)[:, idx]
    assert rel_rms(f64, ref) <= 1e-14
    f32, msg = shs32(env, p, c, s, N)
    assert msg is None, msg
    f32 = f32.cpu().numpy().astype(np.float64).reshape(-1, nlon)[:, idx]
    assert rel_rms(f32, ref) <= 1e-6
