"""Ultra-high degree, nmax 10800, plain FP64 on the GPU.

* Synthesis against the binary128 oracle at 64 latitudes (8 of them within
  0.6 degrees of the poles, where the sectorial terms need the scaled-seed
  path) times 64 of the 21602 GL longitudes (fixture made by
  tests/golden/make_quad_n10800.py).  The whole potential must agree to a
  relative RMS of 2e-14 (3.4e-15 on B200), and its part without the
  degree-0 term to 1e-9 of that part's RMS (6.5e-10 on B200).  The second
  figure is the first one rescaled: the degree-0 term alone is 1e5 times
  larger than the rest, every partial sum carries it, so the FP64 rounding
  of the whole value (a few 1e-15 of it) is a few 1e-10 of the signal, and
  no FP64 evaluation of the full sum can do better.
* SHA(SHS(c)) on the full 10801 x 21602 GL grid must return c to a
  relative RMS of 1e-12."""
import ctypes as ct
import os

import numpy as np
import pytest

from charm_b200.workloads import GM, R_EARTH, coef_rel_rms, kaula, rel_rms

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "shs_gl10800_quad64.npz")
N = 10800


@pytest.fixture(scope="module")
def coefs():
    return kaula(N, 3000, sqrt_scaling=False)


def test_n10800_against_quad_oracle(coefs):
    import charm_b200 as cb
    z = np.load(FIX)
    assert int(z["nmax"]) == N
    lat, idx = z["lat"], z["lon_idx"]
    ref = z["f_hi"] + z["f_lo"]
    nlon = 2 * (N + 1)
    lon = np.arange(nlon) * (np.pi / (N + 1))
    c, s = coefs
    p = cb.PointGrid(lat, lon, np.full(lat.size, R_EARTH))
    f = cb.shs_point(p, cb.Shc(N, GM, R_EARTH, c, s), N)[:, idx]
    assert rel_rms(f, ref) <= 2e-14
    f00 = GM / R_EARTH
    assert rel_rms(f - f00, ref - f00) <= 1e-9


def test_n10800_gl_round_trip(coefs):
    import torch
    import charm_b200 as cb
    from charm_b200._lib import _libcharm as L
    L.charm_b200_shs_point_dev.argtypes = [
        ct.c_void_p, ct.c_ulong, ct.c_double, ct.c_double, ct.c_void_p,
        ct.c_void_p, ct.c_ulong, ct.c_int, ct.c_uint, ct.c_uint, ct.c_uint,
        ct.c_void_p, ct.c_void_p]
    L.charm_b200_sha_point_dev.argtypes = [
        ct.c_void_p, ct.c_void_p, ct.c_ulong, ct.c_double, ct.c_double,
        ct.c_ulong, ct.c_void_p, ct.c_void_p, ct.c_void_p]
    c, s = coefs
    p = cb.PointGridGL(N, R_EARTH)
    dev = torch.device("cuda", 0)
    d_c = torch.from_numpy(c).to(dev)
    d_s = torch.from_numpy(s).to(dev)
    d_f = torch.empty(p.lat.size * p.lon.size, dtype=torch.float64,
                      device=dev)
    o_c = torch.empty_like(d_c)
    o_s = torch.empty_like(d_s)
    err = L.charm_err_init()
    try:
        L.charm_b200_shs_point_dev(ct.cast(p._Point, ct.c_void_p), N, GM,
                                   R_EARTH, d_c.data_ptr(), d_s.data_ptr(), N,
                                   0, 0, 0, 0, d_f.data_ptr(),
                                   ct.cast(err, ct.c_void_p))
        assert L.charm_err_isempty(err)
        L.charm_b200_sha_point_dev(ct.cast(p._Point, ct.c_void_p),
                                   d_f.data_ptr(), N, GM, R_EARTH, N,
                                   o_c.data_ptr(), o_s.data_ptr(),
                                   ct.cast(err, ct.c_void_p))
        assert L.charm_err_isempty(err)
    finally:
        L.charm_err_free(err)
    rt = coef_rel_rms(o_c.cpu().numpy(), o_s.cpu().numpy(), c, s)
    assert rt <= 1e-12
