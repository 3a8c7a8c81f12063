"""The shared-memory row transforms (rfft.cu) against cuFFT on the same
lumped coefficients / grids, through the public synthesis and analysis.

CHARM_B200_ROW_FFT=library routes the longitude transforms through cuFFT
instead; both compute the same unnormalised DFTs, so the outputs agree to a
few units of rounding.  The grids cover every transform plan: direct
mixed radix (H = 2^a 3^b, a >= 6), Bluestein for every other length up to
M = 9216, the quarter-length synthesis of rows of length 4L whose spectra
stop below L (DH2 grids), and lengths where the row transform does not
apply (H < 8)."""
import os

import numpy as np
import pytest

from charm_b200.workloads import GM, R_EARTH, coef_rel_rms, kaula, rel_rms

pytestmark = pytest.mark.gpu

TOL = 1e-14


@pytest.fixture(scope="module")
def cb():
    import charm_b200
    return charm_b200


def both(fn):
    old = os.environ.pop("CHARM_B200_ROW_FFT", None)
    try:
        a = fn()
        os.environ["CHARM_B200_ROW_FFT"] = "library"
        b = fn()
    finally:
        os.environ.pop("CHARM_B200_ROW_FFT", None)
        if old is not None:
            os.environ["CHARM_B200_ROW_FFT"] = old
    return a, b


@pytest.mark.parametrize("grid,N", [
    ("GL", 7),      # H = 8, Bluestein M = 64
    ("GL", 191),    # H = 192 = 2^6 3, direct
    ("GL", 287),    # H = 288 = 2^5 3^2, Bluestein M = 576
    ("GL", 360),    # H = 361 = 19^2, Bluestein M = 768
    ("DH1", 100),   # H = 101, Bluestein M = 256
    # DH2 rows of length 4 (N + 1): synthesis by two DFTs of length N + 1
    # (Bluestein M = 4608) per row, analysis with H = 2 (N + 1), M = 9216
    ("DH2", 2190),
    ("DH2", 2160),
    ("GL", 2190),   # H = 2191, Bluestein M = 4608
    # H = 4000, M = 9216 both ways: the spectrum reaches beyond a quarter
    # of the row, so the quarter-length synthesis does not apply
    ("GL", 3999),
    ("GL", 2),      # H = 3, library transform
])
def test_row_transform_matches_library(cb, grid, N):
    ctor = {"GL": cb.PointGridGL, "DH1": cb.PointGridDH1,
            "DH2": cb.PointGridDH2}[grid]
    c, s = kaula(N, 4242 + N)
    p = ctor(N, R_EARTH)
    shc = cb.Shc(N, GM, R_EARTH, c, s)
    f_row, f_lib = both(lambda: cb.shs_point(p, shc, N))
    assert rel_rms(f_row, f_lib) <= TOL
    a_row, a_lib = both(lambda: cb.sha_point(p, f_lib, N, GM, R_EARTH))
    assert coef_rel_rms(a_row.c, a_row.s, a_lib.c, a_lib.s) <= TOL
    # and the round trip closes through the row transforms alone
    assert coef_rel_rms(a_row.c, a_row.s, c, s) <= 1e-12


def test_row_transform_zero_and_constant_rows(cb):
    """A field that is constant along every row has one nonzero order."""
    N = 360
    c = np.zeros((N + 1) * (N + 2) // 2)
    s = np.zeros_like(c)
    c[0] = 1.0
    c[2] = 0.25    # C20 (order-major triangle: m = 0 column first)
    p = cb.PointGridGL(N, R_EARTH)
    f_row, f_lib = both(lambda: cb.shs_point(p, cb.Shc(N, GM, R_EARTH, c, s),
                                             N))
    assert rel_rms(f_row, f_lib) <= TOL
    assert np.max(np.ptp(f_row, axis=1)) <= 1e-14 * np.max(np.abs(f_row))
