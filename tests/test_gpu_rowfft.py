"""The longitude transforms (rfft.cu) against numpy's FFT in double
precision and against CHarm, through the public synthesis and analysis.

Every transform plan is covered:
  * direct mixed radix (H = 2^a 3^b, a >= 6) and Bluestein with run-time
    and compile-time plans in one CTA (M <= 9216);
  * tiny rows (fewer than 16 points) and rows of odd length (one complex
    DFT of the whole row by Bluestein);
  * rows longer than one CTA's shared memory, transformed by clusters of
    2, 4 and 8 CTAs (e.g. the 21602-point rows of the nmax 10800 GL grid
    and the 43204-point rows of its DH2 grid);
  * the quarter-length synthesis of DH2 rows whose spectra stop below L.

Synthesis reference: the oracle's lumped coefficients of the same
latitudes, summed along the parallels by numpy.fft.irfft (the role FFTW
plays in CHarm, src/shs/shs_grd_fft.c).  Analysis reference: CHarm's own
charm_sha_point (oracle/_ref), or the oracle's analysis (numpy.fft.rfft)
where CHarm's build is absent."""
import numpy as np
import pytest

from charm_b200.workloads import GM, R_EARTH, coef_rel_rms, kaula, rel_rms
from oracle import charm_ref, orc

pytestmark = pytest.mark.gpu

TOL = 1e-13
LATS = np.array([1.3, 0.7, -0.2, -1.1])


@pytest.fixture(scope="module")
def cb():
    import charm_b200
    return charm_b200


def oracle_rows(lat, nlon, N, c, s):
    """Synthesis on the points (lat x 2 pi j / nlon): oracle lumped
    coefficients and numpy's inverse real FFT."""
    lon = 2.0 * np.pi * np.arange(nlon) / nlon
    p = orc.Point(orc.GRID, lat, lon, np.full(lat.size, R_EARTH))
    return orc.shs_point(p, orc.Shc(N, GM, R_EARTH, c, s), N)[0]


@pytest.mark.parametrize("nlon,N", [
    (2, 0), (3, 1), (4, 1), (5, 2), (6, 2), (14, 6), (15, 7), (16, 7),
    (21, 10),
    (384, 120),      # H = 192 = 2^6 3, direct
    (576, 200),      # H = 288, Bluestein M = 576
    (722, 360),      # H = 361, compile-time plan M = 768
    (1001, 300),     # odd, Bluestein of the whole row, M = 2304
    (1082, 300),     # H = 541, compile-time plan M = 1152
    (1802, 500),     # H = 901, compile-time plan M = 2048
    (2522, 600),     # H = 1261, compile-time plan M = 3072
    (3242, 700),     # H = 1621, compile-time plan M = 3456
    (3962, 700),     # H = 1981, compile-time plan M = 4096
    (4382, 700),     # H = 2191, compile-time plan M = 4608
    (8000, 700),     # H = 4000, compile-time plan M = 9216
    (8764, 700),     # 4 x 2191: quarter-length synthesis
    (9218, 700),     # H = 4609: cluster of 2 CTAs, M = 10368
    (9999, 500),     # odd, cluster of 4 CTAs, M = 20736
    (21602, 800),    # H = 10801: cluster of 4 CTAs, M = 24576
    (43204, 600),    # H = 21602: cluster of 8 CTAs, M = 49152
])
def test_synthesis_rows_against_numpy(cb, nlon, N):
    c, s = kaula(N, 4242 + nlon)
    lon = 2.0 * np.pi * np.arange(nlon) / nlon
    p = cb.PointGrid(LATS, lon, np.full(LATS.size, R_EARTH))
    f = cb.shs_point(p, cb.Shc(N, GM, R_EARTH, c, s), N)
    fo = oracle_rows(LATS, nlon, N, c, s)
    assert rel_rms(f, fo) <= TOL
    f00 = GM / R_EARTH
    if N >= 2:
        # the signal without the degree-0 term, against its own size
        assert rel_rms(np.ravel(f) - f00, np.ravel(fo) - f00) <= 1e-9


def test_synthesis_rows_nmax10800_against_numpy(cb):
    """The north-star grid's row length at its full degree: 21602-point
    rows carrying orders 0..10800 (cluster transform, M = 24576)."""
    N = 10800
    c, s = kaula(N, 3000, sqrt_scaling=False)
    lat = LATS[:2]
    nlon = 2 * (N + 1)
    lon = np.arange(nlon) * (np.pi / (N + 1))
    f = cb.shs_point(cb.PointGrid(lat, lon, np.full(lat.size, R_EARTH)),
                     cb.Shc(N, GM, R_EARTH, c, s), N)
    fo = oracle_rows(lat, nlon, N, c, s)
    assert rel_rms(f, fo) <= TOL
    f00 = GM / R_EARTH
    # the signal (a few hundred m^2/s^2) against the rounding of the
    # 6.2e7 m^2/s^2 totals (measured 5.6e-10)
    assert rel_rms(np.ravel(f) - f00, np.ravel(fo) - f00) <= 2e-9


def analysis_reference(kind, N, f):
    if charm_ref.available("d"):
        C = charm_ref.Charm("d")
        k = {"GL": charm_ref.GL, "DH1": charm_ref.DH1, "DH2": charm_ref.DH2}[kind]
        cp, lat, lon, w = C.grid(k, N, R_EARTH)
        return C.sha_point(cp, np.ravel(f), N, GM, R_EARTH)
    ctor = {"GL": lambda: orc.gl(N, R_EARTH),
            "DH1": lambda: orc.dh(N, R_EARTH, orc.DH1),
            "DH2": lambda: orc.dh(N, R_EARTH, orc.DH2)}[kind]
    out = orc.sha_point(ctor(), f, N, GM, R_EARTH)
    return out.c, out.s


@pytest.mark.parametrize("grid,N", [
    ("GL", 191),    # H = 192, direct
    ("GL", 360),    # H = 361, compile-time plan M = 768
    ("DH1", 100),   # H = 101
    ("GL", 540),    # H = 541, compile-time plan M = 1152
    ("GL", 900),    # H = 901, compile-time plan M = 2048
    ("GL", 1260),   # H = 1261, compile-time plan M = 3072
    ("GL", 1620),   # H = 1621, compile-time plan M = 3456
    ("GL", 1980),   # H = 1981, compile-time plan M = 4096
    ("GL", 2190),   # H = 2191, compile-time plan M = 4608
    ("DH2", 2190),  # H = 4382, compile-time plan M = 9216
    ("GL", 4700),   # H = 4701, cluster of 2 CTAs, M = 10368
    ("DH2", 2400),  # H = 4802, cluster of 2 CTAs, M = 10368
])
def test_analysis_rows(cb, grid, N):
    """Analysis of a synthesised grid against CHarm's analysis of the same
    grid values, and the round trip back to the coefficients."""
    ctor = {"GL": cb.PointGridGL, "DH1": cb.PointGridDH1,
            "DH2": cb.PointGridDH2}[grid]
    c, s = kaula(N, 4300 + N)
    p = ctor(N, R_EARTH)
    f = cb.shs_point(p, cb.Shc(N, GM, R_EARTH, c, s), N)
    out = cb.sha_point(p, f, N, GM, R_EARTH)
    cr, sr = analysis_reference(grid, N, f)
    # rounding grows with the degree (measured 1.4e-13 at nmax 4700); at
    # nmax 540 and 1620 CHarm's own analysis (built with -ffast-math)
    # strays: 1.04e-13 and 1.23e-13 from this one, while CHarm and the
    # oracle's restatement differ by 2.2e-13 and 1.2e-13 between
    # themselves (this analysis against the oracle: 1.3e-13, 5.4e-14)
    bound = 3e-13 if N in (540, 1620) else TOL * max(1.0, N / 2190.0)
    assert coef_rel_rms(out.c, out.s, cr, sr) <= bound
    assert coef_rel_rms(out.c, out.s, c, s) <= 1e-12


def test_row_transform_constant_rows(cb):
    """A field that is constant along every row has one nonzero order."""
    N = 360
    c = np.zeros((N + 1) * (N + 2) // 2)
    s = np.zeros_like(c)
    c[0] = 1.0
    c[2] = 0.25    # C20 (order-major triangle: m = 0 column first)
    p = cb.PointGridGL(N, R_EARTH)
    f = cb.shs_point(p, cb.Shc(N, GM, R_EARTH, c, s), N)
    assert np.max(np.ptp(f, axis=1)) <= 1e-14 * np.max(np.abs(f))
