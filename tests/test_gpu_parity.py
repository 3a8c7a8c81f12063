"""The CUDA path (through libcharm.so's C ABI) against the CPU oracle on the
same seeded inputs, at sizes the oracle finishes in seconds, and
size-independent properties (SHA(SHS(c)) = c) at larger sizes.

Tolerances are relative RMS errors: the GPU and the oracle run the same
recurrences in double precision and differ only by rounding (fused
multiply-adds, summation order), so 1e-13 leaves two orders of margin over
what is observed and matches the north-star bound at nmax 2190."""
import numpy as np
import pytest

import golden_data as gd
from charm_b200.workloads import GM, R_EARTH, coef_rel_rms, kaula, rel_rms
from oracle import orc

pytestmark = pytest.mark.gpu

TOL = 1e-13


@pytest.fixture(scope="module")
def cb():
    import charm_b200
    return charm_b200


def ora_shc(nmax, c, s, mu=GM, r=R_EARTH):
    return orc.Shc(nmax, mu, r, c, s)


def test_shs_gl_360_vs_oracle(cb):
    """Config 1: nmax 360 on the GL grid 361 x 722, r = R."""
    N = 360
    c, s = kaula(N, 1000)
    p = cb.PointGridGL(N, R_EARTH)
    f = cb.shs_point(p, cb.Shc(N, GM, R_EARTH, c, s), N)
    fo = orc.shs_point(orc.gl(N, R_EARTH), ora_shc(N, c, s), N)[0]
    assert rel_rms(f, fo) <= TOL


def test_sha_gl_360_vs_oracle(cb):
    N = 360
    c, s = kaula(N, 1001)
    p = cb.PointGridGL(N, R_EARTH)
    f = cb.shs_point(p, cb.Shc(N, GM, R_EARTH, c, s), N)
    out = cb.sha_point(p, f, N, GM, R_EARTH)
    ref = orc.sha_point(orc.gl(N, R_EARTH), f, N, GM, R_EARTH)
    assert coef_rel_rms(out.c, out.s, ref.c, ref.s) <= TOL
    # and the round trip
    assert coef_rel_rms(out.c, out.s, c, s) <= 1e-12


@pytest.mark.parametrize("grid", ["dh1", "dh2"])
def test_dh_above_sphere_vs_oracle(cb, grid):
    """DH grids at r = R + 250 km (the batched workload's grids)."""
    N = 200
    c, s = kaula(N, 4000)
    r = R_EARTH + 250e3
    ctor = cb.PointGridDH1 if grid == "dh1" else cb.PointGridDH2
    kind = orc.DH1 if grid == "dh1" else orc.DH2
    p = ctor(N, r)
    f = cb.shs_point(p, cb.Shc(N, GM, R_EARTH, c, s), N)
    fo = orc.shs_point(orc.dh(N, r, kind), ora_shc(N, c, s), N)[0]
    assert rel_rms(f, fo) <= TOL
    # the transforms compared on the analysis sphere (no rescaling)
    out = cb.sha_point(p, f, N, GM, r)
    ref = orc.sha_point(orc.dh(N, r, kind), f, N, GM, r)
    assert coef_rel_rms(out.c, out.s, ref.c, ref.s) <= TOL
    # round trip referred back to R: CHarm's rescaling by (r/R)^n
    # (src/shc/shc_rescale.c) amplifies the double-precision noise of the
    # field by up to (r/R)^N ~ 2e3 at degree 200, hence the looser bound
    back = cb.sha_point(p, f, N, GM, R_EARTH)
    amp = (r / R_EARTH) ** N
    assert coef_rel_rms(back.c, back.s, c, s) <= 1e-14 * amp


@pytest.mark.parametrize("kind", ["grad1", "grad2"] + [k for k in gd.GURU])
def test_derivatives_vs_oracle(cb, kind):
    """Gradients in the local north-oriented frame and all single
    derivatives at nmax 120, GL grid at R + 5 km (rows within 1 degree of
    the poles excluded, as CHarm's tests exclude the singular rows)."""
    N = 120
    c, s = kaula(N, 77)
    r = R_EARTH + 5000.0
    p = cb.PointGridGL(N, r)
    shc = cb.Shc(N, GM, R_EARTH, c, s)
    if kind == "grad1":
        out = cb.shs_point_grad1(p, shc, N)
    elif kind == "grad2":
        out = cb.shs_point_grad2(p, shc, N)
    else:
        out = [cb.shs_point_guru(p, shc, N, *kind)]
    ref = orc.shs_point(orc.gl(N, r), ora_shc(N, c, s), N, kind)
    keep = np.abs(p.lat) < np.deg2rad(89.0)
    for o, fo in zip(out, ref):
        o = np.asarray(o).reshape(p.lat.size, -1)[keep]
        fo = fo.reshape(p.lat.size, -1)[keep]
        assert rel_rms(o, fo) <= 1e-12


def test_scattered_vs_oracle(cb):
    """Scattered points with heights 0..9000 m (the adjoint workload's
    geometry), nmax 150."""
    N = 150
    rng = np.random.default_rng(5001)
    n = 2000
    lat = np.arcsin(rng.uniform(-1, 1, n))
    lon = rng.uniform(0, 2 * np.pi, n)
    r = R_EARTH + rng.uniform(0, 9000, n)
    c, s = kaula(N, 5000)
    f = cb.shs_point(cb.PointSctr(lat, lon, r), cb.Shc(N, GM, R_EARTH, c, s), N)
    fo = orc.shs_point(orc.Point(orc.SCATTERED, lat, lon, r), ora_shc(N, c, s),
                       N)[0]
    assert rel_rms(f, fo) <= TOL
    g = cb.shs_point_grad1(cb.PointSctr(lat, lon, r),
                           cb.Shc(N, GM, R_EARTH, c, s), N)
    go = orc.shs_point(orc.Point(orc.SCATTERED, lat, lon, r), ora_shc(N, c, s),
                       N, "grad1")
    for a, b in zip(g, go):
        assert rel_rms(a, b) <= 1e-12


def test_polar_rows_high_degree_vs_oracle(cb):
    """X-number range: nmax 2000 at latitudes within 2 degrees of the poles
    (sectorial values down to ~1e-3000), single meridian, against the oracle
    that restates CHarm's X-number arithmetic."""
    N = 2000
    c, s = kaula(N, 2024)
    lat = np.deg2rad(np.concatenate([np.linspace(89.99, 88.0, 12),
                                     [45.0, 10.0, -30.0]]))
    lon = np.array([0.3])
    r = np.full(lat.size, R_EARTH)
    f = cb.shs_point(cb.PointGrid(lat, lon, r), cb.Shc(N, GM, R_EARTH, c, s), N)
    fo = orc.shs_point(orc.Point(orc.GRID, lat, lon, r), ora_shc(N, c, s), N)[0]
    assert rel_rms(f, fo) <= TOL
    rel = np.abs(f.ravel() - fo) / np.abs(fo)
    assert np.max(rel) <= 1e-12


def test_custom_grid_direct_longitudes(cb):
    """A symmetric custom grid whose longitudes do not span 2 pi (no FFT):
    the direct longitude sums against the oracle."""
    N = 80
    c, s = kaula(N, 31)
    lat = np.deg2rad(np.linspace(80.0, -80.0, 33))
    lon = np.deg2rad(np.linspace(10.0, 200.0, 57))
    r = np.full(lat.size, R_EARTH + 100.0)
    f = cb.shs_point(cb.PointGrid(lat, lon, r), cb.Shc(N, GM, R_EARTH, c, s), N)
    fo = orc.shs_point(orc.Point(orc.GRID, lat, lon, r), ora_shc(N, c, s), N)[0]
    assert rel_rms(f, fo) <= TOL


def test_custom_grid_longitude_recurrence_high_degree(cb):
    """A regional grid (longitudes 10..60 degrees, no FFT) at nmax 1500:
    the longitude sums run the rotation recurrence over 1501 orders
    (restarted every 64), against the oracle's direct sums and against
    CHarm's own PSLR path (src/shs/shs_grd_lr.c) where its build exists."""
    from oracle import charm_ref
    N = 1500
    c, s = kaula(N, 37)
    lat = np.deg2rad(np.linspace(50.0, 30.0, 12))
    lon = np.deg2rad(np.linspace(10.0, 60.0, 301))
    r = np.full(lat.size, R_EARTH)
    f = cb.shs_point(cb.PointGrid(lat, lon, r), cb.Shc(N, GM, R_EARTH, c, s), N)
    fo = orc.shs_point(orc.Point(orc.GRID, lat, lon, r), ora_shc(N, c, s), N)[0]
    assert rel_rms(f, fo) <= TOL
    f00 = GM / R_EARTH
    assert rel_rms(np.ravel(f) - f00, np.ravel(fo) - f00) <= 1e-9
    if charm_ref.available("d"):
        C = charm_ref.Charm("d")
        fr = C.shs_point(C.point(charm_ref.GRID, lat, lon, r),
                         C.shc(N, GM, R_EARTH, c, s), N, lat.size * lon.size)
        assert rel_rms(f, fr) <= TOL


@pytest.mark.parametrize("N", [2190])
def test_round_trip_large(cb, N):
    """Config 2: nmax 2190 on GL 2191 x 4382 -- SHA(SHS(c)) recovers c."""
    c, s = kaula(N, 2000)
    p = cb.PointGridGL(N, R_EARTH)
    f = cb.shs_point(p, cb.Shc(N, GM, R_EARTH, c, s), N)
    out = cb.sha_point(p, f, N, GM, R_EARTH)
    assert coef_rel_rms(out.c, out.s, c, s) <= 1e-12


def test_shs_2190_rows_vs_oracle(cb):
    """Config 2 grid synthesis against the oracle on a subset of rows (the
    oracle evaluates the same GL latitudes as a custom grid)."""
    N = 2190
    c, s = kaula(N, 2000)
    p = cb.PointGridGL(N, R_EARTH)
    f = cb.shs_point(p, cb.Shc(N, GM, R_EARTH, c, s), N).reshape(p.lat.size, -1)
    rows = np.array([0, 1, 7, 300, 1095, 1500, 2189, 2190])
    fo = orc.shs_point(orc.Point(orc.GRID, p.lat[rows], p.lon, p.r[rows]),
                       ora_shc(N, c, s), N)[0].reshape(rows.size, -1)
    assert rel_rms(f[rows], fo) <= TOL


def test_polar_optimisation(cb):
    """With CHarm's polar optimisation on (a1 = 100, a2 = 0.01) the results
    stay within 1e-12 (relative RMS) of the full computation."""
    import ctypes as ct
    from charm_b200._lib import _libcharm
    N = 720
    c, s = kaula(N, 9)
    p = cb.PointGridGL(N, R_EARTH)
    shc = cb.Shc(N, GM, R_EARTH, c, s)
    f0 = cb.shs_point(p, shc, N)
    a2 = ct.c_double.in_dll(_libcharm, "charm_glob_polar_optimization_a2")
    old = a2.value
    try:
        a2.value = 0.01
        f1 = cb.shs_point(p, shc, N)
    finally:
        a2.value = old
    assert rel_rms(f1, f0) <= 1e-12


def test_deterministic(cb):
    """Same inputs twice give bitwise-equal outputs (no atomics in the
    summations)."""
    N = 500
    c, s = kaula(N, 5)
    p = cb.PointGridGL(N, R_EARTH)
    shc = cb.Shc(N, GM, R_EARTH, c, s)
    f1 = cb.shs_point(p, shc, N)
    f2 = cb.shs_point(p, shc, N)
    assert np.array_equal(f1, f2)
    o1 = cb.sha_point(p, f1, N, GM, R_EARTH)
    o2 = cb.sha_point(p, f1, N, GM, R_EARTH)
    assert np.array_equal(o1.c, o2.c) and np.array_equal(o1.s, o2.s)
