"""The CUDA path against CHarm 0.4.9 itself (its double-precision build in
oracle/_ref, compiled from CHarm's own sources with OpenMP and AVX-512 /
AVX2, -O3 -ffast-math), on the same seeded inputs and the same points.

Tolerances are relative RMS differences: both sides compute in double
precision and differ by rounding only (CHarm's X-number arithmetic and
SIMD summation order against the GPU's rescaled recurrence and fused
multiply-adds).  The bound at nmax 2190 is 1e-13."""
import numpy as np
import pytest

from charm_b200.workloads import GM, R_EARTH, coef_rel_rms, kaula, rel_rms
from charm_b200.workloads import tri_orders
from oracle import charm_ref

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not charm_ref.available("d"),
                                 reason="oracle/_ref has no CHarm build")]

TOL = 1e-13


@pytest.fixture(scope="module")
def cb():
    import charm_b200
    return charm_b200


@pytest.fixture(scope="module")
def C():
    return charm_ref.Charm("d")


@pytest.mark.parametrize("r", [R_EARTH, R_EARTH + 5000.0])
def test_shs_sha_gl360_vs_charm(cb, C, r):
    """nmax 360, GL grid 361 x 722, on and above the sphere; synthesis
    field and analysis coefficients of the same grid."""
    N = 360
    c, s = kaula(N, 1000)
    p = cb.PointGridGL(N, r)
    f = cb.shs_point(p, cb.Shc(N, GM, R_EARTH, c, s), N)
    cp, lat, lon, w = C.grid(charm_ref.GL, N, r)
    fr = C.shs_point(cp, C.shc(N, GM, R_EARTH, c, s), N, lat.size * lon.size)
    assert rel_rms(f, fr) <= TOL
    out = cb.sha_point(p, f, N, GM, R_EARTH)
    cr, sr = C.sha_point(cp, np.ravel(f), N, GM, R_EARTH)
    assert coef_rel_rms(out.c, out.s, cr, sr) <= TOL


@pytest.mark.parametrize("grid", ["dh1", "dh2"])
def test_grads_dh_vs_charm(cb, C, grid):
    """Potential, grad1 and grad2 on DH grids at R + 250 km (the batched
    workload's grids and quantities), nmax 300."""
    N = 300
    c, s = kaula(N, 4001)
    r = R_EARTH + 250e3
    ctor = cb.PointGridDH1 if grid == "dh1" else cb.PointGridDH2
    kind = charm_ref.DH1 if grid == "dh1" else charm_ref.DH2
    p = ctor(N, r)
    shc = cb.Shc(N, GM, R_EARTH, c, s)
    cp, lat, lon, w = C.grid(kind, N, r)
    csh = C.shc(N, GM, R_EARTH, c, s)
    npt = lat.size * lon.size
    assert rel_rms(cb.shs_point(p, shc, N), C.shs_point(cp, csh, N, npt)) <= TOL
    # the x / y components are singular at a pole (the DH grids' first
    # row): compared off the poles, as CHarm's own tests zero them there
    # (tests/check_shs_point_all.c:229-300)
    keep = np.repeat(np.cos(p.lat) > 1e-8, lon.size)
    for order, fn in ((1, cb.shs_point_grad1), (2, cb.shs_point_grad2)):
        mine = fn(p, shc, N)
        ref = C.shs_point_grad(cp, csh, N, npt, order)
        # each component against the largest component's RMS (single
        # components vanish on parts of the grid)
        scale = max(np.sqrt(np.mean(x[keep] ** 2)) for x in ref)
        for q, (a, b) in enumerate(zip(mine, ref)):
            singular = q < (2 if order == 1 else 5)
            sel = keep if singular else slice(None)
            d = np.ravel(a)[sel] - b[sel]
            assert np.sqrt(np.mean(d * d)) / scale <= 1e-12, (order, q)


def test_shs_2190_rows_vs_charm(cb, C):
    """nmax 2190 synthesis: 24 latitudes of the GL grid (both poles'
    neighbourhoods and the equator included) times all 4382 GL longitudes,
    the same points on both sides."""
    N = 2190
    c, s = kaula(N, 2000)
    g = cb.PointGridGL(N, R_EARTH)
    sel = np.unique(np.concatenate([np.arange(4), np.arange(N - 3, N + 1),
                                    np.linspace(0, N, 16).astype(int)]))
    lat = g.lat[sel].copy()
    lon = g.lon.copy()
    rr = np.full(lat.size, R_EARTH)
    f = cb.shs_point(cb.PointGrid(lat, lon, rr), cb.Shc(N, GM, R_EARTH, c, s), N)
    cp = C.point(charm_ref.GRID, lat, lon, rr)
    fr = C.shs_point(cp, C.shc(N, GM, R_EARTH, c, s), N, lat.size * lon.size)
    assert rel_rms(f, fr) <= TOL
    f00 = GM / R_EARTH
    # the part without the degree-0 term, against its own RMS: the rounding
    # of the 6.2e7 m^2/s^2 totals on either side sets its floor (measured
    # 1.1e-9)
    assert rel_rms(np.ravel(f) - f00, fr - f00) <= 5e-9


def test_sha_2190_vs_charm(cb, C):
    """nmax 2190 analysis: CHarm's and the GPU's analysis of the same grid
    (the GPU's synthesis of seed 2000), the whole triangle and order by
    order (m = 0, 1, 2, N/2 and the last orders), each order's difference
    against the triangle's norm (the grid values' rounding, set by the
    degree-0 term, is the floor of every coefficient's error)."""
    N = 2190
    c, s = kaula(N, 2000)
    p = cb.PointGridGL(N, R_EARTH)
    f = cb.shs_point(p, cb.Shc(N, GM, R_EARTH, c, s), N)
    out = cb.sha_point(p, f, N, GM, R_EARTH)
    cp, lat, lon, w = C.grid(charm_ref.GL, N, R_EARTH)
    cr, sr = C.sha_point(cp, np.ravel(f), N, GM, R_EARTH)
    assert coef_rel_rms(out.c, out.s, cr, sr) <= TOL
    norm = np.sqrt(np.sum(cr * cr + sr * sr))
    m = tri_orders(N)
    for mm in (0, 1, 2, N // 2, N - 2, N - 1, N):
        k = m == mm
        d = np.sqrt(np.sum((out.c[k] - cr[k]) ** 2 + (out.s[k] - sr[k]) ** 2))
        assert d / norm <= TOL, mm
