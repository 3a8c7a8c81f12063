"""The CUDA path against the golden vectors of CHarm's own test-suite, with
CHarm's tolerances (tests/check_shs_point_all.c, check_crd_point_quad.c,
check_sha_point.c), called through the C ABI of libcharm.so."""
import numpy as np
import pytest

import golden_data as gd
from gpu_cases import check_product

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cb():
    import charm_b200
    return charm_b200


@pytest.mark.parametrize("fam", ["pot", "grad1", "grad2", "guru"])
@pytest.mark.parametrize("subset", ["grid", "custom", "sctr", "dsun"])
def test_shs_golden(cb, fam, subset):
    cases = gd.shs_cases(families=(fam,), subsets=(subset,))
    if not cases:
        pytest.skip("no golden files for this combination")
    bad = {}
    for case in cases:
        n = check_product(cb, case)
        if n:
            bad[case.name] = n
    assert not bad, bad


def test_zero_points(cb):
    """Synthesis with zero points is valid and leaves err empty
    (check_shs_point_all.c:352-393)."""
    nmax, mu, r, c, s = gd.test_coefficients()
    shc = cb.Shc(nmax, mu, r, c, s)
    p = cb.PointSctr(np.zeros(0), np.zeros(0), np.zeros(0))
    assert cb.shs_point(p, shc, nmax).size == 0
    assert all(x.size == 0 for x in cb.shs_point_grad1(p, shc, nmax))
    assert all(x.size == 0 for x in cb.shs_point_grad2(p, shc, nmax))
    for dr, dlat, dlon in gd.GURU:
        assert cb.shs_point_guru(p, shc, nmax, dr, dlat, dlon).size == 0


@pytest.mark.parametrize("g", ["gl", "dh1", "dh2"])
def test_crd_golden(cb, g):
    """GL/DH nodes, weights, longitudes and radii computed on the GPU
    (check_crd_point_quad.c:35-95)."""
    G = gd.golden("double")
    eps = 10.0 * gd.THRESHOLD
    ctor = {"gl": cb.PointGridGL, "dh1": cb.PointGridDH1,
            "dh2": cb.PointGridDH2}[g]
    for nmax in range(11):
        for d in range(2):
            p = ctor(nmax, 1.0 + 1000.0 * d)
            key = "crd_nx%d_dr%d_%s_" % (nmax, d, g)
            assert gd.mismatches(p.lat, G[key + "lat"], eps) == 0
            assert gd.mismatches(p.lon, G[key + "lon"], eps) == 0
            assert gd.mismatches(p.r, G[key + "r"], eps) == 0
            assert gd.mismatches(p.w, G[key + "w"], eps) == 0
            assert gd.nearly_equal(np.sum(p.w), 2.0, eps)


def dda(shc_nmax, c1, s1, nmax_out, c2, s2, nmax):
    """Difference degree amplitudes, src/shc/shc_dda.c + shc_ddv.c."""
    out = np.zeros(nmax + 1)
    for n in range(nmax + 1):
        v = 0.0
        for m in range(n + 1):
            dc = c1[gd.tri_index(shc_nmax, n, m)] - c2[gd.tri_index(nmax_out, n, m)]
            ds = s1[gd.tri_index(shc_nmax, n, m)] - s2[gd.tri_index(nmax_out, n, m)]
            v += dc * dc + ds * ds
        out[n] = np.sqrt(v)
    return out


@pytest.mark.parametrize("g", ["gl", "dh1", "dh2"])
def test_sha_round_trip(cb, g):
    """check_sha_point.c:98-156: synthesis at R + 1000 m, analysis on that
    sphere rescaled to R; difference degree amplitudes equal 0 within
    10 * threshold for nmax 0..10."""
    nmax_shc, mu, r, c, s = gd.test_coefficients()
    shc = cb.Shc(nmax_shc, mu, r, c, s)
    ctor = {"gl": cb.PointGridGL, "dh1": cb.PointGridDH1,
            "dh2": cb.PointGridDH2}[g]
    for nmax in range(11):
        p = ctor(nmax, r + 1000.0)
        f = cb.shs_point(p, shc, nmax)
        out = cb.sha_point(p, f, nmax, mu, r)
        d = dda(nmax_shc, c, s, nmax, out.c, out.s, nmax)
        assert gd.mismatches(d, np.zeros_like(d), 10.0 * gd.THRESHOLD) == 0, d


def test_sha_ds_round_trip(cb):
    """check_sha_point.c:176-258: dynamical switching round trip at
    nmax 150..154 with all-ones coefficients, held to threshold2."""
    for nmax in range(150, 155):
        T = (nmax + 1) * (nmax + 2) // 2
        c = np.ones(T)
        s = np.ones(T)
        s[:nmax + 1] = 0.0          # S_n0
        shc = cb.Shc(nmax, 1.0, 1.0, c, s)
        for p in (cb.PointGridGL(nmax, 1.0), cb.PointGridDH1(nmax, 1.0),
                  cb.PointGridDH2(nmax, 1.0)):
            f = cb.shs_point(p, shc, nmax)
            out = cb.sha_point(p, f, nmax, 1.0, 1.0)
            d = dda(nmax, c, s, nmax, out.c, out.s, nmax)
            assert gd.mismatches(d, np.zeros_like(d), gd.THRESHOLD2) == 0, d


def test_errors(cb):
    """Argument errors are reported through charm_err as in CHarm."""
    nmax, mu, r, c, s = gd.test_coefficients()
    shc = cb.Shc(nmax, mu, r, c, s)
    p = cb.PointGridGL(4, r)
    with pytest.raises(cb.CHarmError):
        cb.shs_point(p, shc, nmax + 1)
    with pytest.raises(cb.CHarmError):
        cb.shs_point_guru(p, shc, 4, 1, 1, 1)
    # analysis: grid degree too low
    with pytest.raises(cb.CHarmError):
        cb.sha_point(p, np.zeros(p.lat.size * p.lon.size), 5, mu, r)
    # analysis: unequal radii
    q = cb.PointGrid(p.lat, p.lon, p.r * np.linspace(1, 2, p.r.size),
                     ptype=cb.GRID_GL)
    with pytest.raises(cb.CHarmError):
        cb.sha_point(q, np.zeros(p.lat.size * p.lon.size), 4, mu, r)
    # custom grid with non-constant longitude step
    g = cb.PointGrid([0.1, -0.1], [0.0, 0.1, 0.5], [r, r])
    with pytest.raises(cb.CHarmError):
        cb.shs_point(g, shc, 4)
