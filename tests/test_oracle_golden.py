"""Pins the CPU oracle (oracle/orc.c, oracle/orc.py) against the golden
vectors of CHarm's own test-suite, with the tolerances CHarm applies
(tests/check_shs_point_all.c, tests/check_crd_point_quad.c)."""
import numpy as np
import pytest

import golden_data as gd
from oracle import orc


def oracle_point(case):
    if case.grid is not None:
        g, nmax, r = case.grid
        if g == "gl":
            p = orc.gl(nmax, r)
        else:
            p = orc.dh(nmax, r, orc.DH1 if g == "dh1" else orc.DH2)
        if case.nlon_override is not None:
            p.lon = p.lon[:case.nlon_override].copy()
        if case.lat0_shift:
            p.lat = p.lat.copy()
            p.lat[0] -= case.lat0_shift
        return p
    return orc.Point(case.ptype, case.lat, case.lon, case.r)


def check_case(case, f_list):
    G = gd.golden("double")
    bad = 0
    lat = case_lat(case)
    nlon = case_nlon(case)
    for j, (nm, f) in enumerate(zip(case.golden_names, f_list)):
        if gd.singular_component(case.kind, j):
            f = gd.zero_singular_rows(case.ptype, lat, nlon, f)
        bad += gd.mismatches(f, G[nm], case.eps)
    return bad


def case_lat(case):
    return oracle_point(case).lat


def case_nlon(case):
    return oracle_point(case).nlon


def run_oracle(case):
    p = oracle_point(case)
    nmax_shc, mu, r, c, s = case.coeffs
    shc = orc.Shc(nmax_shc, mu, r, c, s)
    return orc.shs_point(p, shc, case.nmax, case.kind)


CASES = gd.shs_cases()


@pytest.mark.parametrize("fam", ["pot", "grad1", "grad2", "guru"])
@pytest.mark.parametrize("subset", ["grid", "custom", "sctr", "dsun"])
def test_oracle_shs_golden(fam, subset):
    cases = [c for c in gd.shs_cases(families=(fam,), subsets=(subset,))]
    if not cases:
        pytest.skip("no golden files for this combination")
    bad = {}
    for case in cases:
        n = check_case(case, run_oracle(case))
        if n:
            bad[case.name] = n
    assert not bad, bad


@pytest.mark.parametrize("g", ["gl", "dh1", "dh2"])
def test_oracle_crd_golden(g):
    """crd_point_gl/dh1/dh2 nodes, weights, longitudes, radii
    (tests/check_crd_point_quad.c:35-95)."""
    G = gd.golden("double")
    eps = 10.0 * gd.THRESHOLD
    for nmax in range(11):
        for d in range(2):
            r = 1.0 + 1000.0 * d
            if g == "gl":
                p = orc.gl(nmax, r)
            else:
                p = orc.dh(nmax, r, orc.DH1 if g == "dh1" else orc.DH2)
            key = "crd_nx%d_dr%d_%s_" % (nmax, d, g)
            assert gd.mismatches(p.lat, G[key + "lat"], eps) == 0
            assert gd.mismatches(p.lon, G[key + "lon"], eps) == 0
            assert gd.mismatches(p.r, G[key + "r"], eps) == 0
            assert gd.mismatches(p.w, G[key + "w"], eps) == 0
            assert gd.nearly_equal(np.sum(p.w), 2.0, eps)


def test_oracle_quad_crd_golden():
    """The binary128 oracle's GL/DH nodes against CHarm's quad golden files
    to 1e-30 relative."""
    Q = gd.golden("quad")
    for nmax in range(11):
        for g in ("gl", "dh1", "dh2"):
            if g == "gl":
                lat, w = orc.gl(nmax, 0.0, prec="q")
            else:
                lat, w = orc.dh(nmax, 0.0,
                                orc.DH1 if g == "dh1" else orc.DH2, prec="q")
            for nm, arr in (("lat", lat), ("w", w)):
                ref = Q["crd_nx%d_dr0_%s_%s" % (nmax, g, nm)]
                hi, lo = orc.q_to_dd(arr)
                diff = (hi - ref[0]) + (lo - ref[1])
                scale = np.maximum(np.abs(ref[0]), 1e-300)
                assert np.all(np.abs(diff) / scale <= 1e-30), (nmax, g, nm)


def test_oracle_quad_shs_golden():
    """The binary128 oracle reproduces CHarm's quad golden files of grid and
    dynamical-switching potential synthesis to 1e-28 relative."""
    Q = gd.golden("quad")
    e = gd.egm96()
    nmax_shc = int(e["nmax"])
    mu_q = orc.q_from_dd(e["mu_q"][:1], e["mu_q"][1:])
    r_q = orc.q_from_dd(e["r_q"][:1], e["r_q"][1:])
    c_q = orc.q_from_dd(e["c_q"][0], e["c_q"][1])
    s_q = orc.q_from_dd(e["s_q"][0], e["s_q"][1])
    # low-degree overrides: tests/parameters.h:223-230 defines them as double
    # literals, so the quad build sees the double values cast to binary128
    for (n, m, which, v) in ((0, 0, "c", 0.0000001), (1, 0, "c", 0.0000002),
                             (1, 1, "c", 0.0000003), (1, 1, "s", 0.0000004)):
        i = gd.tri_index(nmax_shc, n, m)
        (c_q if which == "c" else s_q)[i] = orc.q_from_dd(np.array([v]))[0]
    worst = 0.0
    for nmax in range(5):
        for d in range(2):
            rg = orc.q_arith("+", r_q, orc.q_from_dd(np.array([1000.0 * d])))
            for g, t in (("gl", orc.GL), ("dh1", orc.DH1), ("dh2", orc.DH2)):
                hi, lo = orc.shs_point_quad_grid(t, nmax, nmax_shc, mu_q, r_q,
                                                 c_q, s_q, rg)
                ref = Q["shs_p_nx%d_dr%d_fft1_%s" % (nmax, d, g)]
                diff = (hi - ref[0]) + (lo - ref[1])
                rel = np.max(np.abs(diff) / np.abs(ref[0]))
                worst = max(worst, rel)
    assert worst <= 1e-28, worst


@pytest.mark.slow
def test_oracle_quad_dsun_golden():
    """Dynamical switching at nmax 150..154 in binary128 (X-numbers with
    radix 2^16000) against CHarm's quad golden files."""
    Q = gd.golden("quad")
    worst = 0.0
    for nmax in (150, 154):
        _, mu, r, c, s = gd.ds_coefficients(nmax)
        # 1/(n+1) in binary128 (check_shs_point_all.c:776-790)
        deg = np.concatenate([np.arange(m, nmax + 1) for m in range(nmax + 1)])
        one = orc.q_from_dd(np.ones(len(c)))
        cq = orc.q_arith("/", one, orc.q_from_dd(deg + 1.0))
        sq = cq.copy()
        sq[s == 0] = 0.0
        for sflag in (0, 1):
            for d in (0, 1):
                shift = None
                if sflag == 0:
                    # BREAK_SYMM is a double literal too (parameters.h:238)
                    shift = orc.q_from_dd(np.array([0.001]))
                rq = orc.q_from_dd(np.array([1.0 + 1000.0 * d]))
                hi, lo = orc.shs_point_quad_grid(
                    orc.GL, nmax, nmax, orc.q_from_dd(np.array([1.0])),
                    orc.q_from_dd(np.array([1.0])), cq, sq, rq,
                    nlon_override=1, lat_shift=shift)
                ref = Q["shs_p_nx%d_n0_dr%d_fft0_s%d_dsun" % (nmax, d, sflag)]
                diff = (hi - ref[0]) + (lo - ref[1])
                nz = ref[0] != 0
                rel = np.max(np.abs(diff[nz]) / np.abs(ref[0][nz]))
                worst = max(worst, rel)
    assert worst <= 1e-26, worst


def _q_dec(sv):
    from decimal import Decimal, getcontext
    getcontext().prec = 60
    d = Decimal(sv)
    hi = float(d)
    return orc.q_from_dd(np.array([hi]), np.array([float(d - Decimal(hi))]))
