"""CHarm 0.4.9 itself, compiled from its own sources into oracle/_ref
(oracle/build_ref.py, FFTW replaced by oracle/fftw_shim), pinned the way
CHarm pins itself: its FFT shim against numpy's FFT, its double build
against the golden files of its own test-suite with its own tolerances
(tests/check_shs_point_all.c), its quad build against the quad golden
files; then the oracle's restatement (oracle/orc.c) against it at degrees
the golden files do not reach.  CPU only."""
import ctypes as ct

import numpy as np
import pytest

import golden_data as gd
from oracle import charm_ref, orc

needs_d = pytest.mark.skipif(not charm_ref.available("d"),
                             reason="oracle/_ref has no double CHarm build")
needs_q = pytest.mark.skipif(not charm_ref.available("q"),
                             reason="oracle/_ref has no quad CHarm build")

GM = 3.986004418e14
R = 6378136.3


@pytest.fixture(scope="module")
def C():
    return charm_ref.Charm("d")


@needs_d
def test_fft_shim_against_numpy(C):
    """FFTW semantics of the shim: unnormalised r2c, and c2r over the
    Hermitian extension ignoring the imaginary parts of the first and (even
    lengths) last bins; direct radices, generic radices and Bluestein."""
    L = C.L
    vp = ct.c_void_p
    for name in ("fftw_plan_dft_r2c_1d", "fftw_plan_dft_c2r_1d"):
        getattr(L, name).argtypes = [ct.c_int, vp, vp, ct.c_uint]
        getattr(L, name).restype = vp
    for name in ("fftw_execute_dft_r2c", "fftw_execute_dft_c2r"):
        getattr(L, name).argtypes = [vp, vp, vp]
    L.fftw_destroy_plan.argtypes = [vp]
    rng = np.random.default_rng(7)
    lengths = list(range(1, 66)) + [97, 128, 313, 626, 722, 4382, 8764, 21602]
    for n in lengths:
        x = rng.standard_normal(n)
        X = np.zeros(n // 2 + 1, np.complex128)
        p = L.fftw_plan_dft_r2c_1d(n, None, None, 1 << 6)
        L.fftw_execute_dft_r2c(p, x.ctypes.data, X.ctypes.data)
        L.fftw_destroy_plan(p)
        ref = np.fft.rfft(x)
        assert np.max(np.abs(X - ref)) <= 1e-13 * np.max(np.abs(ref)), n
        Y = rng.standard_normal(n // 2 + 1) + 1j * rng.standard_normal(n // 2 + 1)
        y = np.zeros(n)
        q = L.fftw_plan_dft_c2r_1d(n, None, None, 1 << 6)
        Yin = Y.copy()          # c2r may overwrite its input
        L.fftw_execute_dft_c2r(q, Yin.ctypes.data, y.ctypes.data)
        L.fftw_destroy_plan(q)
        Z = Y.copy()
        Z[0] = Z[0].real
        if n % 2 == 0:
            Z[-1] = Z[-1].real
        yref = np.fft.irfft(Z, n) * n
        assert np.max(np.abs(y - yref)) <= 1e-13 * np.max(np.abs(yref)), n


def ref_point(C, case):
    if case.grid is not None:
        g, nmax, r = case.grid
        kind = {"gl": charm_ref.GL, "dh1": charm_ref.DH1, "dh2": charm_ref.DH2}[g]
        p, lat, lon, w = C.grid(kind, nmax, r)
        # the dynamical-switching cases keep the grid type, use the first
        # meridian only and move the first latitude, as
        # tests/check_shs_point_all.c:840-870 does to the structure
        if case.nlon_override is not None:
            p.ptr.contents.nlon = case.nlon_override
        if case.lat0_shift:
            lat[0] -= case.lat0_shift
        pt = p.ptr.contents
        return p, np.array(lat[:pt.nlat]), int(pt.nlon), int(pt.nlat * pt.nlon)
    if case.ptype == gd.SCATTERED:
        p = C.point(charm_ref.SCATTERED, case.lat, case.lon, case.r)
        return p, np.asarray(case.lat), 1, len(case.lat)
    p = C.point(charm_ref.GRID, case.lat, case.lon, case.r)
    return p, np.asarray(case.lat), len(case.lon), len(case.lat) * len(case.lon)


def run_ref(C, case):
    p, lat, nlon, npoint = ref_point(C, case)
    nmax_shc, mu, r, c, s = case.coeffs
    shc = C.shc(nmax_shc, mu, r, c, s)
    if case.kind == "pot":
        out = [C.shs_point(p, shc, case.nmax, npoint)]
    elif case.kind == "grad1":
        out = C.shs_point_grad(p, shc, case.nmax, npoint, 1)
    elif case.kind == "grad2":
        out = C.shs_point_grad(p, shc, case.nmax, npoint, 2)
    else:
        dr, dlat, dlon = case.kind
        out = [C.shs_point_guru(p, shc, case.nmax, npoint, dr, dlat, dlon)]
    return lat, nlon, out


@needs_d
@pytest.mark.parametrize("fam", ["pot", "grad1", "grad2", "guru"])
@pytest.mark.parametrize("subset", ["grid", "custom", "sctr", "dsun"])
def test_charm_ref_golden(C, fam, subset):
    """The double build of CHarm reproduces its own golden files."""
    cases = gd.shs_cases(families=(fam,), subsets=(subset,))
    if not cases:
        pytest.skip("no golden files for this combination")
    G = gd.golden("double")
    bad = {}
    for case in cases:
        lat, nlon, out = run_ref(C, case)
        n = 0
        for j, (nm, f) in enumerate(zip(case.golden_names, out)):
            if gd.singular_component(case.kind, j):
                f = gd.zero_singular_rows(case.ptype, lat, nlon, f)
            n += gd.mismatches(f, G[nm], case.eps)
        if n:
            bad[case.name] = n
    assert not bad, bad


@needs_d
def test_charm_ref_crd_golden(C):
    """CHarm's GL / DH1 / DH2 nodes and weights (check_crd_point_quad.c)."""
    G = gd.golden("double")
    eps = 10.0 * gd.THRESHOLD
    for nmax in range(11):
        for g, kind in (("gl", charm_ref.GL), ("dh1", charm_ref.DH1),
                        ("dh2", charm_ref.DH2)):
            p, lat, lon, w = C.grid(kind, nmax, 1.0)
            key = "crd_nx%d_dr0_%s_" % (nmax, g)
            assert gd.mismatches(lat, G[key + "lat"], eps) == 0
            assert gd.mismatches(lon, G[key + "lon"], eps) == 0
            assert gd.mismatches(w, G[key + "w"], eps) == 0


@needs_d
def test_oracle_port_against_charm_nmax360(C):
    """The oracle's restatement against CHarm itself on the nmax 360 GL
    grid at r = R and above it: synthesis of the potential and grad1 on
    sampled rows, and the analysis of CHarm's own grid."""
    from charm_b200.workloads import coef_rel_rms, kaula, rel_rms
    N = 360
    c, s = kaula(N, 1000)
    for r in (R, R + 5000.0):
        p, lat, lon, w = C.grid(charm_ref.GL, N, r)
        shc = C.shc(N, GM, R, c, s)
        f = C.shs_point(p, shc, N, lat.size * lon.size).reshape(lat.size, -1)
        po = orc.gl(N, r)
        fo = orc.shs_point(po, orc.Shc(N, GM, R, c, s), N)[0]
        assert rel_rms(fo, f) <= 1e-14
        g = C.shs_point_grad(p, shc, N, lat.size * lon.size, 1)
        go = orc.shs_point(po, orc.Shc(N, GM, R, c, s), N, "grad1")
        for a, b in zip(go, g):
            assert rel_rms(np.ravel(a), b) <= 1e-13
    p, lat, lon, w = C.grid(charm_ref.GL, N, R)
    shc = C.shc(N, GM, R, c, s)
    f = C.shs_point(p, shc, N, lat.size * lon.size)
    cr, sr = C.sha_point(p, f, N, GM, R)
    ref = orc.sha_point(orc.gl(N, R), f.reshape(lat.size, -1), N, GM, R)
    # C and S together: S alone has no degree-0 term, so its own RMS would
    # measure the rounding noise of the C00-dominated grid values instead
    assert coef_rel_rms(ref.c, ref.s, cr, sr) <= 5e-14


@needs_d
def test_oracle_cells_against_charm(C):
    """The oracle's cell synthesis and analysis against CHarm's own
    charm_shs_cell / charm_sha_cell at nmax 120: a 1-degree cell grid of
    the whole sphere above it (FFT synthesis, approximate-quadrature
    analysis), a regional non-symmetric grid (PSLR path) and scattered
    cells of random size and height."""
    from charm_b200.workloads import coef_rel_rms, kaula, rel_rms
    N = 120
    c, s = kaula(N, 1200)
    shc_c = C.shc(N, GM, R, c, s)
    shc_o = orc.Shc(N, GM, R, c, s)
    # whole sphere, 180 x 360 one-degree cells at r = R + 3 km
    lat_e = np.deg2rad(np.linspace(90.0, -90.0, 181))
    lon_e = np.deg2rad(np.linspace(0.0, 360.0, 361))
    lon_e[-1] = 2.0 * np.pi
    args = (lat_e[1:], lat_e[:-1], lon_e[:-1], lon_e[1:], np.full(180, R + 3e3))
    cc = C.cell(orc.CELL_GRID, *args)
    co = orc.Cell(orc.CELL_GRID, *args)
    f = C.shs_cell(cc, shc_c, N, 180 * 360)
    fo = orc.shs_cell(co, shc_o, N)
    assert rel_rms(fo, f) <= 1e-14
    cr, sr = C.sha_cell(cc, f, N, GM, R)
    out = orc.sha_cell(co, f, N, GM, R)
    assert coef_rel_rms(out.c, out.s, cr, sr) <= 1e-13
    # regional grid (longitudes span 60 degrees: no FFT), not symmetric
    lat_e = np.deg2rad(np.linspace(50.0, 10.0, 41))
    lon_e = np.deg2rad(np.linspace(0.0, 60.0, 121))
    args = (lat_e[1:], lat_e[:-1], lon_e[:-1], lon_e[1:], np.full(40, R))
    f = C.shs_cell(C.cell(orc.CELL_GRID, *args), shc_c, N, 40 * 120)
    fo = orc.shs_cell(orc.Cell(orc.CELL_GRID, *args), shc_o, N)
    assert rel_rms(fo, f) <= 1e-14
    # scattered cells
    rng = np.random.default_rng(77)
    n = 400
    lat0 = np.arcsin(rng.uniform(-0.98, 0.98, n))
    dlat = np.deg2rad(rng.uniform(0.1, 2.0, n))
    lon0 = rng.uniform(0.0, 2.0 * np.pi, n)
    dlon = np.deg2rad(rng.uniform(0.1, 2.0, n))
    args = (lat0 - dlat / 2, lat0 + dlat / 2, lon0, lon0 + dlon,
            R + rng.uniform(0.0, 9000.0, n))
    f = C.shs_cell(C.cell(orc.CELL_SCATTERED, *args), shc_c, N, n)
    fo = orc.shs_cell(orc.Cell(orc.CELL_SCATTERED, *args), shc_o, N)
    assert rel_rms(fo, f) <= 1e-14


@needs_q
def test_charm_quad_golden():
    """CHarm's quad build against its quad golden files of grid synthesis
    (nmax 0..4, GL / DH1 / DH2 at r = R and R + 1000 m) to 1e-28."""
    Q = charm_ref.CharmQ()
    QG = gd.golden("quad")
    e = gd.egm96()
    nmax_shc = int(e["nmax"])
    c_hi, c_lo = e["c_q"][0].copy(), e["c_q"][1].copy()
    s_hi, s_lo = e["s_q"][0].copy(), e["s_q"][1].copy()
    for (n, m, which, v) in ((0, 0, "c", 0.0000001), (1, 0, "c", 0.0000002),
                             (1, 1, "c", 0.0000003), (1, 1, "s", 0.0000004)):
        i = gd.tri_index(nmax_shc, n, m)
        if which == "c":
            c_hi[i], c_lo[i] = v, 0.0
        else:
            s_hi[i], s_lo[i] = v, 0.0
    mu_q = orc.q_from_dd(e["mu_q"][:1], e["mu_q"][1:])
    r_q = orc.q_from_dd(e["r_q"][:1], e["r_q"][1:])
    worst = 0.0
    for nmax in range(5):
        for d in range(2):
            for g, kind in (("gl", orc.GL), ("dh1", orc.DH1), ("dh2", orc.DH2)):
                # the nodes from the oracle's binary128 GL / DH generators
                # (pinned to CHarm's quad crd files by test_oracle_golden)
                if g == "gl":
                    latq, _ = orc.gl(nmax, 0.0, prec="q")
                else:
                    latq, _ = orc.dh(nmax, 0.0, kind, prec="q")
                nlon = {"gl": 2 * nmax + 2, "dh1": 2 * nmax + 2,
                        "dh2": 4 * nmax + 4}[g]
                L = nmax + 1
                piq = orc.q_from_dd(np.array([np.pi]),
                                    np.array([1.2246467991473532e-16]))
                den = float(L if g != "dh2" else 2 * L)
                step = orc.q_arith("/", piq, orc.q_from_dd(np.array([den])))
                lonq = orc.q_arith("*", orc.q_from_dd(
                    np.arange(nlon, dtype=np.float64)), step)
                rg = orc.q_arith("+", r_q, orc.q_from_dd(np.array([1000.0 * d])))
                nlat = latq.shape[0]
                rq = np.repeat(rg, nlat, axis=0)
                pnt = Q.point_raw(charm_ref.GRID, latq, lonq, rq)
                shc = Q.shc(nmax_shc, 0.0, 0.0, c_hi, s_hi, c_lo, s_lo)
                shc.keep[4].mu = charm_ref._F128.from_buffer_copy(mu_q.tobytes())
                shc.keep[4].r = charm_ref._F128.from_buffer_copy(r_q.tobytes())
                hi, lo = Q.shs_point(pnt, shc, nmax, nlat * nlon)
                ref = QG["shs_p_nx%d_dr%d_fft1_%s" % (nmax, d, g)]
                diff = (hi - ref[0]) + (lo - ref[1])
                worst = max(worst, np.max(np.abs(diff) / np.abs(ref[0])))
    assert worst <= 1e-28, worst
