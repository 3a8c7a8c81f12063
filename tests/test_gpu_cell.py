"""Block means in cells on the GPU (charm_shs_cell / charm_sha_cell through
libcharm.so) against CHarm's golden vectors (tests/check_shs_cell.c,
tests/check_sha_cell.c, with CHarm's tolerances), against the oracle's
restatement of CHarm's cell kernels at higher degrees, and against CHarm's
own build where oracle/_ref has it.

Tolerances are relative RMS errors between double-precision evaluations of
the same recurrences (different summation order and fused multiply-adds)."""
import numpy as np
import pytest

import golden_data as gd
from charm_b200.workloads import GM, R_EARTH, coef_rel_rms, kaula, rel_rms
from oracle import charm_ref, orc

pytestmark = pytest.mark.gpu

TOL = 1e-13


@pytest.fixture(scope="module")
def cb():
    import charm_b200
    return charm_b200


def gpu_cell(cb, ctype, cell):
    ctor = cb.CellGrid if ctype == gd.CELL_GRID else cb.CellSctr
    return ctor(*cell)


def test_shs_cell_golden(cb):
    """Every cell-synthesis case of CHarm's test-suite: custom cell grids
    (sums at the cell centres when the cells span pi, FFT when 2 pi;
    symmetric and not) and scattered cells, nmax 0..4."""
    G = gd.golden("double")
    nmax, mu, r, c, s = gd.test_coefficients()
    shc = cb.Shc(nmax, mu, r, c, s)
    bad = []
    for case in gd.shs_cell_cases():
        f = cb.shs_cell(gpu_cell(cb, case.ctype, case.cell), shc, case.nmax)
        if gd.mismatches(f, G[case.golden_names[0]], case.eps):
            bad.append(case.name)
    assert not bad, bad[:10]


def test_sha_cell_golden(cb):
    """Synthesis then approximate-quadrature analysis on the cell grids of
    tests/check_sha_cell.c, against the golden C and S triangles."""
    G = gd.golden("double")
    nmax, mu, r, c, s = gd.test_coefficients()
    shc = cb.Shc(nmax, mu, r, c, s)
    bad = []
    for case in gd.sha_cell_cases():
        cl = gpu_cell(cb, case.ctype, case.cell)
        f = cb.shs_cell(cl, shc, case.nmax)
        out = cb.sha_cell(cl, f, case.nmax, mu=mu, r=r)
        if (gd.mismatches(out.c, G[case.golden_names[0]], case.eps) or
                gd.mismatches(out.s, G[case.golden_names[1]], case.eps)):
            bad.append(case.name)
    assert not bad, bad[:10]


def sphere_cells(nlat, nlon, r):
    lat_e = np.linspace(np.pi / 2, -np.pi / 2, nlat + 1)
    lat_e[0], lat_e[-1] = np.pi / 2, -np.pi / 2
    lon_e = np.arange(nlon + 1) * (2.0 * np.pi / nlon)
    return (lat_e[1:], lat_e[:-1], lon_e[:-1], lon_e[1:], np.full(nlat, r))


@pytest.mark.parametrize("N,nlat,nlon,dr", [
    (360, 361, 722, 0.0),       # odd rows: a middle row astride the equator
    (360, 362, 724, 3000.0),    # above the sphere
    (720, 721, 1442, 0.0),
    # 513 cell-row pairs: two adjacent pairs per lane sharing a boundary
    (1024, 1025, 2050, 3000.0),
    (1024, 1026, 2052, 0.0),
])
def test_cell_grid_sphere_vs_oracle(cb, N, nlat, nlon, dr):
    """Whole-sphere cell grids (FFT synthesis, approximate-quadrature
    analysis): synthesis and analysis against the oracle."""
    c, s = kaula(N, 9100 + N)
    args = sphere_cells(nlat, nlon, R_EARTH + dr)
    f = cb.shs_cell(cb.CellGrid(*args), cb.Shc(N, GM, R_EARTH, c, s), N)
    co = orc.Cell(orc.CELL_GRID, *args)
    fo = orc.shs_cell(co, orc.Shc(N, GM, R_EARTH, c, s), N)
    assert rel_rms(f, fo) <= TOL
    f00 = GM / R_EARTH
    assert rel_rms(np.ravel(f) - f00, fo - f00) <= 1e-9
    out = cb.sha_cell(cb.CellGrid(*args), f, N, mu=GM, r=R_EARTH)
    ref = orc.sha_cell(co, f, N, GM, R_EARTH)
    assert coef_rel_rms(out.c, out.s, ref.c, ref.s) <= TOL


def test_cell_analysis_two_pairs_per_lane(cb):
    """1025 rows (513 cell-row pairs: two pairs per lane, adjacent ones,
    whose common boundary's recurrence is carried once; the analysis
    requires aligned rows, latmin[i] == latmax[i + 1]) against the oracle's
    analysis of the same block means."""
    N = 1024
    c, s = kaula(N, 9400)
    lat_e = np.linspace(np.pi / 2, -np.pi / 2, 1026)
    latmin, latmax = lat_e[1:].copy(), lat_e[:-1].copy()
    lon_e = np.arange(2051) * (2.0 * np.pi / 2050)
    args = (latmin, latmax, lon_e[:-1], lon_e[1:], np.full(1025, R_EARTH))
    cl = cb.CellGrid(*args)
    f = cb.shs_cell(cl, cb.Shc(N, GM, R_EARTH, c, s), N)
    out = cb.sha_cell(cl, f, N, mu=GM, r=R_EARTH)
    ref = orc.sha_cell(orc.Cell(orc.CELL_GRID, *args), f, N, GM, R_EARTH)
    assert coef_rel_rms(out.c, out.s, ref.c, ref.s) <= TOL


def test_cell_grid_odd_rows_analysis(cb):
    """An odd number of cells per parallel (2 nmax + 1, the least the
    analysis accepts): rows transformed by the direct DFT."""
    N = 100
    c, s = kaula(N, 9300)
    args = sphere_cells(N + 1, 2 * N + 1, R_EARTH)
    cl = cb.CellGrid(*args)
    co = orc.Cell(orc.CELL_GRID, *args)
    f = orc.shs_cell(co, orc.Shc(N, GM, R_EARTH, c, s), N)
    out = cb.sha_cell(cl, f, N, mu=GM, r=R_EARTH)
    ref = orc.sha_cell(co, f, N, GM, R_EARTH)
    assert coef_rel_rms(out.c, out.s, ref.c, ref.s) <= TOL


@pytest.mark.parametrize("N", [200, 1500])
def test_cell_grid_regional_vs_oracle(cb, N):
    """A regional, non-symmetric grid of cells (longitudes span 40 degrees:
    sums at the cell centres, the role of CHarm's PSLR path) with radii
    varying by row."""
    c, s = kaula(N, 9200 + N)
    lat_e = np.deg2rad(np.linspace(62.0, 21.0, 42))
    lon_e = np.deg2rad(np.linspace(5.0, 45.0, 161))
    r = R_EARTH + np.linspace(0.0, 4000.0, 41)
    args = (lat_e[1:], lat_e[:-1], lon_e[:-1], lon_e[1:], r)
    f = cb.shs_cell(cb.CellGrid(*args), cb.Shc(N, GM, R_EARTH, c, s), N)
    fo = orc.shs_cell(orc.Cell(orc.CELL_GRID, *args),
                      orc.Shc(N, GM, R_EARTH, c, s), N)
    assert rel_rms(f, fo) <= TOL
    f00 = GM / R_EARTH
    assert rel_rms(np.ravel(f) - f00, fo - f00) <= 1e-9


def test_cell_sctr_vs_oracle(cb):
    """Scattered cells of random size, position and height, nmax 300."""
    N = 300
    c, s = kaula(N, 9400)
    rng = np.random.default_rng(9401)
    n = 700
    lat0 = np.arcsin(rng.uniform(-0.99, 0.99, n))
    dlat = np.deg2rad(rng.uniform(0.05, 2.0, n))
    lon0 = rng.uniform(0.0, 2.0 * np.pi, n)
    dlon = np.deg2rad(rng.uniform(0.05, 2.0, n))
    args = (lat0 - dlat / 2, lat0 + dlat / 2, lon0, lon0 + dlon,
            R_EARTH + rng.uniform(0.0, 9000.0, n))
    f = cb.shs_cell(cb.CellSctr(*args), cb.Shc(N, GM, R_EARTH, c, s), N)
    fo = orc.shs_cell(orc.Cell(orc.CELL_SCATTERED, *args),
                      orc.Shc(N, GM, R_EARTH, c, s), N)
    assert rel_rms(f, fo) <= TOL


def test_cell_polar_rows_high_degree(cb):
    """Cells touching the poles at nmax 2000: the boundary recurrences start
    far below the double range (the X-number regime of CHarm)."""
    N = 2000
    c, s = kaula(N, 9500)
    lat_e = np.deg2rad(np.array([90.0, 89.99, 89.9, 89.0, 88.0, 80.0]))
    args = (lat_e[1:], lat_e[:-1], np.array([0.0]), np.array([0.01]),
            np.full(5, R_EARTH))
    f = cb.shs_cell(cb.CellGrid(*args), cb.Shc(N, GM, R_EARTH, c, s), N)
    fo = orc.shs_cell(orc.Cell(orc.CELL_GRID, *args),
                      orc.Shc(N, GM, R_EARTH, c, s), N)
    assert rel_rms(f, fo) <= TOL
    assert np.max(np.abs(np.ravel(f) - fo) / np.abs(fo)) <= 1e-12


@pytest.mark.skipif(not charm_ref.available("d"),
                    reason="oracle/_ref has no double CHarm build")
def test_cells_vs_charm(cb):
    """Against CHarm's own charm_shs_cell / charm_sha_cell at nmax 360."""
    C = charm_ref.Charm("d")
    N = 360
    c, s = kaula(N, 9600)
    args = sphere_cells(362, 724, R_EARTH + 1000.0)
    cc = C.cell(orc.CELL_GRID, *args)
    fr = C.shs_cell(cc, C.shc(N, GM, R_EARTH, c, s), N, 362 * 724)
    f = cb.shs_cell(cb.CellGrid(*args), cb.Shc(N, GM, R_EARTH, c, s), N)
    assert rel_rms(f, fr) <= TOL
    cr, sr = C.sha_cell(cc, fr, N, GM, R_EARTH)
    out = cb.sha_cell(cb.CellGrid(*args), fr, N, mu=GM, r=R_EARTH)
    assert coef_rel_rms(out.c, out.s, cr, sr) <= TOL


def test_cell_device_entry_points(cb):
    """charm_b200_shs_cell_dev / charm_b200_sha_cell_dev give the host
    entry points' results bit for bit."""
    import ctypes as ct
    import torch
    from charm_b200._lib import _libcharm as L
    N = 200
    c, s = kaula(N, 9700)
    args = sphere_cells(201, 402, R_EARTH)
    cl = cb.CellGrid(*args)
    f_host = cb.shs_cell(cl, cb.Shc(N, GM, R_EARTH, c, s), N)
    P = ct.c_void_p
    L.charm_b200_shs_cell_dev.argtypes = [P, ct.c_ulong, ct.c_double,
                                          ct.c_double, P, P, ct.c_ulong, P, P]
    L.charm_b200_sha_cell_dev.argtypes = [P, P, ct.c_ulong, ct.c_double,
                                          ct.c_double, ct.c_ulong, P, P, P]
    dc = torch.tensor(c, device="cuda")
    ds = torch.tensor(s, device="cuda")
    df = torch.empty(f_host.size, dtype=torch.float64, device="cuda")
    err = L.charm_err_init()
    L.charm_b200_shs_cell_dev(ct.cast(cl._Cell, P), N, GM, R_EARTH,
                              dc.data_ptr(), ds.data_ptr(), N, df.data_ptr(),
                              ct.cast(err, P))
    assert L.charm_err_isempty(err)
    assert np.array_equal(df.cpu().numpy(), np.ravel(f_host))
    oc = torch.empty_like(dc)
    os_ = torch.empty_like(ds)
    L.charm_b200_sha_cell_dev(ct.cast(cl._Cell, P), df.data_ptr(), N, GM,
                              R_EARTH, N, oc.data_ptr(), os_.data_ptr(),
                              ct.cast(err, P))
    assert L.charm_err_isempty(err)
    L.charm_err_free(err)
    ref = cb.sha_cell(cl, f_host, N, mu=GM, r=R_EARTH)
    assert np.array_equal(oc.cpu().numpy(), ref.c)
    assert np.array_equal(os_.cpu().numpy(), ref.s)
