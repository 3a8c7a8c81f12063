"""Golden vectors of CHarm's own test-suite and the cases that produce them.

The fixtures under tests/golden/ were packed from CHarm's data/tests by
tests/golden/make_golden.py.  The enumerators below restate the loops of
tests/check_shs_point_all.c (grids :440-530, custom grids :540-648, scattered
points :656-748, dynamical switching :767-907) and
tests/check_crd_point_quad.c, so each case yields the inputs, the golden
array and the tolerance CHarm's own test applies to it.
"""
import os
from dataclasses import dataclass, field
from functools import lru_cache

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")

SCATTERED, GRID, GL, DH1, DH2 = 1, 2, 3, 4, 5
EPS = np.finfo(np.float64).eps
THRESHOLD = 100.0 * EPS
THRESHOLD2 = 100000.0 * EPS
PI = 3.14159265358979323846
PI_2 = 1.57079632679489661923

GRAD1_ELEM = ["_x", "_y", "_z"]
GRAD2_ELEM = ["_xx", "_xy", "_xz", "_yy", "_yz", "_zz"]
# GURU_LOOP order, tests/check_shs_point_all.c:61-77
GURU = [(dr, dlat, dlon) for dr in range(3) for dlat in range(3)
        for dlon in range(3) if dr + dlat + dlon <= 2]


@lru_cache(maxsize=None)
def golden(prec="double"):
    z = np.load(os.path.join(GOLDEN, "charm_golden_%s.npz" % prec))
    names = str(z["names"]).split("\n")
    off = z["offsets"]
    data = z["data"]
    return {n: data[..., off[i]:off[i + 1]] for i, n in enumerate(names)}


@lru_cache(maxsize=None)
def egm96():
    return dict(np.load(os.path.join(GOLDEN, "egm96_degree10.npz")))


def tri_index(nmax, n, m):
    return m * (2 * nmax + 3 - m) // 2 + n - m


def test_coefficients():
    """EGM96 degree 10 with the low-degree overrides of
    tests/modify_low_degree_coefficients.c (values tests/parameters.h:223-230).
    Returns (nmax, mu, r, c, s)."""
    e = egm96()
    nmax = int(e["nmax"])
    c = e["c"].copy()
    s = e["s"].copy()
    c[tri_index(nmax, 0, 0)] = 0.0000001
    c[tri_index(nmax, 1, 0)] = 0.0000002
    c[tri_index(nmax, 1, 1)] = 0.0000003
    s[tri_index(nmax, 1, 1)] = 0.0000004
    return nmax, float(e["mu"]), float(e["r"]), c, s


def ds_coefficients(nmax):
    """Fake coefficients 1/(n+1) of the dynamical-switching tests
    (check_shs_point_all.c:776-790), with mu = r = 1."""
    T = (nmax + 1) * (nmax + 2) // 2
    c = np.zeros(T)
    s = np.zeros(T)
    for m in range(nmax + 1):
        n = np.arange(m, nmax + 1)
        i0 = tri_index(nmax, m, m)
        c[i0:i0 + nmax + 1 - m] = 1.0 / (n + 1.0)
        if m > 0:
            s[i0:i0 + nmax + 1 - m] = 1.0 / (n + 1.0)
    return nmax, 1.0, 1.0, c, s


def generate_point(ptype, nlat, nlon, r, lat_rng, lon_rng):
    """tests/generate_point.c"""
    nlat2 = nlat - 1 if (ptype == GRID and nlat > 1) else nlat
    lat = np.array([PI_2 - (float(l) / float(nlat2)) * lat_rng
                    for l in range(nlat)], dtype=np.float64)
    lon = np.array([(float(l) / float(nlon)) * lon_rng for l in range(nlon)],
                   dtype=np.float64)
    return lat, lon, np.full(nlat, float(r))


def nearly_equal(a, b, eps):
    """Vectorised src/misc/misc_is_nearly_equal.c:20-31."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    aa, ba = np.abs(a), np.abs(b)
    d = np.abs(a - b)
    s = aa + ba
    with np.errstate(divide="ignore", invalid="ignore"):
        rel = d / np.maximum(aa, ba)
    zero = (a == 0.0) | (b == 0.0) | (s == aa) | (s == ba)
    ok = np.where(zero, d <= eps, rel <= eps)
    return (a == b) | ok


def mismatches(f, ref, eps):
    """Number of elements failing CHarm's validate() (tests/validate.c)."""
    f = np.asarray(f, np.float64).reshape(-1)
    ref = np.asarray(ref, np.float64).reshape(-1)
    assert f.size == ref.size, (f.size, ref.size)
    return int(np.sum(~nearly_equal(f, ref, eps)))


def singular_component(kind, j):
    """zeros_for_singularities, check_shs_point_all.c:270-300."""
    if kind == "pot":
        return False
    if kind == "grad1":
        return j != 2
    if kind == "grad2":
        return j != 5
    dr, dlat, dlon = kind
    return dlat > 0 or dlon > 0


def zero_singular_rows(ptype, lat, nlon, f):
    """treat_singularity, check_shs_point_all.c:229-262."""
    lim = PI_2 - 100.0 * abs(THRESHOLD)
    f = np.array(f, np.float64, copy=True).reshape(-1)
    if ptype == SCATTERED:
        f[np.abs(lat) > lim] = 0.0
    else:
        for i in range(len(lat)):
            if abs(lat[i]) > lim:
                f[i * nlon:(i + 1) * nlon] = 0.0
    return f


def elem_names(kind):
    if kind == "pot":
        return [""]
    if kind == "grad1":
        return GRAD1_ELEM
    if kind == "grad2":
        return GRAD2_ELEM
    return ["_guru%d%d%d" % k for k in GURU]


@dataclass
class Case:
    """One synthesis call of CHarm's test-suite."""
    name: str                  # golden file stem of component 0
    ptype: int
    nmax: int
    coeffs: tuple              # (shc_nmax, mu, r, c, s)
    kind: object               # "pot", "grad1", "grad2" or (dr, dlat, dlon)
    grid: tuple = None         # ("gl"|"dh1"|"dh2", nmax, r) for quad grids
    lat: np.ndarray = None     # custom grids and scattered points
    lon: np.ndarray = None
    r: np.ndarray = None
    nlon_override: int = None  # dsun: first meridian only
    lat0_shift: float = 0.0    # dsun / custom: first latitude moved
    golden_names: list = field(default_factory=list)
    eps: float = 0.0


def _kinds(family):
    return {"pot": ["pot"], "grad1": ["grad1"], "grad2": ["grad2"],
            "guru": [k for k in GURU]}[family]


def shs_cases(families=("pot", "grad1", "grad2", "guru"), subsets=(
        "grid", "custom", "sctr", "dsun")):
    """Every point-synthesis case of CHarm's test-suite that has golden
    files.  Guru cases are emitted one derivative at a time."""
    G = golden("double")
    coeffs = test_coefficients()
    out = []
    for fam in families:
        grad = fam in ("grad1", "grad2")
        gfam = fam != "pot"
        # GL/DH grids, check_shs_point_all.c:440-530
        if "grid" in subsets:
            grids = ["gl", "dh1", "dh2"] if fam == "pot" else ["gl"]
            for g in grids:
                for nmax in range(5):
                    for d in range(2):
                        r = coeffs[2] + 1000.0 * d
                        if fam == "guru":
                            for gi, k in enumerate(GURU):
                                nm = "shs_p_nx%d_dr%d_fft1_%s_guru%d%d%d" % (
                                    nmax, d, g, *k)
                                out.append(Case(nm, {"gl": GL, "dh1": DH1,
                                                     "dh2": DH2}[g], nmax,
                                                coeffs, k, grid=(g, nmax, r),
                                                golden_names=[nm],
                                                eps=1000.0 * THRESHOLD))
                            continue
                        names = ["shs_p_nx%d_dr%d_fft1_%s%s" % (nmax, d, g, e)
                                 for e in elem_names(fam)]
                        out.append(Case(names[0], {"gl": GL, "dh1": DH1,
                                                   "dh2": DH2}[g], nmax,
                                        coeffs, fam, grid=(g, nmax, r),
                                        golden_names=names,
                                        eps=(1000.0 if gfam else 10.0)
                                        * THRESHOLD))
        # custom grids, :540-648 (not for guru)
        if "custom" in subsets and fam != "guru":
            nlats = [1, 1, 3, 10]
            nlons = [1, 2, 8, 22]
            for nmax in range(5):
                for i in range(4):
                    for fft in range(2):
                        if fft == 1 and ((nlons[i] - 1) // 2 < nmax
                                         or nlons[i] < 2):
                            continue
                        for s in range(2):
                            if nlats[i] == 1 and s == 1:
                                continue
                            for d in range(2):
                                r = coeffs[2] + 1000.0 * d
                                lat, lon, rr = generate_point(
                                    GRID, nlats[i], nlons[i], r, PI,
                                    PI if fft == 0 else 2.0 * PI)
                                if s == 0:
                                    lat[0] -= 0.001
                                names = ["shs_p_nx%d_n%d_dr%d_fft%d_s%d%s" % (
                                    nmax, i, d, fft, s, e)
                                    for e in elem_names(fam)]
                                if names[0] not in G:
                                    continue
                                out.append(Case(
                                    names[0], GRID, nmax, coeffs, fam,
                                    lat=lat, lon=lon, r=rr,
                                    golden_names=names,
                                    eps=(1000.0 * THRESHOLD2) if gfam else
                                    (100.0 * THRESHOLD)))
        # scattered points, :656-748
        if "sctr" in subsets:
            nlats = [1, 2, 3, 4, 5, 6, 7, 8, 9, 20, 30, 31]
            if fam == "guru":
                loops = [(4, 11, 1)]
            else:
                loops = [(nmax, i, d) for nmax in range(5) for i in range(12)
                         for d in range(2)]
            for nmax, i, d in loops:
                r = coeffs[2] + 1000.0 * d
                lat, lon, rr = generate_point(SCATTERED, nlats[i], nlats[i],
                                              r, PI, 2.0 * PI)
                if fam == "guru":
                    for k in GURU:
                        nm = "shs_p_nx%d_n%d_dr%d_sctr_guru%d%d%d" % (
                            nmax, i, d, *k)
                        out.append(Case(nm, SCATTERED, nmax, coeffs, k,
                                        lat=lat, lon=lon, r=rr,
                                        golden_names=[nm],
                                        eps=1000.0 * THRESHOLD))
                    continue
                names = ["shs_p_nx%d_n%d_dr%d_sctr%s" % (nmax, i, d, e)
                         for e in elem_names(fam)]
                out.append(Case(names[0], SCATTERED, nmax, coeffs, fam,
                                lat=lat, lon=lon, r=rr, golden_names=names,
                                eps=(1000.0 if gfam else 10.0) * THRESHOLD))
        # dynamical switching and loop unrolling, :767-907 (not for guru)
        if "dsun" in subsets and fam != "guru":
            for nmax in range(150, 155):
                ds = ds_coefficients(nmax)
                for i in range(4):
                    for s in range(2):
                        for d in range(2):
                            r = 1.0 + 1000.0 * d
                            names = [
                                "shs_p_nx%d_n%d_dr%d_fft0_s%d_dsun%s" % (
                                    nmax, i, d, s, e) for e in elem_names(fam)]
                            eps = {"pot": 1.0, "grad1": 10.0,
                                   "grad2": 1000.0}[fam] * THRESHOLD2
                            out.append(Case(names[0], GL, nmax, ds, fam,
                                            grid=("gl", nmax, r),
                                            nlon_override=1,
                                            lat0_shift=0.001 if s == 0 else 0.0,
                                            golden_names=names, eps=eps))
    return out


# ---------------------------------------------------------------------------
# Cells (block-mean values)
# ---------------------------------------------------------------------------
CELL_GRID, CELL_SCATTERED = -2, -1


def generate_cell(nlat, nlon, r, lat_rng, lon_rng):
    """tests/generate_cell.c:18-56 -> (latmin, latmax, lonmin, lonmax, r)."""
    l = np.arange(nlat, dtype=np.float64)
    latmin = PI_2 - ((l + 1.0) / float(nlat)) * lat_rng
    latmax = PI_2 - (l / float(nlat)) * lat_rng
    k = np.arange(nlon, dtype=np.float64)
    lonmin = (k / float(nlon)) * lon_rng
    lonmax = ((k + 1.0) / float(nlon)) * lon_rng
    return latmin, latmax, lonmin, lonmax, np.full(nlat, float(r))


@dataclass
class CellCase:
    """One cell synthesis (or synthesis + analysis) of CHarm's test-suite."""
    name: str
    ctype: int
    nmax: int
    cell: tuple                # (latmin, latmax, lonmin, lonmax, r)
    golden_names: list = field(default_factory=list)
    eps: float = 0.0


def shs_cell_cases():
    """tests/check_shs_cell.c:50-185: custom cell grids (PSLR when the
    cells span pi in longitude, FFT when 2 pi; symmetric and with the first
    cell moved by 0.001) and scattered cells, nmax 0..4, r = R and R + 1 km;
    tolerance threshold2."""
    out = []
    R = test_coefficients()[2]
    nlats = [1, 1, 3, 10]
    nlons = [1, 2, 8, 22]
    for nmax in range(5):
        for i in range(4):
            for fft in range(2):
                if fft == 1 and ((nlons[i] - 1) // 2 < nmax or nlons[i] < 2):
                    continue
                for s in range(2):
                    if nlats[i] == 1 and s == 1:
                        continue
                    for d in range(2):
                        cl = generate_cell(nlats[i], nlons[i], R + 1000.0 * d,
                                           PI, PI if fft == 0 else 2.0 * PI)
                        if s == 0:
                            cl[1][0] -= 0.001
                        nm = "shs_c_nx%d_n%d_dr%d_fft%d_s%d" % (nmax, i, d,
                                                               fft, s)
                        out.append(CellCase(nm, CELL_GRID, nmax, cl, [nm],
                                            THRESHOLD2))
    nlats = [1, 2, 3, 4, 5, 6, 7, 8, 9, 20, 30, 31]
    for nmax in range(5):
        for i in range(12):
            for d in range(2):
                cl = generate_cell(nlats[i], nlats[i], R + 1000.0 * d, PI,
                                   2.0 * PI)
                nm = "shs_c_nx%d_n%d_dr%d_sctr" % (nmax, i, d)
                out.append(CellCase(nm, CELL_SCATTERED, nmax, cl, [nm],
                                    THRESHOLD2))
    return out


def sha_cell_cases():
    """tests/check_sha_cell.c:50-160: synthesis then analysis (approximate
    quadrature) on cell grids spanning the sphere; the non-symmetric
    variant moves the boundary between the first two cell rows by 0.001;
    golden C and S triangles, tolerance 10 threshold2."""
    out = []
    R = test_coefficients()[2]
    nlats = [1, 1, 3, 10]
    nlons = [1, 2, 8, 22]
    for nmax in range(5):
        for i in range(4):
            for s in range(2):
                if nlats[i] == 1 and s == 1:
                    continue
                if nlats[i] >= nmax + 1 and s == 0 and nmax == 0:
                    continue
                for d in range(2):
                    if nlats[i] < nmax + 1:
                        continue
                    cl = generate_cell(nlats[i], nlons[i], R + 1000.0 * d, PI,
                                       2.0 * PI)
                    if s == 0:
                        cl[0][0] += 0.001
                        cl[1][1] += 0.001
                    stem = "sha_c_nx%d_n%d_dr%d_s%d" % (nmax, i, d, s)
                    out.append(CellCase(stem, CELL_GRID, nmax, cl,
                                        [stem + "_c", stem + "_s"],
                                        10.0 * THRESHOLD2))
    return out
