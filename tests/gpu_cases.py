"""Runs the golden-vector cases of CHarm's test-suite through libcharm.so
(the CUDA path) via its PyHarm-style Python interface."""
import numpy as np

import golden_data as gd


def product_point(cb, case):
    if case.grid is not None:
        g, nmax, r = case.grid
        if g == "gl":
            p = cb.PointGridGL(nmax, r)
        elif g == "dh1":
            p = cb.PointGridDH1(nmax, r)
        else:
            p = cb.PointGridDH2(nmax, r)
        if case.nlon_override is None and not case.lat0_shift:
            return p
        # CHarm's dynamical-switching tests keep the GL type but use the
        # first meridian only and move the first latitude
        lat = p.lat.copy()
        lat[0] -= case.lat0_shift
        lon = p.lon[:case.nlon_override].copy() if case.nlon_override else \
            p.lon.copy()
        return cb.PointGrid(lat, lon, p.r.copy(), ptype=p.type)
    if case.ptype == gd.SCATTERED:
        return cb.PointSctr(case.lat, case.lon, case.r)
    return cb.PointGrid(case.lat, case.lon, case.r)


def run_product(cb, case):
    p = product_point(cb, case)
    nmax_shc, mu, r, c, s = case.coeffs
    shc = cb.Shc(nmax_shc, mu, r, c, s)
    if case.kind == "pot":
        out = [cb.shs_point(p, shc, case.nmax)]
    elif case.kind == "grad1":
        out = cb.shs_point_grad1(p, shc, case.nmax)
    elif case.kind == "grad2":
        out = cb.shs_point_grad2(p, shc, case.nmax)
    else:
        dr, dlat, dlon = case.kind
        out = [cb.shs_point_guru(p, shc, case.nmax, dr, dlat, dlon)]
    return p, [np.asarray(o).reshape(-1) for o in out]


def check_product(cb, case):
    """Number of golden mismatches of one case (CHarm's validate())."""
    G = gd.golden("double")
    p, out = run_product(cb, case)
    bad = 0
    for j, (nm, f) in enumerate(zip(case.golden_names, out)):
        if gd.singular_component(case.kind, j):
            f = gd.zero_singular_rows(case.ptype, p.lat, len(p.lon), f)
        bad += gd.mismatches(f, G[nm], case.eps)
    return bad
