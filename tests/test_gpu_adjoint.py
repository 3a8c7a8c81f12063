"""The adjoint of the scattered-point synthesis (charm_b200.autograd and
charm_b200_shs_point_sctr_adjoint).

CHarm has no transpose routine, so the reference transpose is built from its
forward synthesis: (i) explicit columns A e_k of the CPU oracle at nmax 20,
whose transpose applied to y must match the GPU adjoint; (ii) the
dot-product test <A x, y> = <x, A^T y> at nmax 360 with points off the
sphere.  Then the torch.autograd path against finite differences, and CGLS
on a small fit."""
import ctypes as ct

import numpy as np
import pytest

from charm_b200.workloads import GM, R_EARTH, kaula
from oracle import orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods():
    import torch
    import charm_b200 as cb
    from charm_b200 import autograd as ag
    return torch, cb, ag


def points(n, seed, hmax):
    rng = np.random.default_rng(seed)
    lat = np.arcsin(rng.uniform(-1.0, 1.0, n))
    lon = rng.uniform(0.0, 2.0 * np.pi, n)
    r = R_EARTH + rng.uniform(0.0, hmax, n)
    return lat, lon, r


def test_adjoint_matches_oracle_columns(mods):
    torch, cb, ag = mods
    N, npt = 20, 300
    lat, lon, r = points(npt, 11, 9000.0)
    T = (N + 1) * (N + 2) // 2
    op = orc.Point(orc.SCATTERED, lat, lon, r)
    A = np.zeros((npt, 2 * T))
    for k in range(2 * T):
        c = np.zeros(T)
        s = np.zeros(T)
        (c if k < T else s)[k % T] = 1.0
        A[:, k] = orc.shs_point(op, orc.Shc(N, GM, R_EARTH, c, s), N)[0]
    y = np.random.default_rng(12).standard_normal(npt)
    ref = A.T @ y
    p = cb.PointSctr(lat, lon, r)
    g = torch.from_numpy(y).cuda()
    gc, gs = ag._adjoint(g, p, N, GM, R_EARTH)
    got = np.concatenate([gc.cpu().numpy(), gs.cpu().numpy()])
    assert np.linalg.norm(got - ref) <= 1e-13 * np.linalg.norm(ref)
    # the host entry point gives the same numbers
    from charm_b200._lib import _libcharm as L
    L.charm_b200_shs_point_sctr_adjoint.argtypes = [
        ct.c_void_p, ct.POINTER(ct.c_double), ct.c_ulong, ct.c_void_p,
        ct.c_void_p]
    out = cb.Shc(N, GM, R_EARTH)
    err = L.charm_err_init()
    yy = np.ascontiguousarray(y)
    L.charm_b200_shs_point_sctr_adjoint(
        ct.cast(p._Point, ct.c_void_p),
        yy.ctypes.data_as(ct.POINTER(ct.c_double)), N,
        ct.cast(out._Shc, ct.c_void_p), ct.cast(err, ct.c_void_p))
    assert L.charm_err_isempty(err)
    L.charm_err_free(err)
    host = np.concatenate([out.c, out.s])
    assert np.array_equal(host, got)


def test_dot_product_identity(mods):
    torch, cb, ag = mods
    N, npt = 360, 20000
    lat, lon, r = points(npt, 21, 9000.0)
    p = cb.PointSctr(lat, lon, r)
    c, s = kaula(N, 22)
    x_c = torch.from_numpy(c).cuda()
    x_s = torch.from_numpy(s).cuda()
    y = torch.from_numpy(np.random.default_rng(23).standard_normal(npt)).cuda()
    ax = ag._synthesis(x_c, x_s, p, N, GM, R_EARTH)
    aty_c, aty_s = ag._adjoint(y, p, N, GM, R_EARTH)
    lhs = float(torch.dot(ax, y))
    rhs = float(torch.dot(x_c, aty_c) + torch.dot(x_s, aty_s))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_autograd_against_finite_differences(mods):
    torch, cb, ag = mods
    N, npt = 120, 5000
    lat, lon, r = points(npt, 31, 5000.0)
    p = cb.PointSctr(lat, lon, r)
    c, s = kaula(N, 32)
    obs = ag._synthesis(torch.from_numpy(c).cuda(), torch.from_numpy(s).cuda(),
                        p, N, GM, R_EARTH)
    c0, s0 = kaula(N, 33)
    xc = torch.from_numpy(c0).cuda().requires_grad_(True)
    xs = torch.from_numpy(s0).cuda().requires_grad_(True)
    f = ag.shs_point_sctr(xc, xs, p, N, GM, R_EARTH)
    loss = 0.5 * ((f - obs) ** 2).sum()
    loss.backward()
    rng = np.random.default_rng(34)
    dc = torch.from_numpy(rng.standard_normal(c.size) * 1e-6).cuda()
    ds = torch.from_numpy(rng.standard_normal(s.size) * 1e-6).cuda()
    m = torch.from_numpy(np.repeat(np.arange(N + 1),
                                   np.arange(N + 1, 0, -1))).cuda()
    ds[m == 0] = 0.0          # S_n0 does not exist

    def L(a, b):
        d = ag._synthesis(a, b, p, N, GM, R_EARTH) - obs
        return 0.5 * float((d * d).sum())

    with torch.no_grad():
        fd = (L(xc + dc, xs + ds) - L(xc - dc, xs - ds)) / 2.0
        an = float(torch.dot(xc.grad, dc) + torch.dot(xs.grad, ds))
    # the loss is quadratic: central differences are exact up to rounding
    assert abs(fd - an) <= 1e-7 * abs(an)


def test_cgls_fit_reduces_misfit(mods):
    torch, cb, ag = mods
    N, npt = 30, 4000
    lat, lon, r = points(npt, 41, 9000.0)
    p = cb.PointSctr(lat, lon, r)
    c, s = kaula(N, 42)
    truth = ag._synthesis(torch.from_numpy(c).cuda(),
                          torch.from_numpy(s).cuda(), p, N, GM, R_EARTH)
    xc, xs, hist = ag.cgls(p, truth, N, GM, R_EARTH, iters=60)
    assert all(b <= a * (1 + 1e-12) for a, b in zip(hist, hist[1:]))
    assert hist[-1] <= 1e-8 * hist[0]
    err_c = np.linalg.norm(xc.cpu().numpy() - c) / np.linalg.norm(c)
    assert err_c <= 1e-6
