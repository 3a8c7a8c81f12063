"""Batched synthesis (charm_b200_shs_point_batch_dev): many coefficient sets
of different degrees on one grid, the potential and its first and second
gradients in one launch per kind, against one charm_shs_point /
charm_shs_point_grad1 / charm_shs_point_grad2 call per set.

The batch shares the recurrence tables of the largest degree, so the sums
round differently from the single calls; 1e-13 relative RMS per component
(gradients 1e-12) leaves a wide margin over what is observed."""
import ctypes as ct

import numpy as np
import pytest

from charm_b200.workloads import GM, R_EARTH, kaula, rel_rms

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    import charm_b200 as cb
    from charm_b200._lib import _libcharm as L
    P = ct.c_void_p
    L.charm_b200_shs_point_batch_dev.argtypes = [
        P, ct.c_size_t, ct.POINTER(ct.c_ulong), ct.POINTER(ct.c_ulong),
        ct.POINTER(ct.c_double), ct.c_double, ct.POINTER(ct.c_void_p),
        ct.POINTER(ct.c_void_p), ct.c_int, ct.POINTER(ct.c_void_p), P]
    return torch, cb, L


def batch(env, pnt, sets, r, kgrad):
    torch, cb, L = env
    n = len(sets)
    ncomp = {0: 1, 1: 3, 2: 6, 3: 10}[kgrad]
    nm = (ct.c_ulong * n)(*[s[0] for s in sets])
    mu = (ct.c_double * n)(*[s[3] for s in sets])
    keep = []
    dc = (ct.c_void_p * n)()
    ds = (ct.c_void_p * n)()
    df = (ct.c_void_p * n)()
    outs = []
    for j, (N, c, s, _) in enumerate(sets):
        tc = torch.from_numpy(c).cuda()
        ts = torch.from_numpy(s).cuda()
        tf = torch.full((ncomp * pnt.lat.size * pnt.lon.size,), np.nan,
                        dtype=torch.float64, device="cuda")
        keep += [tc, ts]
        outs.append(tf)
        dc[j], ds[j], df[j] = tc.data_ptr(), ts.data_ptr(), tf.data_ptr()
    err = L.charm_err_init()
    L.charm_b200_shs_point_batch_dev(ct.cast(pnt._Point, ct.c_void_p), n, nm,
                                     nm, mu, r, dc, ds, kgrad, df,
                                     ct.cast(err, ct.c_void_p))
    msg = None
    if not L.charm_err_isempty(err):
        msg = ct.string_at(err.contents.msg).decode()
    L.charm_err_free(err)
    assert msg is None, msg
    shape = (ncomp, pnt.lat.size, pnt.lon.size)
    return [o.cpu().numpy().reshape(shape) for o in outs]


def make_sets(seed, nmaxes):
    sets = []
    for j, N in enumerate(nmaxes):
        c, s = kaula(N, seed + j)
        sets.append((N, c, s, GM * (1.0 + 0.01 * j)))
    return sets


def test_batch_all_ten_on_dh2_above_the_sphere(env):
    torch, cb, L = env
    nmaxes = [300, 41, 187, 96, 250, 120]
    Ng = max(nmaxes)
    r = R_EARTH
    p = cb.PointGridDH2(Ng, R_EARTH + 250e3)
    sets = make_sets(100, nmaxes)
    got = batch(env, p, sets, r, 3)
    for (N, c, s, mu), g in zip(sets, got):
        shc = cb.Shc(N, mu, r, c, s)
        pot = cb.shs_point(p, shc, N)
        g1 = cb.shs_point_grad1(p, shc, N)
        g2 = cb.shs_point_grad2(p, shc, N)
        assert rel_rms(g[0], pot) <= 1e-13
        for q in range(3):
            assert rel_rms(g[1 + q], g1[q]) <= 1e-12, (N, q)
        for q in range(6):
            assert rel_rms(g[4 + q], g2[q]) <= 1e-12, (N, q)


def test_batch_reused_buffers_low_degree_sets(env):
    """A second call of the same shape, now with sets of lower degree, must
    not see the orders the first call left in the lumped-coefficient
    buffer."""
    torch, cb, L = env
    p = cb.PointGridDH2(240, R_EARTH)
    batch(env, p, make_sets(300, [240, 240, 240]), R_EARTH, 1)
    sets = make_sets(310, [240, 35, 120])
    got = batch(env, p, sets, R_EARTH, 1)
    for (N, c, s, mu), g in zip(sets, got):
        shc = cb.Shc(N, mu, R_EARTH, c, s)
        g1 = cb.shs_point_grad1(p, shc, N)
        for q in range(3):
            assert rel_rms(g[q], g1[q]) <= 1e-12, (N, q)


def test_batch_potential_on_gl(env):
    torch, cb, L = env
    nmaxes = [360, 90, 359, 2, 200]
    p = cb.PointGridGL(360, R_EARTH)
    sets = make_sets(200, nmaxes)
    got = batch(env, p, sets, R_EARTH, 0)
    for (N, c, s, mu), g in zip(sets, got):
        ref = cb.shs_point(p, cb.Shc(N, mu, R_EARTH, c, s), N)
        assert rel_rms(g[0], ref) <= 1e-13, N
