"""Split-precision batched synthesis (charm_b200_shs_point_batch_i8_dev):
the degree sums on the tensor cores as exact INT8 digit products, against
the FP64 batched path (itself checked against charm_shs_point per set in
test_gpu_batch.py) on the same grids and coefficients.

Both operands carry 54-bit fixed-point values and the dropped digit levels
lie below 2^-47 of the largest products, so the fields agree with the FP64
path to about 1e-15 relative RMS; the tolerance is 1e-13 per set, the same
as the FP64 batch's against single calls."""
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
    for f in (L.charm_b200_shs_point_batch_dev,
              L.charm_b200_shs_point_batch_i8_dev):
        f.argtypes = [P, ct.c_size_t, ct.POINTER(ct.c_ulong),
                      ct.POINTER(ct.c_ulong), ct.POINTER(ct.c_double),
                      ct.c_double, ct.POINTER(ct.c_void_p),
                      ct.POINTER(ct.c_void_p), ct.c_int,
                      ct.POINTER(ct.c_void_p), P]
    return torch, cb, L


def run(env, fn, pnt, sets, r, kgrad=0):
    torch, cb, L = env
    n = len(sets)
    nm = (ct.c_ulong * n)(*[s[0] for s in sets])
    mu = (ct.c_double * n)(*[s[3] for s in sets])
    keep, outs = [], []
    dc = (ct.c_void_p * n)()
    ds = (ct.c_void_p * n)()
    df = (ct.c_void_p * n)()
    for j, (N, c, s, _) in enumerate(sets):
        tc = torch.from_numpy(c).cuda()
        ts = torch.from_numpy(s).cuda()
        tf = torch.full((pnt.lat.size * pnt.lon.size,), np.nan,
                        dtype=torch.float64, device="cuda")
        keep += [tc, ts]
        outs.append(tf)
        dc[j], ds[j], df[j] = tc.data_ptr(), ts.data_ptr(), tf.data_ptr()
    err = L.charm_err_init()
    fn(ct.cast(pnt._Point, ct.c_void_p), n, nm, nm, mu, r, dc, ds, kgrad, df,
       ct.cast(err, ct.c_void_p))
    msg = None
    if not L.charm_err_isempty(err):
        msg = ct.string_at(err.contents.msg).decode()
    L.charm_err_free(err)
    if msg is not None:
        return None, msg
    shape = (pnt.lat.size, pnt.lon.size)
    return [o.cpu().numpy().reshape(shape) for o in outs], None


def make_sets(seed, nmaxes):
    sets = []
    for j, N in enumerate(nmaxes):
        c, s = kaula(N, seed + j)
        sets.append((N, c, s, GM * (1.0 + 0.01 * j)))
    return sets


def compare(env, pnt, sets, r, tol=1e-13):
    torch, cb, L = env
    ref, msg = run(env, L.charm_b200_shs_point_batch_dev, pnt, sets, r)
    assert msg is None, msg
    got, msg = run(env, L.charm_b200_shs_point_batch_i8_dev, pnt, sets, r)
    assert msg is None, msg
    worst = 0.0
    for (N, *_), g, f in zip(sets, got, ref):
        assert np.all(np.isfinite(g))
        e = rel_rms(g, f)
        worst = max(worst, e)
        assert e <= tol, (N, e)
    return worst


def test_i8_gl_on_the_sphere(env):
    torch, cb, L = env
    p = cb.PointGridGL(360, R_EARTH)
    w = compare(env, p, make_sets(900, [360, 90, 359, 2, 200]), R_EARTH)
    print("GL 360 worst relative RMS %.2e" % w)


def test_i8_dh2_above_the_sphere_two_groups(env):
    """20 sets: two launches of 16 and 4; r = R + 250 km (R/r folded into
    the recurrence)."""
    torch, cb, L = env
    rng = np.random.default_rng(910)
    nmaxes = [int(v) for v in rng.integers(20, 301, size=20)]
    nmaxes[7] = 300
    p = cb.PointGridDH2(300, R_EARTH + 250e3)
    w = compare(env, p, make_sets(920, nmaxes), R_EARTH)
    print("DH2 300 (20 sets) worst relative RMS %.2e" % w)


def test_i8_small_degrees_and_ragged_tiles(env):
    """Degrees 0..3 (a single partial chunk) and a grid whose latitude pairs
    fill neither a 128-pair tile nor a 64-degree chunk."""
    torch, cb, L = env
    p = cb.PointGridDH1(3, R_EARTH)
    compare(env, p, make_sets(930, [3, 0, 1, 2]), R_EARTH)
    p = cb.PointGridGL(150, R_EARTH + 1000.0)
    compare(env, p, make_sets(940, [150, 64, 63, 65, 127, 128]), R_EARTH)


def test_i8_below_the_sphere(env):
    """r < R: (R/r)^(n+1) grows with the degree; the fixed-point bound
    follows it."""
    torch, cb, L = env
    p = cb.PointGridDH2(120, R_EARTH - 5000.0)
    compare(env, p, make_sets(950, [120, 80, 120]), R_EARTH)


def test_i8_rejects_gradients(env):
    torch, cb, L = env
    p = cb.PointGridGL(30, R_EARTH)
    _, msg = run(env, L.charm_b200_shs_point_batch_i8_dev, p,
                 make_sets(960, [30]), R_EARTH, kgrad=1)
    assert msg is not None and "kgrad" in msg
