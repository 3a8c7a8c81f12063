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
    ncomp = {0: 1, 1: 3, 2: 6, 3: 10}.get(kgrad, 1)
    for j, (N, c, s, _) in enumerate(sets):
        tc = torch.from_numpy(c).cuda()
        ts = torch.from_numpy(s).cuda()
        tf = torch.full((ncomp * pnt.lat.size * pnt.lon.size,), np.nan,
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
    if kgrad:
        shape = (ncomp,) + shape
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


NAMES = {1: ["x", "y", "z"], 2: ["xx", "xy", "xz", "yy", "yz", "zz"],
         3: ["V", "x", "y", "z", "xx", "xy", "xz", "yy", "yz", "zz"]}


# Per-component bounds of the split-precision path against the FP64 path
# (relative RMS off the poles).  The fixed-point digits carry ~2^-56 of each
# column's largest term; the components formed as differences of the
# families' sums lose more: x, y, xz, yz through the 1 / u of the
# derivative relation, xy most, through 1 / u^2 and two cancelling terms
# (measured up to 6e-12 at nmax 300, 8e-10 in the 64-set nmax 2160 batch).
I8_BOUND = {"V": 1e-12, "z": 1e-12, "zz": 1e-12, "xx": 1e-12, "yy": 1e-12,
            "x": 1e-11, "y": 1e-11, "xz": 1e-11, "yz": 1e-11, "xy": 1e-10}


def interior(pnt):
    """Rows off the poles: the x / y components are singular at a pole
    (CHarm's tests zero them there, tests/check_shs_point_all.c:229-300)."""
    return np.cos(pnt.lat) > 1e-8


@pytest.mark.parametrize("grid,N,h,kgrad", [
    ("GL", 300, 0.0, 3),
    ("DH2", 200, 250e3, 3),      # the batched workload's height, pole row
    ("DH1", 150, -5000.0, 1),
    ("GL", 129, 1000.0, 2),
])
def test_i8_gradients_against_fp64(env, grid, N, h, kgrad):
    """grad1 / grad2 / all ten quantities through the gradient families on
    the tensor cores, 4 sets (launches of 3 and 1), each component against
    the FP64 batch's, relative to that component's RMS off the poles."""
    torch, cb, L = env
    ctor = {"GL": cb.PointGridGL, "DH1": cb.PointGridDH1,
            "DH2": cb.PointGridDH2}[grid]
    p = ctor(N, R_EARTH + h)
    sets = make_sets(970 + N, [N, N // 2, N - 1, 3])
    ref, msg = run(env, L.charm_b200_shs_point_batch_dev, p, sets, R_EARTH,
                   kgrad)
    assert msg is None, msg
    got, msg = run(env, L.charm_b200_shs_point_batch_i8_dev, p, sets, R_EARTH,
                   kgrad)
    assert msg is None, msg
    keep = interior(p)
    worst = {}
    for (Ns, *_), g, f in zip(sets, got, ref):
        for q, name in enumerate(NAMES[kgrad]):
            a, b = g[q][keep], f[q][keep]
            assert np.all(np.isfinite(a)), (Ns, name)
            e = rel_rms(a, b)
            worst[name] = max(worst.get(name, 0.0), e)
            assert e <= I8_BOUND[name], (Ns, name, e)
        # the non-singular components on the pole rows too
        for q, name in enumerate(NAMES[kgrad]):
            if name in ("V", "z", "zz"):
                assert rel_rms(g[q], f[q]) <= 1e-12, (Ns, name)
    print(grid, N, kgrad, {k: "%.1e" % v for k, v in worst.items()})


def test_i8_gradients_against_oracle(env):
    """All ten quantities of one set at nmax 120 on the DH2 grid at
    R + 250 km against the CPU oracle on 6 interior rows."""
    from oracle import orc
    torch, cb, L = env
    N, h = 120, 250e3
    p = cb.PointGridDH2(N, R_EARTH + h)
    sets = make_sets(990, [N])
    got, msg = run(env, L.charm_b200_shs_point_batch_i8_dev, p, sets, R_EARTH,
                   3)
    assert msg is None, msg
    rows = np.linspace(3, p.lat.size - 4, 6).astype(int)
    po = orc.Point(orc.GRID, p.lat[rows], p.lon,
                   np.full(rows.size, R_EARTH + h))
    N_, c, s, mu = sets[0]
    shc = orc.Shc(N, mu, R_EARTH, c, s)
    ref = (orc.shs_point(po, shc, N, "pot") + orc.shs_point(po, shc, N, "grad1")
           + orc.shs_point(po, shc, N, "grad2"))
    for q, name in enumerate(NAMES[3]):
        e = rel_rms(got[0][q][rows], np.reshape(ref[q], (rows.size, -1)))
        assert e <= 1e-12, (name, e)


def test_i8_rejects_bad_kgrad(env):
    torch, cb, L = env
    p = cb.PointGridGL(30, R_EARTH)
    _, msg = run(env, L.charm_b200_shs_point_batch_i8_dev, p,
                 make_sets(960, [30]), R_EARTH, kgrad=4)
    assert msg is not None and "kgrad" in msg
