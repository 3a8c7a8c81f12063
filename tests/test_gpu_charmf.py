"""The single-precision ABI (charmf_*, CHarm's float build's entry points)
against CHarm's own float build (oracle/_ref/libcharmf.so) and against the
FP64 path on the same inputs.

CHarm's float build computes everything in float (its X-numbers included);
charmf_* runs the single-precision kernels (FP32 recurrence and sums) for
the potential on FFT grids with nmax <= 2200 and the FP64 path, rounded to
float, for everything else.  Float keeps about 7 significant digits, so the
two implementations agree to a relative RMS of about 1e-6 of the field;
the bounds below leave a factor of ten or more over what is measured."""
import ctypes as ct

import numpy as np
import pytest

from charm_b200.workloads import GM, R_EARTH, kaula, rel_rms
from oracle import charm_ref

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not charm_ref.available("f"),
                                 reason="oracle/_ref has no float CHarm build")]


class PointF(ct.Structure):
    _fields_ = [("type", ct.c_int), ("nlat", ct.c_size_t),
                ("nlon", ct.c_size_t), ("npoint", ct.c_size_t),
                ("lat", ct.POINTER(ct.c_float)),
                ("lon", ct.POINTER(ct.c_float)),
                ("r", ct.POINTER(ct.c_float)), ("w", ct.POINTER(ct.c_float)),
                ("owner", ct.c_bool), ("distributed", ct.c_bool)]


class ShcF(ct.Structure):
    _fields_ = [("nmax", ct.c_ulong), ("mu", ct.c_float), ("r", ct.c_float),
                ("nc", ct.c_size_t), ("ns", ct.c_size_t),
                ("c", ct.POINTER(ct.POINTER(ct.c_float))),
                ("s", ct.POINTER(ct.POINTER(ct.c_float))),
                ("owner", ct.c_bool), ("distributed", ct.c_bool)]


@pytest.fixture(scope="module")
def F():
    """ctypes view of libcharm.so's charmf_* entry points."""
    import charm_b200  # noqa: F401  (loads the library)
    from charm_b200._lib import _libcharm as L, _Err
    P, UL, FL = ct.POINTER, ct.c_ulong, ct.c_float
    sig = {
        "charmf_err_init": ([], P(_Err)),
        "charmf_err_free": ([P(_Err)], None),
        "charmf_err_isempty": ([P(_Err)], ct.c_bool),
        "charmf_crd_point_gl": ([UL, FL], P(PointF)),
        "charmf_crd_point_dh1": ([UL, FL], P(PointF)),
        "charmf_crd_point_dh2": ([UL, FL], P(PointF)),
        "charmf_crd_point_free": ([P(PointF)], None),
        "charmf_shc_init": ([UL, FL, FL, P(FL), P(FL)], P(ShcF)),
        "charmf_shc_free": ([P(ShcF)], None),
        "charmf_shs_point": ([P(PointF), P(ShcF), UL, P(FL), P(_Err)], None),
        "charmf_shs_point_grad1": ([P(PointF), P(ShcF), UL, P(P(FL)),
                                    P(_Err)], None),
        "charmf_sha_point": ([P(PointF), P(FL), UL, P(ShcF), P(_Err)], None),
    }
    for name, (a, r) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = a
        fn.restype = r
    return L


@pytest.fixture(scope="module")
def CF():
    return charm_ref.Charm("f")


def _grid(F, kind, N, r):
    fn = {"gl": F.charmf_crd_point_gl, "dh1": F.charmf_crd_point_dh1,
          "dh2": F.charmf_crd_point_dh2}[kind]
    p = fn(N, r)
    assert p
    return p


def _check(F, err):
    assert F.charmf_err_isempty(err), ct.string_at(err.contents.msg).decode()


def _fp(a):
    return a.ctypes.data_as(ct.POINTER(ct.c_float))


def shs_f(F, kind, N, r, c, s):
    p = _grid(F, kind, N, r)
    c32 = c.astype(np.float32)
    s32 = s.astype(np.float32)
    h = F.charmf_shc_init(N, GM, R_EARTH, _fp(c32), _fp(s32))
    f = np.empty(p.contents.npoint, np.float32)
    err = F.charmf_err_init()
    F.charmf_shs_point(p, h, N, _fp(f), err)
    _check(F, err)
    F.charmf_err_free(err)
    F.charmf_shc_free(h)
    return p, f


def charm_float(CF, kind, N, r, c, s):
    k = {"gl": charm_ref.GL, "dh1": charm_ref.DH1, "dh2": charm_ref.DH2}[kind]
    cp, lat, lon, w = CF.grid(k, N, r)
    sh = CF.shc(N, GM, R_EARTH, c, s)
    return cp, sh, CF.shs_point(cp, sh, N, lat.size * lon.size)


@pytest.mark.parametrize("kind,N", [("gl", 360), ("dh1", 200), ("gl", 2190)])
def test_charmf_potential_vs_charm_float(F, CF, kind, N):
    """The single-precision kernels against CHarm's float build and the
    FP64 path."""
    import charm_b200 as cb
    c, s = kaula(N, 1100 + N)
    p, f = shs_f(F, kind, N, R_EARTH, c, s)
    _, _, fref = charm_float(CF, kind, N, R_EARTH, c, s)
    ctor = cb.PointGridGL if kind == "gl" else cb.PointGridDH1
    f64 = np.ravel(cb.shs_point(ctor(N, R_EARTH), cb.Shc(N, GM, R_EARTH, c, s),
                                N))
    assert rel_rms(f, f64) <= 1e-6
    assert rel_rms(fref, f64) <= 1e-5
    assert rel_rms(f, fref) <= 1e-5
    F.charmf_crd_point_free(p)


def test_charmf_grad1_vs_charm_float(F, CF):
    """grad1 on the DH2 grid above the sphere (FP64 path, rounded)."""
    N, r = 200, R_EARTH + 250e3
    c, s = kaula(N, 1200)
    p = _grid(F, "dh2", N, r)
    c32, s32 = c.astype(np.float32), s.astype(np.float32)
    h = F.charmf_shc_init(N, GM, R_EARTH, _fp(c32), _fp(s32))
    out = [np.empty(p.contents.npoint, np.float32) for _ in range(3)]
    arr = (ct.POINTER(ct.c_float) * 3)(*[_fp(x) for x in out])
    err = F.charmf_err_init()
    F.charmf_shs_point_grad1(p, h, N, arr, err)
    _check(F, err)
    by_addr = {x.ctypes.data: x for x in out}
    mine = [by_addr[ct.cast(arr[i], ct.c_void_p).value] for i in range(3)]
    cp, sh, _ = charm_float(CF, "dh2", N, r, c, s)
    ref = CF.shs_point_grad(cp, sh, N, p.contents.npoint, 1)
    scale = max(np.sqrt(np.mean(x.astype(np.float64) ** 2)) for x in ref)
    for a, b in zip(mine, ref):
        d = a.astype(np.float64) - b.astype(np.float64)
        assert np.sqrt(np.mean(d * d)) / scale <= 1e-4
    F.charmf_err_free(err)
    F.charmf_shc_free(h)
    F.charmf_crd_point_free(p)


@pytest.mark.parametrize("kind,N", [("gl", 360), ("gl", 2300)])
def test_charmf_analysis(F, CF, kind, N):
    """charmf_sha_point of the float grid of charmf_shs_point: against
    CHarm's float analysis of the same float grid, and the round trip
    (single-precision kernels at nmax 360, the FP64 path above 2200)."""
    c, s = kaula(N, 1300 + N)
    p, f = shs_f(F, kind, N, R_EARTH, c, s)
    T = (N + 1) * (N + 2) // 2
    oc = np.zeros(T, np.float32)
    os_ = np.zeros(T, np.float32)
    h = F.charmf_shc_init(N, GM, R_EARTH, _fp(oc), _fp(os_))
    err = F.charmf_err_init()
    F.charmf_sha_point(p, _fp(f), N, h, err)
    _check(F, err)
    cp, lat, lon, w = CF.grid(charm_ref.GL, N, R_EARTH)
    cr, sr = CF.sha_point(cp, f, N, GM, R_EARTH)

    def joint(a, b, ra, rb):
        d = np.concatenate([a - ra, b - rb]).astype(np.float64)
        r = np.concatenate([ra, rb]).astype(np.float64)
        return np.sqrt(np.sum(d * d) / np.sum(r * r))
    # CHarm's float analysis carries float rounding of every step (measured
    # 1e-5 at nmax 360, 1e-4 at 2300 against the FP64 path's result)
    assert joint(oc, os_, cr, sr) <= 5e-4
    assert joint(oc, os_, c, s) <= 1e-4
    F.charmf_err_free(err)
    F.charmf_shc_free(h)
    F.charmf_crd_point_free(p)
