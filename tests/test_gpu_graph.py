"""Batched synthesis captured into a CUDA graph
(charm_b200_shs_point_batch_graph / charm_b200_graph_launch): a replay
reproduces the direct call bit for bit, and follows changes of the
coefficient buffers' contents between launches."""
import ctypes as ct

import numpy as np
import pytest

from charm_b200.workloads import GM, R_EARTH, kaula

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    import charm_b200 as cb
    from charm_b200._lib import _libcharm as L
    P = ct.c_void_p
    args = [P, ct.c_size_t, ct.POINTER(ct.c_ulong), ct.POINTER(ct.c_ulong),
            ct.POINTER(ct.c_double), ct.c_double, ct.POINTER(ct.c_void_p),
            ct.POINTER(ct.c_void_p), ct.c_int, ct.POINTER(ct.c_void_p)]
    L.charm_b200_shs_point_batch_dev.argtypes = args + [P]
    L.charm_b200_shs_point_batch_i8_dev.argtypes = args + [P]
    L.charm_b200_shs_point_batch_graph.argtypes = args + [ct.c_int, P]
    L.charm_b200_shs_point_batch_graph.restype = ct.c_void_p
    L.charm_b200_graph_launch.argtypes = [P, P]
    L.charm_b200_graph_free.argtypes = [P]
    return torch, cb, L


class Batch:
    def __init__(self, env, pnt, nmaxes, ncomp, seed):
        torch, cb, L = env
        n = len(nmaxes)
        self.n = n
        self.nm = (ct.c_ulong * n)(*nmaxes)
        self.mu = (ct.c_double * n)(*([GM] * n))
        self.c, self.s, self.f = [], [], []
        for j, N in enumerate(nmaxes):
            c, s = kaula(N, seed + j)
            self.c.append(torch.from_numpy(c).cuda())
            self.s.append(torch.from_numpy(s).cuda())
            self.f.append(torch.full((ncomp * pnt.lat.size * pnt.lon.size,),
                                     np.nan, dtype=torch.float64,
                                     device="cuda"))
        self.pc = (ct.c_void_p * n)(*[t.data_ptr() for t in self.c])
        self.ps = (ct.c_void_p * n)(*[t.data_ptr() for t in self.s])
        self.pf = (ct.c_void_p * n)(*[t.data_ptr() for t in self.f])

    def outputs(self):
        return [t.cpu().numpy().copy() for t in self.f]


def check(L, err):
    msg = None
    if not L.charm_err_isempty(err):
        msg = ct.string_at(err.contents.msg).decode()
        L.charm_err_reset(err)
    assert msg is None, msg


@pytest.mark.parametrize("split,kgrad", [(1, 0), (0, 3)])
def test_graph_replays_the_call(env, split, kgrad):
    torch, cb, L = env
    ncomp = 10 if kgrad == 3 else 1
    pnt = cb.PointGridDH2(260, R_EARTH + 2e4)
    b = Batch(env, pnt, [260, 77, 190], ncomp, 1300 + split)
    P = ct.c_void_p
    err = L.charm_err_init()
    direct = (L.charm_b200_shs_point_batch_i8_dev if split
              else L.charm_b200_shs_point_batch_dev)
    direct(ct.cast(pnt._Point, P), b.n, b.nm, b.nm, b.mu, R_EARTH, b.pc, b.ps,
           kgrad, b.pf, ct.cast(err, P))
    check(L, err)
    ref = b.outputs()
    for t in b.f:
        t.fill_(np.nan)
    g = L.charm_b200_shs_point_batch_graph(ct.cast(pnt._Point, P), b.n, b.nm,
                                           b.nm, b.mu, R_EARTH, b.pc, b.ps,
                                           kgrad, b.pf, split, ct.cast(err, P))
    check(L, err)
    assert g
    try:
        for t in b.f:
            t.fill_(np.nan)
        for _ in range(3):
            L.charm_b200_graph_launch(g, ct.cast(err, P))
            check(L, err)
        for a, r in zip(b.outputs(), ref):
            assert np.array_equal(a, r)
        # new coefficients in the same buffers: the replay follows them
        for t in b.c + b.s:
            t.mul_(2.0)
        L.charm_b200_graph_launch(g, ct.cast(err, P))
        check(L, err)
        for a, r in zip(b.outputs(), ref):
            assert np.array_equal(a, 2.0 * r)
    finally:
        L.charm_b200_graph_free(g)
        L.charm_err_free(err)


def test_graph_refuses_replay_after_buffers_changed(env):
    """A call with larger sizes between capture and replay reallocates the
    library's cached buffers the graph reads by address: the replay is
    refused with an error (no kernel touches freed memory), and a graph
    captured again replays."""
    torch, cb, L = env
    P = ct.c_void_p
    pnt = cb.PointGridGL(150, R_EARTH)
    b = Batch(env, pnt, [150, 90], 1, 1400)
    err = L.charm_err_init()
    args = (ct.cast(pnt._Point, P), b.n, b.nm, b.nm, b.mu, R_EARTH, b.pc, b.ps,
            0, b.pf)
    g = L.charm_b200_shs_point_batch_graph(*args, 0, ct.cast(err, P))
    check(L, err)
    L.charm_b200_graph_launch(g, ct.cast(err, P))
    check(L, err)
    ref = b.outputs()
    # a larger synthesis in between: grows the cached buffers
    big = cb.PointGridGL(1200, R_EARTH)
    c, s = kaula(1200, 1401)
    cb.shs_point(big, cb.Shc(1200, GM, R_EARTH, c, s), 1200)
    L.charm_b200_graph_launch(g, ct.cast(err, P))
    assert not L.charm_err_isempty(err)
    assert b"capture the graph again" in ct.string_at(err.contents.msg)
    L.charm_err_reset(err)
    L.charm_b200_graph_free(g)
    g = L.charm_b200_shs_point_batch_graph(*args, 0, ct.cast(err, P))
    check(L, err)
    for t in b.f:
        t.fill_(np.nan)
    L.charm_b200_graph_launch(g, ct.cast(err, P))
    check(L, err)
    for a, r in zip(b.outputs(), ref):
        assert np.array_equal(a, r)
    L.charm_b200_graph_free(g)
    L.charm_err_free(err)
