"""Differentiable scattered-point synthesis for PyTorch.

`shs_point_sctr(c, s, pnt, nmax, mu, r)` evaluates CHarm's potential
synthesis at scattered points (charm_shs_point on a
CHARM_CRD_POINT_SCATTERED point set) on the GPU and is differentiable with
respect to the coefficient triangles c and s: its backward pass is the
hand-written adjoint kernel (charm_b200_shs_point_sctr_adjoint_dev), not a
recorded graph.  `cgls` fits coefficients to observations at the points
with conjugate gradients on the normal equations, one synthesis and one
adjoint per iteration.

Tensors are float64 on the current CUDA device, order-major triangles of
degree nmax (CHarm's c[m][n - m] layout flattened).  The library runs on its
own stream; the current torch stream is synchronised before each call and
the library returns with its stream idle."""
import ctypes as ct

import torch

from ._lib import _libcharm as _L

__all__ = ["shs_point_sctr", "ScatteredSynthesis", "cgls"]

_P = ct.c_void_p
_L.charm_b200_shs_point_dev.argtypes = [
    _P, ct.c_ulong, ct.c_double, ct.c_double, _P, _P, ct.c_ulong, ct.c_int,
    ct.c_uint, ct.c_uint, ct.c_uint, _P, _P]
_L.charm_b200_shs_point_sctr_adjoint_dev.argtypes = [
    _P, _P, ct.c_ulong, ct.c_double, ct.c_double, ct.c_ulong, _P, _P, _P]


class CHarmGpuError(RuntimeError):
    pass


def _call(fn, *args):
    err = _L.charm_err_init()
    try:
        torch.cuda.current_stream().synchronize()
        fn(*args, ct.cast(err, _P))
        if not _L.charm_err_isempty(err):
            raise CHarmGpuError(ct.string_at(err.contents.msg).decode())
    finally:
        _L.charm_err_free(err)


def _tri(nmax):
    return (nmax + 1) * (nmax + 2) // 2


def _check(t, n, name):
    if t.dtype != torch.float64 or not t.is_cuda or t.numel() != n:
        raise ValueError("%s must be a float64 CUDA tensor of %d elements"
                         % (name, n))
    return t.contiguous()


def _synthesis(c, s, pnt, nmax, mu, r):
    c = _check(c, _tri(nmax), "c")
    s = _check(s, _tri(nmax), "s")
    f = torch.empty(pnt.npoint, dtype=torch.float64, device=c.device)
    _call(_L.charm_b200_shs_point_dev, ct.cast(pnt._Point, _P), nmax,
          float(mu), float(r), c.data_ptr(), s.data_ptr(), nmax, 0, 0, 0, 0,
          f.data_ptr())
    return f


def _adjoint(g, pnt, nmax, mu, r):
    g = _check(g, pnt.npoint, "g")
    T = _tri(nmax)
    gc = torch.empty(T, dtype=torch.float64, device=g.device)
    gs = torch.empty(T, dtype=torch.float64, device=g.device)
    _call(_L.charm_b200_shs_point_sctr_adjoint_dev, ct.cast(pnt._Point, _P),
          g.data_ptr(), nmax, float(mu), float(r), nmax, gc.data_ptr(),
          gs.data_ptr())
    return gc, gs


class ScatteredSynthesis(torch.autograd.Function):
    """f = A(c, s) at scattered points; backward: A^T g."""

    @staticmethod
    def forward(ctx, c, s, pnt, nmax, mu, r):
        ctx.pnt, ctx.nmax, ctx.mu, ctx.r = pnt, nmax, mu, r
        return _synthesis(c, s, pnt, nmax, mu, r)

    @staticmethod
    def backward(ctx, grad_f):
        gc, gs = _adjoint(grad_f.contiguous(), ctx.pnt, ctx.nmax, ctx.mu,
                          ctx.r)
        return gc, gs, None, None, None, None


def shs_point_sctr(c, s, pnt, nmax, mu, r):
    """Differentiable potential synthesis at the scattered points `pnt`
    (a charm_b200.PointSctr) from the degree-nmax triangles c, s of the
    model (mu, r)."""
    return ScatteredSynthesis.apply(c, s, pnt, nmax, mu, r)


def cgls(pnt, obs, nmax, mu, r, iters=20, callback=None):
    """Least-squares coefficients of degree nmax for the observations `obs`
    at `pnt`: CGLS (conjugate gradients on A^T A x = A^T b) from x = 0 with
    `iters` iterations.  Returns (c, s, residual norms per iteration)."""
    obs = _check(obs, pnt.npoint, "obs")
    T = _tri(nmax)
    dev = obs.device
    xc = torch.zeros(T, dtype=torch.float64, device=dev)
    xs = torch.zeros(T, dtype=torch.float64, device=dev)
    res = obs.clone()
    sc, ss = _adjoint(res, pnt, nmax, mu, r)
    pc, ps = sc.clone(), ss.clone()
    gamma = float(torch.dot(sc, sc) + torch.dot(ss, ss))
    hist = [float(torch.linalg.norm(res))]
    for it in range(iters):
        if gamma == 0.0:
            break
        q = _synthesis(pc, ps, pnt, nmax, mu, r)
        qq = float(torch.dot(q, q))
        if qq == 0.0:
            break
        alpha = gamma / qq
        xc.add_(pc, alpha=alpha)
        xs.add_(ps, alpha=alpha)
        res.add_(q, alpha=-alpha)
        sc, ss = _adjoint(res, pnt, nmax, mu, r)
        gamma_new = float(torch.dot(sc, sc) + torch.dot(ss, ss))
        beta = gamma_new / gamma
        gamma = gamma_new
        pc.mul_(beta).add_(sc)
        ps.mul_(beta).add_(ss)
        hist.append(float(torch.linalg.norm(res)))
        if callback is not None:
            callback(it, xc, xs, hist[-1])
    return xc, xs, hist
