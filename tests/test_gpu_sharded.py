"""Latitude-band sharding on one GPU: the band analyses of a partition of
the latitude pairs (charm_b200_sha_point_dev_band) sum to the whole
analysis, the band syntheses reproduce the whole grid's rows, and the
sharded drivers (charm_b200.sharded) run end to end without a process
group (one rank).  The multi-rank collectives are covered on CPU by
tests/test_sharded.py (gloo)."""
import numpy as np
import pytest

from charm_b200.workloads import GM, R_EARTH, coef_rel_rms, kaula, rel_rms

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("grid,N,nb", [("GL", 360, 3), ("DH2", 300, 4),
                                       ("DH1", 201, 5)])
def test_bands_sum_to_the_whole(grid, N, nb):
    import torch
    import charm_b200 as cb
    from charm_b200.replicas import split_range
    from charm_b200.sharded import (grid_pairs, gpu_engine,
                                    sharded_analysis, sharded_synthesis)
    ctor = {"GL": cb.PointGridGL, "DH1": cb.PointGridDH1,
            "DH2": cb.PointGridDH2}[grid]
    p = ctor(N, R_EARTH)
    c, s = kaula(N, 5100 + N)
    f = cb.shs_point(p, cb.Shc(N, GM, R_EARTH, c, s), N)
    full = cb.sha_point(p, f, N, GM, R_EARTH)
    synth_rows, analyse_band, set_grid = gpu_engine(p, N, GM, R_EARTH)
    row_n, row_s = grid_pairs(p._Point, p.lat.size)
    d_f = torch.from_numpy(np.ascontiguousarray(f).ravel()).cuda()
    set_grid(d_f)
    acc_c = torch.zeros(c.size, dtype=torch.float64, device="cuda")
    acc_s = torch.zeros_like(acc_c)
    dc = torch.from_numpy(c).cuda()
    ds = torch.from_numpy(s).cuda()
    covered = []
    for b in range(nb):
        p0, p1 = split_range(len(row_n), b, nb)
        bc, bs = analyse_band(p0, p1)
        acc_c += bc
        acc_s += bs
        from charm_b200.sharded import band_rows
        rows = band_rows(row_n, row_s, p0, p1)
        covered += rows
        vals = synth_rows(rows, dc, ds).cpu().numpy()
        assert rel_rms(vals, f[rows]) <= 1e-14
    assert sorted(covered) == list(range(p.lat.size))
    assert coef_rel_rms(acc_c.cpu().numpy(), acc_s.cpu().numpy(),
                        full.c, full.s) <= 1e-14
    # the drivers with a single rank
    rows, vals = sharded_synthesis(row_n, row_s, dc.clone(), ds.clone(),
                                   synth_rows)
    assert rel_rms(vals.cpu().numpy(), f[rows]) <= 1e-14
    oc, os_ = sharded_analysis(len(row_n), analyse_band)
    assert coef_rel_rms(oc.cpu().numpy(), os_.cpu().numpy(),
                        full.c, full.s) <= 1e-14


def test_band_rejects_out_of_range():
    import ctypes as ct
    import torch
    import charm_b200 as cb
    from charm_b200._lib import _libcharm as L
    from charm_b200.sharded import gpu_engine
    N = 40
    p = cb.PointGridGL(N, R_EARTH)
    _, analyse_band, set_grid = gpu_engine(p, N, GM, R_EARTH)
    set_grid(torch.zeros(p.lat.size * p.lon.size, dtype=torch.float64,
                         device="cuda"))
    with pytest.raises(cb.CHarmError):
        analyse_band(0, 10 ** 6)
    # an empty band contributes zeros
    bc, bs = analyse_band(5, 5)
    assert float(bc.abs().max()) == 0.0 and float(bs.abs().max()) == 0.0
