"""Latitude-band sharding (charm_b200.sharded) on CPU: two gloo ranks
(127.0.0.1) split the latitude pairs of a GL grid, broadcast the
coefficients, synthesise their bands and all-reduce their band analyses;
the CPU oracle computes each band.  The union of the bands must be every
row exactly once, the band rows must equal the whole grid's, and the
reduced triangle must equal the single-rank analysis."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from charm_b200.workloads import GM, R_EARTH, coef_rel_rms, kaula, rel_rms

N = 24


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_engine(p, f_full):
    """synth_rows / analyse_band computed by the CPU oracle."""
    from oracle import orc
    from charm_b200.sharded import grid_pairs

    def synth_rows(rows, c, s):
        q = orc.Point(orc.GRID, p.lat[rows], p.lon, np.asarray(p.r)[rows])
        f = orc.shs_point(q, orc.Shc(N, GM, R_EARTH, c.numpy(), s.numpy()),
                          N)[0]
        return torch.from_numpy(np.ascontiguousarray(f).reshape(len(rows),
                                                                 -1))

    def analyse_band(p0, p1):
        row_n, row_s = grid_pairs(p._Point, p.lat.size)
        keep = np.zeros(p.lat.size, bool)
        keep[row_n[p0:p1]] = True
        keep[[r for r in row_s[p0:p1] if r >= 0]] = True
        f = np.where(keep[:, None], f_full, 0.0)
        out = orc.sha_point(orc.gl(N, R_EARTH), f, N, GM, R_EARTH)
        return torch.from_numpy(out.c.copy()), torch.from_numpy(out.s.copy())

    return synth_rows, analyse_band


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    from oracle import orc
    import charm_b200.pyharm as ph
    from charm_b200.sharded import (grid_pairs, sharded_analysis,
                                    sharded_synthesis)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        g = orc.gl(N, R_EARTH)
        p = ph.PointGrid(g.lat, g.lon, np.full(g.lat.size, R_EARTH),
                         ptype=ph.GRID_GL)
        c, s = kaula(N, 77)
        f_full = orc.shs_point(g, orc.Shc(N, GM, R_EARTH, c, s),
                               N)[0].reshape(g.lat.size, -1)
        synth_rows, analyse_band = _oracle_engine(p, f_full)
        row_n, row_s = grid_pairs(p._Point, p.lat.size)
        # rank 0's coefficients must reach the other rank
        tc = torch.from_numpy(c.copy()) if rank == 0 else torch.zeros(c.size,
                                                                       dtype=torch.float64)
        ts = torch.from_numpy(s.copy()) if rank == 0 else torch.zeros(s.size,
                                                                       dtype=torch.float64)
        rows, vals = sharded_synthesis(row_n, row_s, tc, ts, synth_rows)
        band_err = rel_rms(vals.numpy(), f_full[rows])
        cr, sr = sharded_analysis(len(row_n), analyse_band)
        full = orc.sha_point(g, f_full, N, GM, R_EARTH)
        coef_err = coef_rel_rms(cr.numpy(), sr.numpy(), full.c, full.s)
        all_rows = [None] * world
        dist.all_gather_object(all_rows, rows)
        q.put((rank, band_err, coef_err, all_rows, len(row_n), p.lat.size))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_latitude_bands():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=180) for _ in range(world)),
                 key=lambda x: x[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank, band_err, coef_err, all_rows, npairs, nlat in res:
        assert band_err <= 1e-14
        assert coef_err <= 1e-14
        flat = sorted(r for rows in all_rows for r in rows)
        assert flat == list(range(nlat))       # every row exactly once
        assert npairs == (nlat + 1) // 2


def _file_worker(rank, world, port, path, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    from charm_b200.sharded import coefficients_from_file
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        c, s, mu, r = coefficients_from_file(path, 30, "cpu")
        # a failed read on rank 0 reaches every rank as an error
        try:
            coefficients_from_file(path + ".missing", 30, "cpu")
            failed = False
        except Exception:
            failed = True
        q.put((rank, c.numpy().copy(), s.numpy().copy(), mu, r, failed))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_coefficients_from_file(tmp_path):
    """A binary coefficient file read by rank 0 and broadcast: every rank
    holds rank 0's triangles (the file's first 30 degrees), mu and r."""
    import ctypes as ct
    import charm_b200.pyharm as ph
    from charm_b200._lib import _libcharm as L
    nmax = 40
    T = (nmax + 1) * (nmax + 2) // 2
    rng = np.random.default_rng(3)
    c = rng.standard_normal(T)
    s = rng.standard_normal(T)
    s[:nmax + 1] = 0.0
    shc = ph.Shc(nmax, 3.986e14, 6378136.3, c, s)
    path = str(tmp_path / "m.shcs")
    L.charm_shc_write_bin.argtypes = [ct.c_void_p, ct.c_ulong, ct.c_char_p,
                                      ct.c_void_p]
    err = L.charm_err_init()
    L.charm_shc_write_bin(ct.cast(shc._Shc, ct.c_void_p), nmax, path.encode(),
                          ct.cast(err, ct.c_void_p))
    assert L.charm_err_isempty(err)
    L.charm_err_free(err)
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_file_worker, args=(r, world, port, path, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=180) for _ in range(world)),
                 key=lambda x: x[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    want_c = np.concatenate([c[m * (2 * nmax + 3 - m) // 2:
                               m * (2 * nmax + 3 - m) // 2 + 31 - m]
                             for m in range(31)])
    for rank, rc, rs, mu, r, failed in res:
        assert np.array_equal(rc, want_c)
        assert mu == 3.986e14 and r == 6378136.3
        assert failed
    assert np.array_equal(res[0][2], res[1][2])
