"""Latitude-band sharding of one grid transform over the ranks of a
torch.distributed process group (one process per GPU; NCCL on GPUs, gloo
for the CPU tests).

CHarm's MPI build distributes the latitudes of a grid in chunks over its
processes and sums the coefficient contributions of the chunks
(src/mpi, src/shc/shc_block_set_coeffs.c:80-86, shc_block_get_coeffs.c:
80-86).  Here the unit of distribution is the latitude pair (a northern row
and its mirror row, the grouping every kernel uses, charm_b200_grid_pairs):
rank k of w owns the contiguous pairs split_range(npairs, k, w).

* Synthesis: rank 0's coefficient triangle is broadcast; every rank
  synthesises the rows of its band (a user grid of the band's latitudes with
  the grid's longitudes, northern members then their mirrors, so that the
  pairs keep their symmetry) into its own buffer.  No further exchange.
* Analysis: every rank analyses the band it holds
  (charm_b200_sha_point_dev_band); one all_reduce(SUM) of the 2 T
  coefficients gives every rank the whole analysis.

The band logic and the collectives are independent of the engine: the
`synth_rows` / `analyse_band` callables compute one band, so the same
drivers run the GPU library (gpu_engine) or a CPU oracle in the tests.
"""
import ctypes as ct

import numpy as np

from .replicas import split_range

__all__ = ["grid_pairs", "band_rows", "sharded_synthesis",
           "sharded_analysis", "gpu_engine", "coefficients_from_file"]


def _dist():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist
    return None


def grid_pairs(pnt_ptr, nlat):
    """(row_n, row_s) of a charm_point (ctypes pointer): the latitude pairs
    as the transforms group them (row_s -1 where a row has no mirror)."""
    from ._lib import _libcharm as L
    L.charm_b200_grid_pairs.restype = ct.c_int
    L.charm_b200_grid_pairs.argtypes = [ct.c_void_p, ct.c_void_p,
                                        ct.c_void_p, ct.c_int]
    cap = int(nlat) + 1
    rn = np.zeros(cap, np.int32)
    rs = np.zeros(cap, np.int32)
    n = L.charm_b200_grid_pairs(ct.cast(pnt_ptr, ct.c_void_p), rn.ctypes.data,
                                rs.ctypes.data, cap)
    return rn[:n].copy(), rs[:n].copy()


def band_rows(row_n, row_s, p0, p1):
    """Grid rows of the pairs [p0, p1): the northern members in order, then
    the mirrors in grid order (north to south)."""
    north = [int(r) for r in row_n[p0:p1]]
    south = sorted(int(r) for r in row_s[p0:p1] if r >= 0)
    return north + south


def _rank_world(group):
    dist = _dist()
    if dist is None:
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def sharded_synthesis(row_n, row_s, c, s, synth_rows, group=None):
    """Broadcasts the triangles (c, s: tensors, rank 0's values win) and
    returns (rows, values) of this rank's band: values = synth_rows(rows,
    c, s), one row of the grid per entry of rows."""
    dist = _dist()
    if dist is not None:
        dist.broadcast(c, src=0, group=group)
        dist.broadcast(s, src=0, group=group)
    rank, world = _rank_world(group)
    p0, p1 = split_range(len(row_n), rank, world)
    rows = band_rows(row_n, row_s, p0, p1)
    return rows, synth_rows(rows, c, s)


def sharded_analysis(npairs, analyse_band, group=None):
    """(c, s) of the whole analysis on every rank: analyse_band(p0, p1)
    returns this rank's contribution (tensors), summed over the ranks by
    one all_reduce each."""
    rank, world = _rank_world(group)
    p0, p1 = split_range(npairs, rank, world)
    c, s = analyse_band(p0, p1)
    dist = _dist()
    if dist is not None:
        dist.all_reduce(c, group=group)
        dist.all_reduce(s, group=group)
    return c, s


def coefficients_from_file(path, nmax, device, group=None):
    """(c, s, mu, r) of a coefficient file in CHarm's binary format
    (charm_shc_read_bin), read by rank 0 and broadcast to every rank of the
    group: c, s are order-major triangles of degree nmax on `device`.  On a
    CUDA device rank 0 streams the file straight into device memory
    (charm_b200_shc_read_bin_dev: chunks of orders through page-locked
    buffers, the disk reads overlapping the copies); on the CPU it reads
    the host triangles with charm_shc_read_bin."""
    import torch
    from . import pyharm
    from ._lib import _libcharm as L
    dist = _dist()
    rank, _ = _rank_world(group)
    T = (int(nmax) + 1) * (int(nmax) + 2) // 2
    c = torch.zeros(T, dtype=torch.float64, device=device)
    s = torch.zeros(T, dtype=torch.float64, device=device)
    # mu, r and 1 when rank 0 read the file (every rank learns of a failed
    # read before it waits for the triangles)
    hdr = torch.zeros(3, dtype=torch.float64, device=device)
    msg = None
    if rank == 0:
        err = L.charm_err_init()
        if torch.device(device).type == "cuda":
            P = ct.c_void_p
            L.charm_b200_shc_read_bin_dev.restype = ct.c_ulong
            L.charm_b200_shc_read_bin_dev.argtypes = [
                ct.c_char_p, ct.c_ulong, ct.c_ulong, P, P,
                ct.POINTER(ct.c_double), ct.POINTER(ct.c_double), P]
            mu, r = ct.c_double(), ct.c_double()
            L.charm_b200_shc_read_bin_dev(str(path).encode(), int(nmax),
                                          int(nmax), c.data_ptr(),
                                          s.data_ptr(), ct.byref(mu),
                                          ct.byref(r), ct.cast(err, P))
            hdr[0], hdr[1] = mu.value, r.value
        else:
            L.charm_shc_read_bin.restype = ct.c_ulong
            L.charm_shc_read_bin.argtypes = [ct.c_char_p, ct.c_ulong,
                                             ct.c_void_p, ct.c_void_p]
            shc = pyharm.Shc(int(nmax), 1.0, 1.0)
            L.charm_shc_read_bin(str(path).encode(), int(nmax),
                                 ct.cast(shc._Shc, ct.c_void_p),
                                 ct.cast(err, ct.c_void_p))
            c.copy_(torch.from_numpy(shc.c))
            s.copy_(torch.from_numpy(shc.s))
            hdr[0], hdr[1] = shc.mu, shc.r
        if not L.charm_err_isempty(err):
            msg = ct.string_at(err.contents.msg).decode()
        L.charm_err_free(err)
        hdr[2] = 0.0 if msg else 1.0
    if dist is not None:
        dist.broadcast(hdr, src=0, group=group)
    if float(hdr[2]) != 1.0:
        raise pyharm.CHarmError(msg or "rank 0 failed to read %s" % path)
    if dist is not None:
        dist.broadcast(c, src=0, group=group)
        dist.broadcast(s, src=0, group=group)
    return c, s, float(hdr[0]), float(hdr[1])


def gpu_engine(pnt, nmax, mu, r):
    """synth_rows / analyse_band on this process's GPU for the grid `pnt`
    (a charm_b200.PointGridGL/DH1/DH2): synthesis of rows through
    charm_b200_shs_point_dev on a user grid of those rows' latitudes,
    analysis of the device grid set with set_grid through
    charm_b200_sha_point_dev_band."""
    import torch
    from . import pyharm
    from ._lib import _libcharm as L
    P = ct.c_void_p
    L.charm_b200_shs_point_dev.argtypes = [
        P, ct.c_ulong, ct.c_double, ct.c_double, P, P, ct.c_ulong, ct.c_int,
        ct.c_uint, ct.c_uint, ct.c_uint, P, P]
    L.charm_b200_sha_point_dev_band.argtypes = [
        P, P, ct.c_ulong, ct.c_double, ct.c_double, ct.c_ulong, ct.c_int,
        ct.c_int, P, P, P]
    T = (nmax + 1) * (nmax + 2) // 2
    state = {"grid": None}

    def check(err):
        ok = L.charm_err_isempty(err)
        msg = None if ok else ct.string_at(err.contents.msg).decode()
        L.charm_err_free(err)
        if msg:
            raise pyharm.CHarmError(msg)

    def synth_rows(rows, c, s):
        lat = np.ascontiguousarray(pnt.lat[rows])
        sub = pyharm.PointGrid(lat, pnt.lon, np.asarray(pnt.r)[rows])
        out = torch.empty(len(rows) * pnt.lon.size, dtype=torch.float64,
                          device=c.device)
        if len(rows) == 0:
            return out.view(0, pnt.lon.size)
        err = L.charm_err_init()
        L.charm_b200_shs_point_dev(ct.cast(sub._Point, P), nmax, mu, r,
                                   c.data_ptr(), s.data_ptr(), nmax, 0, 0, 0,
                                   0, out.data_ptr(), ct.cast(err, P))
        check(err)
        return out.view(len(rows), pnt.lon.size)

    def set_grid(d_f):
        state["grid"] = d_f

    def analyse_band(p0, p1):
        d_f = state["grid"]
        c = torch.empty(T, dtype=torch.float64, device=d_f.device)
        s = torch.empty_like(c)
        err = L.charm_err_init()
        L.charm_b200_sha_point_dev_band(ct.cast(pnt._Point, P), d_f.data_ptr(),
                                        nmax, mu, r, nmax, p0, p1,
                                        c.data_ptr(), s.data_ptr(),
                                        ct.cast(err, P))
        check(err)
        return c, s

    return synth_rows, analyse_band, set_grid
