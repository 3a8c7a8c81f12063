"""CHarm's binary coefficient files (src/shc/shc_read_bin.c,
shc_write_bin.c) through libcharm.so, without a GPU: round trips, reading
fewer degrees than the file holds, the maximum-degree query, the error
cases, and byte-identical files / equal coefficients against CHarm's own
build where oracle/_ref has it."""
import ctypes as ct
import os

import numpy as np
import pytest

from oracle import charm_ref

NMAX_MODEL = (1 << 64) - 2
NMAX_ERROR = (1 << 64) - 1


@pytest.fixture(scope="module")
def L():
    from charm_b200._lib import _libcharm, _Err, _Shc
    P = ct.POINTER
    _libcharm.charm_shc_read_bin.restype = ct.c_ulong
    _libcharm.charm_shc_read_bin.argtypes = [ct.c_char_p, ct.c_ulong,
                                             P(_Shc), P(_Err)]
    _libcharm.charm_shc_write_bin.restype = None
    _libcharm.charm_shc_write_bin.argtypes = [P(_Shc), ct.c_ulong,
                                              ct.c_char_p, P(_Err)]
    return _libcharm


def shc_of(nmax, mu, r, seed):
    import charm_b200 as cb
    T = (nmax + 1) * (nmax + 2) // 2
    rng = np.random.default_rng(seed)
    c = rng.standard_normal(T)
    s = rng.standard_normal(T)
    s[:nmax + 1] = 0.0             # S_n0 = 0 as CHarm stores it
    return cb.Shc(nmax, mu, r, c, s)


def read(L, path, nmax, shc):
    err = L.charm_err_init()
    n = L.charm_shc_read_bin(path.encode(), nmax, shc._Shc if shc else None,
                             err)
    msg = None if L.charm_err_isempty(err) else \
        ct.string_at(err.contents.msg).decode()
    L.charm_err_free(err)
    return n, msg


def write(L, shc, nmax, path):
    err = L.charm_err_init()
    L.charm_shc_write_bin(shc._Shc, nmax, path.encode(), err)
    msg = None if L.charm_err_isempty(err) else \
        ct.string_at(err.contents.msg).decode()
    L.charm_err_free(err)
    return msg


def tri(nmax, a, n):
    """degree-n triangle (order-major) of the degree-nmax triangle a"""
    out = []
    for m in range(n + 1):
        c0 = m * (2 * nmax + 3 - m) // 2
        out.append(a[c0:c0 + n + 1 - m])
    return np.concatenate(out)


def test_round_trip_and_partial_reads(L, tmp_path):
    import charm_b200 as cb
    path = str(tmp_path / "model.shcs")
    src = shc_of(40, 3.986e14, 6378136.3, 7)
    assert write(L, src, 40, path) is None
    # header: nmax (unsigned long), mu, r, then C and S columns
    assert os.path.getsize(path) == 8 + 16 + 2 * 8 * (41 * 42 // 2)
    assert read(L, path, NMAX_MODEL, None) == (40, None)
    dst = cb.Shc(40, 1.0, 1.0)
    assert read(L, path, 40, dst) == (40, None)
    assert dst.mu == src.mu and dst.r == src.r
    assert np.array_equal(dst.c, src.c) and np.array_equal(dst.s, src.s)
    # fewer degrees into a larger triangle: the rest is zero
    dst = cb.Shc(50, 1.0, 1.0)
    assert read(L, path, 25, dst) == (40, None)
    assert np.array_equal(tri(50, dst.c, 25), tri(40, src.c, 25))
    assert np.array_equal(tri(50, dst.s, 25), tri(40, src.s, 25))
    assert np.count_nonzero(dst.c) == np.count_nonzero(tri(40, src.c, 25))
    # writing fewer degrees than the triangle holds
    path2 = str(tmp_path / "model25.shcs")
    assert write(L, src, 25, path2) is None
    dst = cb.Shc(25, 1.0, 1.0)
    assert read(L, path2, 25, dst) == (25, None)
    assert np.array_equal(dst.c, tri(40, src.c, 25))


def test_errors(L, tmp_path):
    import charm_b200 as cb
    n, msg = read(L, str(tmp_path / "missing.shcs"), 10, cb.Shc(10, 1, 1))
    assert n == NMAX_ERROR and "Couldn't open" in msg
    path = str(tmp_path / "m.shcs")
    assert write(L, shc_of(10, 1.0, 1.0, 3), 10, path) is None
    n, msg = read(L, path, 11, cb.Shc(11, 1, 1))
    assert n == 10 and "Not enough coefficients" in msg
    n, msg = read(L, path, 10, cb.Shc(9, 1, 1))
    assert n == 10 and "Too low maximum degree" in msg
    # CHarm's writer creates the file before it checks nmax
    assert "Not enough coefficients" in write(L, shc_of(5, 1, 1, 1), 6, path)
    assert os.path.getsize(path) == 0
    # a truncated file
    assert write(L, shc_of(10, 1.0, 1.0, 3), 10, path) is None
    with open(path, "r+b") as fh:
        fh.truncate(8 + 16 + 40)
    n, msg = read(L, path, 10, cb.Shc(10, 1, 1))
    assert n == 10 and "Failed to read the \"C\" coefficients" in msg


@pytest.mark.skipif(not charm_ref.available("d"),
                    reason="oracle/_ref has no double CHarm build")
def test_files_match_charm(L, tmp_path):
    """CHarm's writer and this one produce the same bytes; each reads the
    other's file to the same coefficients."""
    import charm_b200 as cb
    C = charm_ref.Charm("d")
    P = ct.POINTER
    C.fn("shc_write_bin").argtypes = [P(C.Shc), ct.c_ulong, ct.c_char_p,
                                      P(C.Err)]
    C.fn("shc_read_bin").argtypes = [ct.c_char_p, ct.c_ulong, P(C.Shc),
                                     P(C.Err)]
    C.fn("shc_read_bin").restype = ct.c_ulong
    src = shc_of(60, 3.986e14, 6378136.3, 11)
    mine, theirs = str(tmp_path / "mine.shcs"), str(tmp_path / "theirs.shcs")
    assert write(L, src, 50, mine) is None
    csrc = C.shc(60, src.mu, src.r, src.c, src.s)
    C.fn("shc_write_bin")(csrc.ptr, 50, theirs.encode(), C.err)
    C.check()
    assert open(mine, "rb").read() == open(theirs, "rb").read()
    out = C.shc(60, 1.0, 1.0, np.zeros(src.c.size), np.zeros(src.c.size))
    assert C.fn("shc_read_bin")(mine.encode(), 40, out.ptr, C.err) == 50
    C.check()
    dst = cb.Shc(60, 1.0, 1.0)
    assert read(L, theirs, 40, dst) == (50, None)
    assert np.array_equal(dst.c, out.keep[0]) and np.array_equal(dst.s, out.keep[1])


@pytest.mark.gpu
def test_read_bin_streamed_to_device(L, tmp_path):
    """charm_b200_shc_read_bin_dev: the file's triangles streamed into
    device triangles equal charm_shc_read_bin's host triangles bit for bit
    (a degree-2190 file read whole, read to a lower degree into a larger
    triangle; a file of several staging chunks), and it rejects what
    charm_shc_read_bin rejects."""
    import charm_b200 as cb
    import torch
    P = ct.c_void_p
    L.charm_b200_shc_read_bin_dev.restype = ct.c_ulong
    L.charm_b200_shc_read_bin_dev.argtypes = [
        ct.c_char_p, ct.c_ulong, ct.c_ulong, P, P, ct.POINTER(ct.c_double),
        ct.POINTER(ct.c_double), P]
    path = str(tmp_path / "big.shcs")
    src = shc_of(2190, 3.986004418e14, 6378136.3, 21)
    assert write(L, src, 2190, path) is None

    def dev_read(nmax, shc_nmax):
        T = (shc_nmax + 1) * (shc_nmax + 2) // 2
        dc = torch.full((T,), 7.0, dtype=torch.float64, device="cuda")
        ds = torch.full((T,), 7.0, dtype=torch.float64, device="cuda")
        mu, r = ct.c_double(), ct.c_double()
        err = L.charm_err_init()
        n = L.charm_b200_shc_read_bin_dev(path.encode(), nmax, shc_nmax,
                                          dc.data_ptr(), ds.data_ptr(),
                                          ct.byref(mu), ct.byref(r),
                                          ct.cast(err, P))
        msg = None if L.charm_err_isempty(err) else \
            ct.string_at(err.contents.msg).decode()
        L.charm_err_free(err)
        return n, msg, dc.cpu().numpy(), ds.cpu().numpy(), mu.value, r.value

    n, msg, c, s, mu, r = dev_read(2190, 2190)
    assert (n, msg) == (2190, None)
    assert np.array_equal(c, src.c) and np.array_equal(s, src.s)
    assert mu == src.mu and r == src.r
    n, msg, c, s, mu, r = dev_read(1000, 1500)
    assert (n, msg) == (2190, None)
    host = cb.Shc(1500, 1.0, 1.0)
    assert read(L, path, 1000, host) == (2190, None)
    assert np.array_equal(c, host.c) and np.array_equal(s, host.s)
    n, msg, *_ = dev_read(2191, 2191)
    assert n == NMAX_ERROR and "Not enough coefficients" in msg
    n, msg, *_ = dev_read(100, 50)
    assert n == NMAX_ERROR and "shc_nmax" in msg
