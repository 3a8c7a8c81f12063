"""Binary128 oracle values of the nmax 10800 potential at 64 seeded
latitudes x 64 of the Gauss-Legendre longitudes, for the FP64 GPU path's
ultra-high-degree check (tests/test_gpu_n10800.py).

Full-grid quad synthesis at nmax 10800 is out of reach on a CPU, so the
check runs on a user grid: 64 latitudes (56 uniform on the sphere, 8 within
0.6 degrees of the poles, where the sectorial terms underflow double by
thousands of orders of magnitude) times all 21602 GL longitudes (so the GPU
takes the FFT path), of which 64 are compared.

Coefficients: Kaula decay sigma_n = 1e-5 n^-2 (C00 = 1, degree 1 zero,
S_n0 = 0), standard normals from numpy's default_rng(3000), the order-major
triangle of charm_b200.workloads.kaula(10800, 3000, sqrt_scaling=False).
The oracle sums in binary128 (oracle/orc.c built with -DORC_QUAD) and
returns (hi, lo) float64 pairs.

Run from the repository root: python tests/golden/make_quad_n10800.py
(about 5 minutes on 8 cores)."""
import math
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(
    __file__))))
sys.path.insert(0, ROOT)

from charm_b200.workloads import GM, R_EARTH, kaula  # noqa: E402
from oracle import orc  # noqa: E402

NMAX = 10800
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                   "shs_gl10800_quad64.npz")


def points():
    """The 64 latitudes (north to south) and the indices of the 64 compared
    longitudes among the 2 (nmax + 1) GL longitudes."""
    rng = np.random.default_rng(3001)
    lat = np.arcsin(rng.uniform(-1.0, 1.0, 56))
    polar = math.pi / 2 - rng.uniform(0.0, 0.01, 8)
    polar[4:] *= -1.0
    lat = np.sort(np.concatenate([lat, polar]))[::-1].copy()
    nlon = 2 * (NMAX + 1)
    lon_idx = np.sort(np.random.default_rng(3002).choice(nlon, 64,
                                                          replace=False))
    return lat, lon_idx


def main():
    lat, lon_idx = points()
    c, s = kaula(NMAX, 3000, sqrt_scaling=False)
    L = NMAX + 1
    nrow = lat.size
    cq = orc.q_from_dd(c)
    sq = orc.q_from_dd(s)
    latq = orc.q_from_dd(lat)
    ones = orc.q_from_dd(np.ones(nrow))
    out = [np.zeros((nrow * L, 2)) for _ in range(4)]
    t0 = time.time()
    orc.lib("q").orc_q_shs_lumped(
        NMAX, NMAX, orc._ptr(cq), orc._ptr(sq), nrow, orc._ptr(latq),
        orc._ptr(ones), orc._ptr(ones.copy()),
        orc._ptr(np.zeros(nrow, np.int32)), 0, 0, 0, 0,
        *[orc._ptr(o) for o in out])
    t1 = time.time()
    # longitudes j pi / (nmax + 1) and GM / R in binary128
    piq = orc.q_from_dd(np.array([math.pi]), np.array([1.2246467991473532e-16]))
    step = orc.q_arith("/", piq, orc.q_from_dd(np.array([float(L)])))
    lonq = orc.q_arith("*", orc.q_from_dd(lon_idx.astype(np.float64)), step)
    mur = orc.q_arith("/", orc.q_from_dd(np.array([GM])),
                      orc.q_from_dd(np.array([R_EARTH])))
    f = np.zeros((nrow * lon_idx.size, 2))
    orc.lib("q").orc_q_lonsum(nrow, L, orc._ptr(out[0]), orc._ptr(out[1]),
                              lon_idx.size, orc._ptr(lonq), orc._ptr(mur),
                              orc._ptr(f))
    hi, lo = orc.q_to_dd(f)
    np.savez_compressed(OUT, nmax=NMAX, seed=3000, lat=lat, lon_idx=lon_idx,
                        f_hi=hi.reshape(nrow, -1), f_lo=lo.reshape(nrow, -1))
    print("lumped %.0f s, longitude sums %.0f s -> %s" % (
        t1 - t0, time.time() - t1, OUT))


if __name__ == "__main__":
    main()
