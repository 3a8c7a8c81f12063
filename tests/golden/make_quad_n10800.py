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
The values come from CHarm's own quad-precision build (charmq_shs_point of
CHarm 0.4.9 compiled by oracle/build_ref.py, binary128 throughout, its FFT
through oracle/fftw_shim), stored as (hi, lo) float64 pairs.

Run from the repository root after `python oracle/build_ref.py --reference
<CHarm source tree> --variants q`:
    python tests/golden/make_quad_n10800.py     (a few minutes on 8 cores)"""
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
    from oracle import charm_ref
    lat, lon_idx = points()
    c, s = kaula(NMAX, 3000, sqrt_scaling=False)
    L = NMAX + 1
    nlon = 2 * L
    nrow = lat.size
    Q = charm_ref.CharmQ()
    # longitudes j pi / (nmax + 1) exact in binary128: CHarm checks that a
    # grid's longitudes increase linearly within its quad threshold before
    # it takes the FFT path (src/shs/shs_grd_point_fft_check.c)
    piq = orc.q_from_dd(np.array([math.pi]), np.array([1.2246467991473532e-16]))
    step = orc.q_arith("/", piq, orc.q_from_dd(np.array([float(L)])))
    lonq = orc.q_arith("*", orc.q_from_dd(np.arange(nlon, dtype=np.float64)),
                       step)
    pnt = Q.point_raw(charm_ref.GRID, orc.q_from_dd(lat), lonq,
                      orc.q_from_dd(np.full(nrow, R_EARTH)))
    shc = Q.shc(NMAX, GM, R_EARTH, c, s)
    t0 = time.time()
    hi, lo = Q.shs_point(pnt, shc, NMAX, nrow * nlon)
    hi = hi.reshape(nrow, nlon)[:, lon_idx]
    lo = lo.reshape(nrow, nlon)[:, lon_idx]
    np.savez_compressed(OUT, nmax=NMAX, seed=3000, lat=lat, lon_idx=lon_idx,
                        f_hi=hi, f_lo=lo, source=np.array(Q.path.split("/")[-1]))
    print("charmq_shs_point %.0f s -> %s" % (time.time() - t0, OUT))


if __name__ == "__main__":
    main()
