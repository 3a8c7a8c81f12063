"""Binary128 reference values of the nmax 2190 potential (Kaula
coefficients of seed 2000, r = R) at 16 latitudes of the nmax 2190
Gauss-Legendre grid (both polar caps and the equator band) times 128 of its
4382 longitudes, for the error statement of the single-precision mode and
of the FP64 path against a quad-precision oracle (tests/test_gpu_f32.py).

The values come from CHarm's own quad-precision build (charmq_shs_point of
CHarm 0.4.9 compiled by oracle/build_ref.py, binary128 throughout, its FFT
through oracle/fftw_shim) on a user grid of those latitudes and all 4382 GL
longitudes (so that CHarm takes its FFT path), stored as (hi, lo) float64
pairs.  The latitudes are CHarm's double-precision GL nodes (oracle/_ref).

Run from the repository root after `python oracle/build_ref.py --reference
<CHarm source tree>`:
    python tests/golden/make_quad_n2190.py      (a few seconds)"""
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(
    __file__))))
sys.path.insert(0, ROOT)

from charm_b200.workloads import GM, R_EARTH, kaula  # noqa: E402
from oracle import charm_ref, orc  # noqa: E402

NMAX = 2190
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                   "shs_gl2190_quad16.npz")


def main():
    D = charm_ref.Charm("d")
    _, lat_all, _, _ = D.grid(charm_ref.GL, NMAX, R_EARTH)
    rows = np.unique(np.concatenate([np.arange(3), np.arange(NMAX - 2, NMAX + 1),
                                     np.linspace(3, NMAX - 3, 10).astype(int)]))
    lat = np.array(lat_all[rows])
    L = NMAX + 1
    nlon = 2 * L
    lon_idx = np.sort(np.random.default_rng(2001).choice(nlon, 128,
                                                         replace=False))
    c, s = kaula(NMAX, 2000)
    Q = charm_ref.CharmQ()
    piq = orc.q_from_dd(np.array([math.pi]), np.array([1.2246467991473532e-16]))
    step = orc.q_arith("/", piq, orc.q_from_dd(np.array([float(L)])))
    lonq = orc.q_arith("*", orc.q_from_dd(np.arange(nlon, dtype=np.float64)),
                       step)
    pnt = Q.point_raw(charm_ref.GRID, orc.q_from_dd(lat), lonq,
                      orc.q_from_dd(np.full(lat.size, R_EARTH)))
    hi, lo = Q.shs_point(pnt, Q.shc(NMAX, GM, R_EARTH, c, s), NMAX,
                         lat.size * nlon)
    np.savez_compressed(OUT, nmax=NMAX, seed=2000, rows=rows, lat=lat,
                        lon_idx=lon_idx,
                        f_hi=hi.reshape(lat.size, nlon)[:, lon_idx],
                        f_lo=lo.reshape(lat.size, nlon)[:, lon_idx],
                        source=np.array(os.path.basename(Q.path)))
    print(OUT)


if __name__ == "__main__":
    main()
