"""Packs CHarm's own golden test vectors for the point-synthesis path into
small fixtures under tests/golden/.

Run once in a container that has the CHarm source tree (its path is the
first argument); the tests only read the .npz files
this writes, so the GPU machine never needs the reference tree.

Sources (CHarm 0.4.9):
  data/tests/{double,quad}/shs_p_*.txt   point synthesis golden outputs
                                          (tests/check_shs_point_all.c)
  data/tests/{double,quad}/shs_c_nx*.txt cell synthesis golden outputs
                                          (tests/check_shs_cell.c)
  data/tests/{double,quad}/sha_c_nx*.txt cell analysis golden outputs
                                          (tests/check_sha_cell.c)
  data/tests/{double,quad}/crd_*.txt     GL/DH grid nodes and weights
                                          (tests/check_crd_point_quad.c)
  data/tests/double/gfm_sgfm_g_*.txt     degree amplitudes of the global
                                          gravity forward modelling tests
                                          (tests/check_gfm_sgfm_all.c.in)
  data/input/EGM96-degree10-mtx.txt      input coefficients of those tests
                                          (tests/parameters.h:46-48)
  data/input/MoonTopo2600p_to10-tbl.txt, the lunar shape and density
  data/input/moon-rho{0,1}_to10.tbl      inputs of the gfm tests
                                          (tests/parameters.h:298-306)

Outputs:
  charm_golden_double.npz  every hot-path golden file as float64
  charm_golden_quad.npz    the binary128 golden files of the potential (no
                           gradient suffix) and of the grids, each stored as
                           a (2, n) float64 (hi, lo) pair
  egm96_degree10.npz       nmax, mu, R and the C, S triangles (order-major)
                           parsed both as float64 and as (hi, lo) pairs
"""
import os
import re
import sys
from decimal import Decimal, getcontext

import numpy as np

getcontext().prec = 60


def dd(s):
    """Decimal string -> (hi, lo) float64 pair carrying ~32 digits."""
    d = Decimal(s)
    hi = float(d)
    lo = float(d - Decimal(hi))
    return hi, lo


def pack(path, table):
    """One concatenated array plus a name index (keeps the zip small)."""
    names = sorted(table)
    sizes = [table[k].shape[-1] for k in names]
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    data = np.concatenate([table[k] for k in names], axis=-1)
    np.savez_compressed(path, names=np.array("\n".join(names)),
                        offsets=offsets, data=data)


HOT = re.compile(r"^(shs_p_|shs_c_nx|sha_c_nx|crd_nx|gfm_sgfm_g_).*\.txt$")
GRAD_SUFFIX = re.compile(r"_(x|y|z|xx|xy|xz|yy|yz|zz|guru\d+)\.txt$")


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <CHarm source tree>")
    ref = sys.argv[1]
    here = os.path.dirname(os.path.abspath(__file__))
    dbl = {}
    for name in sorted(os.listdir(os.path.join(ref, "data/tests/double"))):
        if not HOT.match(name):
            continue
        with open(os.path.join(ref, "data/tests/double", name)) as fh:
            vals = [float(t) for t in fh.read().split()]
        dbl[name[:-4]] = np.array(vals, dtype=np.float64)
    pack(os.path.join(here, "charm_golden_double.npz"), dbl)

    quad = {}
    for name in sorted(os.listdir(os.path.join(ref, "data/tests/quad"))):
        if not HOT.match(name) or GRAD_SUFFIX.search(name):
            continue
        with open(os.path.join(ref, "data/tests/quad", name)) as fh:
            pairs = [dd(t) for t in fh.read().split()]
        quad[name[:-4]] = np.array(pairs, dtype=np.float64).T.copy()
    pack(os.path.join(here, "charm_golden_quad.npz"), quad)

    # EGM96 degree-10 coefficients in the "mtx" layout
    # (src/shc/shc_read_mtx.c:165-250): row >= col -> C[col][row - col],
    # otherwise S[row + 1][col - row - 1].
    with open(os.path.join(ref, "data/input/EGM96-degree10-mtx.txt")) as fh:
        toks = fh.read().split()
    nmax = int(toks[0])
    mu_s, r_s = toks[1], toks[2]
    vals = toks[3:]
    T = (nmax + 1) * (nmax + 2) // 2
    col0 = np.cumsum([0] + [nmax + 1 - m for m in range(nmax)])
    c = np.zeros(T)
    s = np.zeros(T)
    cq = np.zeros((2, T))
    sq = np.zeros((2, T))
    k = 0
    for row in range(nmax + 1):
        for col in range(nmax + 1):
            v = vals[k]
            k += 1
            if row >= col:
                i = col0[col] + row - col
                c[i] = float(v)
                cq[:, i] = dd(v)
            else:
                m = row + 1
                i = col0[m] + col - m
                s[i] = float(v)
                sq[:, i] = dd(v)
    np.savez_compressed(
        os.path.join(here, "egm96_degree10.npz"),
        nmax=np.array(nmax), mu=np.array(float(mu_s)), r=np.array(float(r_s)),
        mu_q=np.array(dd(mu_s)), r_q=np.array(dd(r_s)),
        c=c, s=s, c_q=cq, s_q=sq)
    # the gfm tests' inputs in the "tbl" layout
    # (src/shc/shc_read_tbl.c: "nmax mu r", then lines "n m C S")
    moon = {}
    for key, name in (("shape", "MoonTopo2600p_to10-tbl.txt"),
                      ("rho0", "moon-rho0_to10.tbl"),
                      ("rho1", "moon-rho1_to10.tbl")):
        with open(os.path.join(ref, "data/input", name)) as fh:
            toks = fh.read().split()
        nm = int(toks[0])
        T = (nm + 1) * (nm + 2) // 2
        cc = np.zeros(T)
        ss = np.zeros(T)
        vals = toks[3:]
        for k in range(0, len(vals), 4):
            n, m = int(vals[k]), int(vals[k + 1])
            i = m * (2 * nm + 3 - m) // 2 + n - m
            cc[i] = float(vals[k + 2])
            ss[i] = float(vals[k + 3])
        moon[key + "_nmax"] = np.array(nm)
        moon[key + "_mu"] = np.array(float(toks[1]))
        moon[key + "_r"] = np.array(float(toks[2]))
        moon[key + "_c"] = cc
        moon[key + "_s"] = ss
    np.savez_compressed(os.path.join(here, "moon_gfm_inputs.npz"), **moon)
    print(len(dbl), "double files;", len(quad), "quad files")


if __name__ == "__main__":
    main()
