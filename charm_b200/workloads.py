"""Seeded synthetic inputs of the benchmark workloads.

Coefficients follow Kaula's rule: C_nm, S_nm ~ N(0, 1) * sigma_n with
sigma_n = 1e-5 n^-2 / sqrt(2n + 1) (or 1e-5 n^-2 for the degree-10800
workload), C_00 = 1, degree 1 and S_n0 zero, drawn with numpy's PCG64 in
CHarm's order-major triangle layout (C_nm at m (2N + 3 - m)/2 + n - m).
"""
import numpy as np

GM = 3.986004418e14
R_EARTH = 6378136.3


def tri_size(nmax):
    return (nmax + 1) * (nmax + 2) // 2


def tri_degrees(nmax):
    """Degree n of every entry of the order-major triangle."""
    return np.concatenate([np.arange(m, nmax + 1) for m in range(nmax + 1)])


def tri_orders(nmax):
    return np.concatenate([np.full(nmax + 1 - m, m) for m in range(nmax + 1)])


def kaula(nmax, seed, sqrt_scaling=True):
    """(c, s) triangles of degree nmax."""
    rng = np.random.default_rng(seed)
    T = tri_size(nmax)
    c = rng.standard_normal(T)
    s = rng.standard_normal(T)
    n = tri_degrees(nmax).astype(np.float64)
    m = tri_orders(nmax)
    with np.errstate(divide="ignore"):
        sig = 1e-5 * n ** -2.0
        if sqrt_scaling:
            sig = sig / np.sqrt(2.0 * n + 1.0)
    sig[n < 2] = 0.0
    c *= sig
    s *= sig
    c[0] = 1.0
    s[m == 0] = 0.0
    return c, s


def rel_rms(x, ref):
    x = np.asarray(x, np.float64).ravel()
    ref = np.asarray(ref, np.float64).ravel()
    den = np.sqrt(np.mean(ref ** 2))
    return float(np.sqrt(np.mean((x - ref) ** 2)) / den) if den > 0 else \
        float(np.sqrt(np.mean((x - ref) ** 2)))


def coef_rel_rms(c, s, ref_c, ref_s):
    """Relative RMS difference of a whole coefficient set (C and S together):
    sqrt(sum dC^2 + dS^2) / sqrt(sum C^2 + S^2).  Normalising S on its own
    would measure the double-precision noise floor of the smallest
    coefficients instead of the agreement of the transforms."""
    d = np.concatenate([np.ravel(c) - np.ravel(ref_c),
                        np.ravel(s) - np.ravel(ref_s)])
    r = np.concatenate([np.ravel(ref_c), np.ravel(ref_s)])
    return float(np.sqrt(np.sum(d * d) / np.sum(r * r)))
