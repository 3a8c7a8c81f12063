// Legendre-recurrence machinery shared by the synthesis and analysis kernels.
//
// CHarm generates fully normalised associated Legendre functions with
//     P_n,m = a_nm t P_n-1,m - b_nm P_n-2,m
// (src/leg/leg_func_xnum.h:29-31, leg_func_anm_bnm.c:46-60), three FP64
// operations per degree and latitude.  The kernels here run the same
// recurrence on R_n = P_n / c_n with c_n = prod_{k=m+1..n} a_km:
//     R_n = t R_n-1 - beta_n R_n-2,   beta_n = b_nm / (a_nm a_n-1,m),
// two operations per step; c_n is folded into the coefficients
// (c_n C_nm, c_n S_nm) for synthesis and applied to the sums for analysis.
// c_n grows like 2^(n-m), so the degrees are cut into chunks of LEG_CHUNK
// and every chunk j carries its own power of two: ct_n = c_n 2^-g_j and
// R~_n = R_n 2^g_j, with R~ multiplied by 2^(g_j+1 - g_j) at chunk entry.
// beta, ct and the chunk multipliers depend only on (n, m) and are built
// once per maximum degree (tables.cu) in double-double arithmetic from the
// same a_nm, b_nm as CHarm, then rounded.
//
// Values far below the double range (high orders near the poles) are
// handled like CHarm's X-numbers (leg_func_xnum.h:64-287), but with one
// binary exponent E shared by the two recurrence terms of a latitude: the
// recurrence is linear, so scaling both terms by a power of two is exact.
// While E != 0 ("scaled") the latitude contributes nothing; at each chunk
// boundary scaled latitudes are renormalised and switch to unscaled
// arithmetic once |R~| reaches 2^LEG_SWITCH_EXP.  The contributions dropped
// this way are below 2^-440 relative to the coefficients, as CHarm drops
// X-numbers below its range.
#pragma once

#include "common.cuh"

namespace cb
{

constexpr int LEG_CHUNK = 64;        // degrees per staged chunk
constexpr int LEG_SWITCH_EXP = -600;

// Renormalises the scaled state (x, y, E) of one latitude; returns true if
// it switched to unscaled arithmetic now.
__device__ __forceinline__ bool leg_fixup(double &x, double &y, int &E)
{
    if (E == 0)
        return false;
    double mx = fmax(fabs(x), fabs(y));
    if (!(mx > 0.0) || !isfinite(mx))
        return false;
    int e = expo_of(mx);
    int tot = E + e;
    if (tot >= LEG_SWITCH_EXP)
    {
        x = scalbn(x, E);
        y = scalbn(y, E);
        E = 0;
        return true;
    }
    x = scalbn(x, -e);
    y = scalbn(y, -e);
    E = tot;
    return false;
}

__device__ __forceinline__ void leg_seed_normalise(double &x, int &E)
{
    double y = 0.0;
    leg_fixup(x, y, E);
}

// u^m = mant * 2^ex for u > 0 by binary powering with the exponent carried
// separately (no underflow for any m); relative error below 2 log2(m) ulp.
__device__ __forceinline__ void pow_me(double u, long long m, double &mant,
                                       int &ex)
{
    int eu;
    double b = frexp(fabs(u), &eu);
    double r = 1.0;
    int er = 0, eb = 0;
    long long k = m;
    while (k)
    {
        if (k & 1)
        {
            int e;
            r = frexp(r * b, &e);
            er += eb + e;
        }
        k >>= 1;
        if (k)
        {
            int e;
            b = frexp(b * b, &e);
            eb = 2 * eb + e;
        }
    }
    mant = (u < 0.0 && (m & 1)) ? -r : r;
    ex = er + (int)(m * (long long)eu);
}

// Seed R~_mm of order m at one latitude: sg = (S_m 2^g0, unused) with
// S_m = P_mm(u) / u^m (sqrt(3) prod d_k, src/leg/leg_func_prepare.c) and g0
// the chunk-0 power of two; rho^(m+1+dorder) for r != R.
__device__ __forceinline__ void leg_seed(double sigma, double u, double rho,
                                         bool use_rho, long long m,
                                         int dorder, double &x, int &E)
{
    double um;
    int eu;
    pow_me(u, m, um, eu);
    x = sigma * um;
    E = eu;
    if (use_rho)
    {
        double rm;
        int er;
        pow_me(rho, m + 1 + dorder, rm, er);
        x *= rm;
        E += er;
    }
    leg_seed_normalise(x, E);
}

} // namespace cb
