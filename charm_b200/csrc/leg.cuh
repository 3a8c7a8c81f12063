// Legendre-recurrence machinery shared by the synthesis and analysis kernels.
//
// Fully normalised associated Legendre functions are generated by the
// three-term recurrence of CHarm (src/leg/leg_func_xnum.h:29-31,
// src/leg/leg_func_anm_bnm.c:46-60)
//     P_n,m = a_nm t P_n-1,m - b_nm P_n-2,m,
// seeded by the sectorial P_m,m.  Where the values are far below the double
// range (high orders near the poles), CHarm switches to X-numbers
// (x * 2^(960 ix), leg_func_xnum.h:64-287) until both recurrence values are
// back in range.  Here each latitude carries (x, y) with one common binary
// exponent E instead: the recurrence is linear, so scaling both terms by the
// same power of two is exact.  While E != 0 ("scaled") the values are below
// 2^-1000 and contribute nothing; every 16 degrees the scaled latitudes are
// renormalised and switch to unscaled arithmetic once their magnitude
// reaches 2^-1000.  Contributions of smaller magnitude are dropped, as
// CHarm's conversion of X-numbers below its range also drops them.
#pragma once

#include "common.cuh"

namespace cb
{

constexpr int LEG_CHUNK = 64;       // degrees staged per shared-memory chunk
constexpr int LEG_FIX_EVERY = 16;   // degrees between renormalisations
constexpr int LEG_SWITCH_EXP = -1000;

// Renormalises the scaled recurrence state (x, y, E) of one latitude.
// Returns true if the latitude switched to unscaled arithmetic now.
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

// Normalises a value with exponent E so that |x| is near 1 (or converts it
// to unscaled form when large enough).  Used on the sectorial seeds.
__device__ __forceinline__ void leg_seed_normalise(double &x, int &E)
{
    double y = 0.0;
    leg_fixup(x, y, E);
}

} // namespace cb
