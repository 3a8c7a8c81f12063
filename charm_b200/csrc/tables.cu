// Recurrence tables of the rescaled Legendre recurrence (see leg.cuh), the
// per-call scaling of the coefficients, and the reduction of the analysis
// partial sums.
//
// For every order m the table kernel walks n = m..nmax once with
//     a_nm = sqrt(2n-1) w,  b_nm = sqrt(n-m-1) sqrt(n+m-1) / sqrt(2n-3) w,
//     w = sqrt(2n+1) / (sqrt(n-m) sqrt(n+m)),   a_m+1,m = sqrt(2m+3)
// (CHarm src/leg/leg_func_anm_bnm.c:14-65, same operations and rounding),
// and e_nm (src/leg/leg_func_enm.c:14-55), and accumulates
// c_n = prod a_km in double-double.  It writes per (n, m)
//     tb = (beta_n, e_n / a_n),  ct = c_n 2^-g_j,
// per (m, chunk j) the multiplier 2^(g_j - g_j-1), and per m the seed
// factor S_m 2^g_0 (S_m from the host, long double).
#include <cstdint>

#include "common.cuh"
#include "kernels.h"
#include "leg.cuh"

namespace cb
{

namespace
{

struct dd
{
    double hi, lo;
};

__device__ __forceinline__ dd dd_mul_d(dd a, double b)
{
    double p = a.hi * b;
    double e = fma(a.hi, b, -p);
    e = fma(a.lo, b, e);
    double s = p + e;
    return {s, e - (s - p)};
}

// a / (b1 * b2) in double-double, rounded to double
__device__ __forceinline__ double div_prod(double a, double b1, double b2)
{
    double ph = b1 * b2;
    double pl = fma(b1, b2, -ph);
    double q = a / ph;
    double r = fma(-q, ph, a) - q * pl;
    return q + r / ph;
}

} // namespace

__global__ void k_tables(long long nmax, const double *__restrict__ r,
                         const double *__restrict__ ri,
                         const double *__restrict__ smm, double2 *tb,
                         double *tc, double *tmul, int ldmul, double *sg)
{
    long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (m > nmax)
        return;
    const long long c0 = tri_col0(nmax, m);
    const long long ncol = nmax - m + 1;
    const int nch = (int)((ncol + LEG_CHUNK - 1) / LEG_CHUNK);
    // c = (c.hi + c.lo) 2^ec; renormalised at every chunk start so that the
    // growth within one chunk (below 2^330 for any m) stays in range
    dd c = {1.0, 0.0};
    int ec = 0;
    double a_prev = 0.0;
    int g_prev = 0, g0 = 0;
    for (int j = 0; j < nch; j++)
    {
        if (j > 0)
        {
            int e = expo_of(c.hi);
            c.hi = scalbn(c.hi, -e);
            c.lo = scalbn(c.lo, -e);
            ec += e;
        }
        long long n0 = m + (long long)j * LEG_CHUNK;
        long long n1 = n0 + LEG_CHUNK - 1;
        if (n1 > nmax)
            n1 = nmax;
        for (long long n = n0; n <= n1; n++)
        {
            double a = 0.0, b = 0.0, e = 0.0;
            if (n == m + 1)
                a = r[2 * m + 3];
            else if (n >= m + 2)
            {
                double w = r[2 * n + 1] * ri[n - m] * ri[n + m];
                a = r[2 * n - 1] * w;
                b = r[n - m - 1] * r[n + m - 1] * ri[2 * n - 3] * w;
            }
            if (n > m)
            {
                e = r[2 * n + 1] * r[n - m] * r[n + m] * ri[2 * n - 1];
                c = dd_mul_d(c, a);
            }
            double beta = (n >= m + 2) ? div_prod(b, a, a_prev) : 0.0;
            double et = (n > m) ? e / a : 0.0;
            tb[c0 + n - m] = make_double2(beta, et);
            tc[c0 + n - m] = c.hi;
            a_prev = a;
        }
        long long nm = n0 + LEG_CHUNK / 2;
        if (nm > n1)
            nm = n1;
        int grel = expo_of(tc[c0 + nm - m]);
        for (long long n = n0; n <= n1; n++)
            tc[c0 + n - m] = scalbn(tc[c0 + n - m], -grel);
        int g = ec + grel;   // absolute power of two of chunk j
        if (j == 0)
        {
            g0 = g;
            tmul[m * ldmul] = 1.0;
        }
        else
            tmul[m * ldmul + j] = scalbn(1.0, g - g_prev);
        g_prev = g;
    }
    sg[2 * m] = scalbn(smm[m], g0);
    sg[2 * m + 1] = (double)g0;
}

// (ct C_nm, ct S_nm) of the degree-nmax triangle from the caller's C, S
// triangles of degree shc_nmax; S_n0 forced to zero (CHarm never reads it,
// src/shs/shs_point_kernel.c:1014-1248).
__global__ void k_scale_cs(long long nmax, long long shc_nmax,
                           const double *__restrict__ c,
                           const double *__restrict__ s,
                           const double *__restrict__ tc, double2 *cs,
                           long long m_lo)
{
    long long m = m_lo + blockIdx.x;
    if (m > nmax)
        return;
    long long c0 = tri_col0(nmax, m);
    long long s0 = tri_col0(shc_nmax, m);
    for (long long n = m + threadIdx.x; n <= nmax; n += blockDim.x)
    {
        double k = tc[c0 + n - m];
        cs[c0 + n - m] = make_double2(k * c[s0 + n - m],
                                      m == 0 ? 0.0 : k * s[s0 + n - m]);
    }
}

// k_scale_cs for one set of a batch: the degree-nmax set in the layout of
// the degree-ntab tables, zero above nmax.
__global__ void k_scale_cs_set(long long ntab, long long nmax,
                               long long shc_nmax,
                               const double *__restrict__ c,
                               const double *__restrict__ s,
                               const double *__restrict__ tc, double2 *cs)
{
    long long m = blockIdx.x;
    if (m > ntab)
        return;
    long long c0 = tri_col0(ntab, m);
    long long s0 = tri_col0(shc_nmax, m);
    for (long long n = m + threadIdx.x; n <= ntab; n += blockDim.x)
    {
        double2 v = make_double2(0.0, 0.0);
        if (n <= nmax)
        {
            double k = tc[c0 + n - m];
            v = make_double2(k * c[s0 + n - m],
                             m == 0 ? 0.0 : k * s[s0 + n - m]);
        }
        cs[c0 + n - m] = v;
    }
}

// Sums the group partials of the analysis, applies ct_n, a constant factor
// and the degree-wise rescaling of src/shc/shc_rescale.c (rescale[n], or
// none when null), and writes C, S in the caller's layout (degree shc_nmax,
// zero above nmax).
__global__ void k_sha_reduce(long long nmax, long long shc_nmax, int ngroups,
                             long long T, const double2 *__restrict__ part,
                             const double *__restrict__ tc,
                             const double *__restrict__ rescale, double scale,
                             double *c, double *s, long long m_lo)
{
    long long m = m_lo + blockIdx.x;
    if (m > shc_nmax)
        return;
    long long d0 = tri_col0(shc_nmax, m);
    long long c0 = tri_col0(nmax, m);
    for (long long n = m + threadIdx.x; n <= shc_nmax; n += blockDim.x)
    {
        double vc = 0.0, vs = 0.0;
        if (m <= nmax && n <= nmax)
        {
            for (int g = 0; g < ngroups; g++)
            {
                double2 v = part[(size_t)g * T + c0 + n - m];
                vc += v.x;
                vs += v.y;
            }
            double k = tc[c0 + n - m] * scale;
            vc *= k;
            vs *= k;
            if (rescale)
            {
                vc *= rescale[n];
                vs *= rescale[n];
            }
        }
        c[d0 + n - m] = vc;
        s[d0 + n - m] = vs;
    }
}

cudaError_t launch_tables(long long nmax, const double *r, const double *ri,
                          const double *smm, double2 *tb, double *tc,
                          double *tmul, int ldmul, double *sg,
                          cudaStream_t st)
{
    int threads = 64;
    int blocks = (int)((nmax + 1 + threads - 1) / threads);
    k_tables<<<blocks, threads, 0, st>>>(nmax, r, ri, smm, tb, tc, tmul,
                                          ldmul, sg);
    return cudaGetLastError();
}

cudaError_t launch_scale_cs_set(long long ntab, long long nmax,
                                long long shc_nmax, const double *c,
                                const double *s, const double *tc,
                                double2 *cs, cudaStream_t st)
{
    // orders above nmax are never read: only columns m <= nmax are written
    k_scale_cs_set<<<(int)(nmax + 1), 128, 0, st>>>(ntab, nmax, shc_nmax, c,
                                                     s, tc, cs);
    return cudaGetLastError();
}

cudaError_t launch_scale_cs(long long nmax, long long shc_nmax,
                            const double *c, const double *s,
                            const double *tc, double2 *cs, cudaStream_t st)
{
    k_scale_cs<<<(int)(nmax + 1), 128, 0, st>>>(nmax, shc_nmax, c, s, tc, cs,
                                                0);
    return cudaGetLastError();
}

cudaError_t launch_scale_cs_orders(long long nmax, long long shc_nmax,
                                   const double *c, const double *s,
                                   const double *tc, double2 *cs,
                                   long long m_lo, long long m_hi,
                                   cudaStream_t st)
{
    if (m_hi <= m_lo)
        return cudaSuccess;
    k_scale_cs<<<(int)(m_hi - m_lo), 128, 0, st>>>(nmax, shc_nmax, c, s, tc,
                                                   cs, m_lo);
    return cudaGetLastError();
}

cudaError_t launch_sha_reduce(long long nmax, long long shc_nmax, int ngroups,
                              long long T, const double2 *part,
                              const double *tc, const double *rescale,
                              double scale, double *c, double *s,
                              cudaStream_t st)
{
    k_sha_reduce<<<(int)(shc_nmax + 1), 128, 0, st>>>(
        nmax, shc_nmax, ngroups, T, part, tc, rescale, scale, c, s, 0);
    return cudaGetLastError();
}

cudaError_t launch_sha_reduce_orders(long long nmax, long long shc_nmax,
                                     int ngroups, long long T,
                                     const double2 *part, const double *tc,
                                     const double *rescale, double scale,
                                     double *c, double *s, long long m_lo,
                                     long long m_hi, cudaStream_t st)
{
    if (m_hi <= m_lo)
        return cudaSuccess;
    k_sha_reduce<<<(int)(m_hi - m_lo), 128, 0, st>>>(
        nmax, shc_nmax, ngroups, T, part, tc, rescale, scale, c, s, m_lo);
    return cudaGetLastError();
}

} // namespace cb
