// Quadrature grids on the GPU: Gauss--Legendre nodes by Newton iteration on
// P_L (CHarm src/crd/crd_point_gl_chunk.c:122-173) and Driscoll--Healy
// weights by the Chebyshev-accelerated sum (src/crd/crd_point_dh_lat_w_chunk.c
// :49-92).  One thread per northern latitude; the southern half follows by
// symmetry exactly as in CHarm.
#include <cfloat>

#include "common.cuh"
#include "kernels.h"

namespace cb
{

__device__ __forceinline__ bool nearly_zero(double a, double eps)
{
    // misc_is_nearly_equal(a, 0, eps)
    return a == 0.0 || fabs(a) <= eps;
}

__global__ void k_gl_nodes(unsigned long nmax, double *lat, double *w,
                           unsigned *status)
{
    const unsigned long L = nmax + 1;
    const size_t nlat = L;
    const size_t nnorth = (nlat + 1) / 2;
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nnorth)
        return;
    const double PI = 3.14159265358979323846;
    const double Lf = (double)L;
    const double c1 = Lf + 0.5;
    double z = cos(PI * ((double)(i + 1) - 0.25) / c1), z1, p1, p2, p3, pp;
    unsigned long it = 0;
    do
    {
        p1 = 1.0;
        p2 = 0.0;
        for (unsigned long j = 1; j <= L; j++)
        {
            p3 = p2;
            p2 = p1;
            p1 = ((double)(2 * j - 1) * z * p2 - (double)(j - 1) * p3) /
                 (double)j;
        }
        pp = Lf * (z * p1 - p2) / (z * z - 1.0);
        z1 = z;
        z -= p1 / pp;
        it++;
    } while (fabs(z - z1) > DBL_EPSILON && it < 1000);
    if (it >= 1000 || !isfinite(z))
        atomicOr(status, DEV_ERR_BAD_ARGS);
    size_t north = i, south = nlat - 1 - i;
    lat[south] = -asin(z);
    w[south] = 2.0 / ((1.0 - z * z) * pp * pp);
    if (nearly_zero(lat[south], 100.0 * DBL_EPSILON))
        return;
    lat[north] = -lat[south];
    w[north] = w[south];
}

__global__ void k_dh_nodes(unsigned long nmax, double *lat, double *w)
{
    const unsigned long L = nmax + 1;
    const size_t nlat = 2 * L;
    const size_t nnorth = nlat / 2 + 1;
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nnorth)
        return;
    const double PI = 3.14159265358979323846;
    const double PI_2 = 1.57079632679489661923;
    const double Lf = (double)L;
    const double c = 2.0 / Lf;
    const double M_PI_2L = PI / (2.0 * Lf);
    double clti = M_PI_2L * (double)i;
    size_t north = i, south = nlat - i;
    lat[north] = PI_2 - clti;
    double sclti = sin(clti);
    if (nmax == 0)
        w[north] = c * sclti;
    else
    {
        double s0 = 0.0, s1 = sclti, cc2 = 2.0 * cos(clti), s2, wt = s1;
        for (unsigned long k = 1; k < L; k++)
        {
            s2 = cc2 * s1 - s0;
            s0 = s1;
            s1 = s2;
            s2 = cc2 * s1 - s0;
            wt += s2 / (double)(2 * k + 1);
            s0 = s1;
            s1 = s2;
        }
        w[north] = c * sclti * wt;
    }
    if (i == 0)
        return;
    if (nearly_zero(lat[north], 100.0 * DBL_EPSILON))
        return;
    w[south] = w[north];
    lat[south] = -lat[north];
}

cudaError_t launch_gl_nodes(unsigned long nmax, double *lat, double *w,
                            unsigned *status, cudaStream_t st)
{
    size_t nnorth = (nmax + 2) / 2;
    k_gl_nodes<<<(int)((nnorth + 127) / 128), 128, 0, st>>>(nmax, lat, w,
                                                             status);
    return cudaGetLastError();
}

cudaError_t launch_dh_nodes(unsigned long nmax, double *lat, double *w,
                            cudaStream_t st)
{
    size_t nnorth = nmax + 2;
    k_dh_nodes<<<(int)((nnorth + 127) / 128), 128, 0, st>>>(nmax, lat, w);
    return cudaGetLastError();
}

} // namespace cb
