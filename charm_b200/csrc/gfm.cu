// Elementwise steps of the global spectral gravity forward modelling
// (CHarm src/gfm/gfm_sgfm.c, SGFM_GLOBAL): the shape-density function of
// topography power p and density order i on the Gauss--Legendre grid, and
// the accumulation of its analysed coefficients into the potential.  The
// syntheses and analyses between them are the library's grid transforms.
#include "common.cuh"
#include "kernels.h"

namespace cb
{

// rho[k] = rho[k] * (s^p R^i) with s = (shape[k] - R) / R, the power by
// p - 1 repeated products in CHarm's order (gfm_sgfm.c:640-660); with rho
// null (constant density) the power itself is written to out.
__global__ void k_gfm_power(size_t n, const double *__restrict__ shape,
                            double R, unsigned p, double Ri,
                            double *__restrict__ rho, double *__restrict__ out)
{
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    const double s = __ddiv_rn(__dsub_rn(shape[k], R), R);
    double sp = s;
    for (unsigned q = 2; q <= p; q++)
        sp = __dmul_rn(sp, s);
    if (rho)
        rho[k] = __dmul_rn(rho[k], __dmul_rn(sp, Ri));
    else
        out[k] = sp;
}

// pot[m][n] += a[m][n] * v[n] for the degree-na triangle a into the
// degree-np triangle pot (both CHarm's order-major layout); the product is
// rounded before the sum, as CHarm scales the coefficients and then adds
// them (gfm_sgfm.c:700-760).  With scaled non-null the products are also
// written back to a (the potential contribution of this power).
__global__ void k_gfm_accum(long long na, long long np,
                            const double *__restrict__ v, double *ac,
                            double *as, double *pc, double *ps, int scaled)
{
    const long long m = blockIdx.x;
    if (m > na)
        return;
    const long long a0 = tri_col0(na, m);
    const long long p0 = tri_col0(np, m);
    for (long long n = m + threadIdx.x; n <= na; n += blockDim.x)
    {
        const double xc = __dmul_rn(ac[a0 + n - m], v[n]);
        const double xs = __dmul_rn(as[a0 + n - m], v[n]);
        if (scaled)
        {
            ac[a0 + n - m] = xc;
            as[a0 + n - m] = xs;
        }
        if (pc)
        {
            pc[p0 + n - m] = __dadd_rn(pc[p0 + n - m], xc);
            ps[p0 + n - m] = __dadd_rn(ps[p0 + n - m], xs);
        }
    }
}

cudaError_t launch_gfm_power(size_t n, const double *shape, double R,
                             unsigned p, double Ri, double *rho, double *out,
                             cudaStream_t st)
{
    if (n == 0)
        return cudaSuccess;
    const int threads = 256;
    k_gfm_power<<<(unsigned)((n + threads - 1) / threads), threads, 0, st>>>(
        n, shape, R, p, Ri, rho, out);
    return cudaGetLastError();
}

cudaError_t launch_gfm_accum(long long na, long long np, const double *v,
                             double *ac, double *as, double *pc, double *ps,
                             bool scaled, cudaStream_t st)
{
    k_gfm_accum<<<(unsigned)(na + 1), 128, 0, st>>>(na, np, v, ac, as, pc, ps,
                                                    scaled ? 1 : 0);
    return cudaGetLastError();
}

} // namespace cb
