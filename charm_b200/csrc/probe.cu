// FP64 throughput probe: the denominator of the roofline of the Legendre
// kernels (the measured-peaks file of this machine carries no FP64 figure).
// Every thread runs 8 independent fused multiply-add chains so that the
// FP64 pipe, not the chain latency, is the limit.
#include "kernels.h"

namespace cb
{

__global__ void k_fp64_fma(long long iters, double seed, double *sink)
{
    double a0 = seed + threadIdx.x, a1 = a0 + 1.0, a2 = a0 + 2.0,
           a3 = a0 + 3.0, a4 = a0 + 4.0, a5 = a0 + 5.0, a6 = a0 + 6.0,
           a7 = a0 + 7.0;
    const double b = 0.999999999, c = 1e-9;
    for (long long i = 0; i < iters; i++)
    {
        a0 = fma(a0, b, c);
        a1 = fma(a1, b, c);
        a2 = fma(a2, b, c);
        a3 = fma(a3, b, c);
        a4 = fma(a4, b, c);
        a5 = fma(a5, b, c);
        a6 = fma(a6, b, c);
        a7 = fma(a7, b, c);
    }
    double r = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (r == 12345.678) // never true; keeps the chains alive
        sink[threadIdx.x] = r;
}

cudaError_t launch_fp64_probe(long long iters, int blocks, int threads,
                              double *sink, cudaStream_t st)
{
    k_fp64_fma<<<blocks, threads, 0, st>>>(iters, 0.5, sink);
    return cudaGetLastError();
}

} // namespace cb
