// Quantities accumulated by the synthesis kernels and the post-processing of
// their lumped coefficients (CHarm src/shs/shs_point_kernel.c:176-612 for
// the sums, :1643-1946 for the derivative post-processing and the local
// north-oriented frame of grad2).
#pragma once

namespace cb
{

// KIND 0: one quantity ampl(n) D^DL P (potential and the "guru" single
//         derivatives; DR = radial order, dlon applied at the end);
// KIND 1: full first-order gradient (P, (n+1)P, dP);
// KIND 2: full second-order gradient (P, (n+1)P, dP, (n+1)(n+2)P,
//         (n+1)dP, ddP), src/shs/shs_lc_struct.h:17-72.
template <int KIND, int DL, int DR>
struct Qty
{
    static constexpr int NQ = KIND == 0 ? 1 : (KIND == 1 ? 3 : 6);
    static constexpr int NEEDD = KIND == 0 ? DL : (KIND == 1 ? 1 : 2);
    // sign of the quantity under t -> -t, relative to (-1)^(n+m)
    __device__ static constexpr int parity(int q)
    {
        if (KIND == 0)
            return DL == 1 ? -1 : 1;
        return (q == 2 || q == 4) ? -1 : 1;
    }
    // value of quantity q at degree n (np1 = n + 1)
    __device__ static __forceinline__ double val(int q, double p, double dp,
                                                 double ddp, double np1)
    {
        if (KIND == 0)
        {
            double base = DL == 0 ? p : (DL == 1 ? dp : ddp);
            if (DR == 1)
                return np1 * base;
            if (DR == 2)
                return (np1 * (np1 + 1.0)) * base;
            return base;
        }
        switch (q)
        {
        case 0: return p;
        case 1: return np1 * p;
        case 2: return dp;
        case 3: return (np1 * (np1 + 1.0)) * p;
        case 4: return np1 * dp;
        default: return ddp;
        }
    }
};

template <int NQ, int NP, int K>
struct Acc
{
    // [q][C or S][parity class][k]
    double v[NQ][2][NP][K];
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int q = 0; q < NQ; q++)
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < NP; j++)
#pragma unroll
                    for (int k = 0; k < K; k++)
                        v[q][i][j][k] = 0.0;
    }
    __device__ __forceinline__ void zero_k(int k)
    {
#pragma unroll
        for (int q = 0; q < NQ; q++)
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < NP; j++)
                    v[q][i][j][k] = 0.0;
    }
};

// Derivative post-processing of the lumped coefficients a[q], b[q] of one
// order m at one latitude (tuh = tan(lat) of that latitude, ur = 1/cos,
// u2 = 1/cos^2).  Output order: "pot"/single quantity; grad1 l, r, p;
// grad2 ll, lr, lp, rr, rp, pp (src/shs/shs_grd_fft_lc.c:120-150).
template <int KIND, int DR, int NQ>
__device__ __forceinline__ void lumped_post(double (&a)[NQ], double (&b)[NQ],
                                            double md, double ur, double u2,
                                            double tuh, int dlon)
{
    if (KIND == 0)
    {
        if (DR == 1)
        {
            a[0] = -a[0];
            b[0] = -b[0];
        }
        if (dlon == 1)
        {
            double ta = ur * a[0], tb = ur * b[0];
            a[0] = md * tb;
            b[0] = md * (-ta);
        }
        else if (dlon == 2)
        {
            double ta = u2 * a[0], tb = u2 * b[0];
            a[0] = (md * md) * (-ta);
            b[0] = (md * md) * (-tb);
        }
    }
    else if (KIND == 1)
    {
        a[1] = -a[1];
        b[1] = -b[1];
        double ta = a[0], tb = b[0];
        // dlon1, change of sign, times 1/cos(lat)
        a[0] = ur * (-(md * tb));
        b[0] = ur * (-(md * (-ta)));
    }
    else
    {
        a[1] = -a[1];
        b[1] = -b[1];
        a[4] = -a[4];
        b[4] = -b[4];
        // xx
        a[5] = a[1] + a[5];
        b[5] = b[1] + b[5];
        double a_ = a[0], b_ = b[0];
        // yy
        double mm = md * md;
        double ya = mm * (-a[0]), yb = mm * (-b[0]);
        a[0] = (u2 * ya - tuh * a[2]) + a[1];
        b[0] = (u2 * yb - tuh * b[2]) + b[1];
        // xz
        a[4] = a[4] - a[2];
        b[4] = b[4] - b[2];
        // xy
        double pa = md * b[2], pb = md * (-a[2]);
        double la = md * b_, lb = md * (-a_);
        a[2] = -(ur * pa) - (tuh * ur) * la;
        b[2] = -(ur * pb) - (tuh * ur) * lb;
        // yz
        double ra = md * b[1], rb = md * (-a[1]);
        a[1] = ur * (la - ra);
        b[1] = ur * (lb - rb);
    }
}

// cos(m lon), sin(m lon) with the angle formed exactly (two-product) and the
// rounding residual applied to first order.
__device__ __forceinline__ void sincos_mlon(double md, double lon, double *s,
                                            double *c)
{
    double th = md * lon;
    double tl = fma(md, lon, -th);
    double ss, cc;
    sincos(th, &ss, &cc);
    *c = fma(-ss, tl, cc);
    *s = fma(cc, tl, ss);
}

} // namespace cb
