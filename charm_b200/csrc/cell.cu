// Block-mean values in cells: CHarm's cell synthesis on grids and at
// scattered cells (src/shs/shs_cell_grd.c:42-884, shs_cell_sctr.c,
// shs_cell_kernel.c:16-476) and its approximate-quadrature analysis of cell
// grids (src/sha/sha_cell.c:37-1487).
//
// A cell row [latmin, latmax] integrates the Legendre functions over
// latitude, I_nm = int P_nm(sin phi) cos phi dphi.  CHarm evaluates the
// integrals by the recurrences of src/leg/leg_func_gm_hm.c (Fukushima 2014,
// after Paul 1978), with t = sin and u = cos of the two boundaries:
//   I_mm    = g_m I_m-2,m-2 + (t2 P_mm(t2) - t1 P_mm(t1)) / (m + 1)
//   I_m+1,m = -a_m+1,m / (m + 2) (u2^2 P_mm(t2) - u1^2 P_mm(t1))
//   I_nm    = h_n b_nm I_n-2,m - a_nm / (n + 1) (u2^2 P_n-1,m(t2) - ...)
// and for m = 0 from the un-normalised polynomials,
//   I_n0 = ((P_n+1 - P_n-1)(t2) - (P_n+1 - P_n-1)(t1)) / sqrt(2n + 1).
// Here the two boundary recurrences run in the rescaled form of leg.cuh
// (R_n = P_n / c_n) and the integral in the same units, J_n = I_n / c_n:
//   J_n = h_n beta_n J_n-2 - (u2^2 R_n-1(t2) - u1^2 R_n-1(t1)) / (n + 1),
// so that the scaled coefficients ct_n C_nm of the point synthesis, the
// chunk multipliers and the analysis reduction (which applies ct_n) serve
// unchanged.  A boundary whose P_nm is still below the double range (E != 0
// in leg.cuh) adds nothing to the integral, as CHarm's X-numbers below the
// range convert to zero.  Per degree and pair of cell rows: 4 FP64
// operations for the two boundary recurrences, 4 for the integral and 2 for
// the sums.
//
// The longitude integrals (shs_grd_fft_lc.c:73-118, shs_grd_lr.c:68-99,
// sha_cell.c:790-840) multiply the lumped coefficients of order m by
//   FFT grids:   sm = sin(m dlon) / m,  cm = (cos(m dlon) - 1) / m,
//   other grids and scattered cells: (2 / m) sin(m dlon / 2) about the
//   cell's central longitude,
// and the block mean divides by the cell area (sin latmax - sin latmin)
// dlon on the unit sphere.
//
// Work decomposition: grid synthesis and analysis take one warp per (order,
// tile of 32 cell-row pairs); scattered cells take one warp per tile of 32
// cells walking all orders, as the scattered-point synthesis does.  The
// per-degree tables (beta_n, ct C_nm, ct S_nm, h_n, 1 / (n + 1)) of each
// 64-degree chunk are staged in shared memory by the warp with coalesced
// loads; nothing waits on another warp.
#include <cstdint>

#include "common.cuh"
#include "kernels.h"
#include "leg.cuh"

namespace cb
{

namespace
{

constexpr int CELL_WARPS = 4;

// per warp: LEG_CHUNK x (tb, cs, hn) double2
constexpr size_t CELL_STAGE_BYTES = 3 * LEG_CHUNK * sizeof(double2);
// analysis: the staging of (tb, hn) (no coefficients) and the 32 x 32
// transpose of the partial sums, element (row, col) at row * 32 +
// (col ^ row) so that neither the row-wise stores nor the column-wise
// reads meet bank conflicts: 18 KB per warp, three blocks of four warps per
// SM
constexpr size_t CELL_SHA_WARP_BYTES =
    2 * LEG_CHUNK * sizeof(double2) + 32 * 32 * sizeof(double2);

struct Stage
{
    double2 *tb, *cs, *hn;
};

__device__ __forceinline__ Stage warp_stage(unsigned char *base)
{
    double2 *p = reinterpret_cast<double2 *>(base);
    return Stage{p, p + LEG_CHUNK, p + 2 * LEG_CHUNK};
}

// the analysis stage: no coefficient column
__device__ __forceinline__ Stage warp_stage_sha(unsigned char *base)
{
    double2 *p = reinterpret_cast<double2 *>(base);
    return Stage{p, nullptr, p + LEG_CHUNK};
}

// Stages chunk j of order m: entries n = m + 64 j + i, i < cnt, of the
// order's column (tb, cs) and (h_n beta_n, 1 / (n + 1)) in hn.  The warp
// reads the stage only after the __syncwarp that ends this function.
__device__ __forceinline__ void stage_chunk(const Stage &S, const CellArgs &A,
                                            long long c0, long long m, int j,
                                            int cnt, unsigned lane)
{
    __syncwarp();
    const long long off = (long long)j * LEG_CHUNK;
#pragma unroll
    for (int h = 0; h < 2; h++)
    {
        const int i = (int)lane + 32 * h;
        if (i < cnt)
        {
            const double2 b = A.tb[c0 + off + i];
            const double2 h = A.hn[m + off + i];
            S.tb[i] = b;
            if (S.cs)
                S.cs[i] = A.cs[c0 + off + i];
            // h_n beta_n formed once here instead of by every lane per
            // degree
            S.hn[i] = make_double2(h.x * b.x, h.y);
        }
        else
        {
            S.tb[i] = make_double2(0.0, 0.0);
            if (S.cs)
                S.cs[i] = make_double2(0.0, 0.0);
            S.hn[i] = make_double2(0.0, 0.0);
        }
    }
    __syncwarp();
}

// The two boundary recurrences and the integral of one cell row: state
// (x, y, E) per boundary as in leg.cuh, (J0, J1) = (J~_n-2, J~_n-1), and
// the weights w = u^2 of the boundaries that are in the double range.
struct CellRec
{
    double t1, t2, u1s, u2s;
    double x1, y1, x2, y2;
    int E1, E2;
    double w1, w2;
    double J0, J1;

    // degree n >= m + 1 with beta = beta_n, hb = h_n beta_n, inv = 1/(n+1);
    // returns J~_n
    __device__ __forceinline__ double step(double beta, double hb, double inv)
    {
        const double d = fma(w2, x2, -(w1 * x1));
        const double J = fma(hb, J0, -(d * inv));
        J0 = J1;
        J1 = J;
        const double z1 = fma(t1, x1, -(beta * y1));
        y1 = x1;
        x1 = z1;
        const double z2 = fma(t2, x2, -(beta * y2));
        y2 = x2;
        x2 = z2;
        return J;
    }

    __device__ __forceinline__ void scale(double mul)
    {
        x1 *= mul;
        y1 *= mul;
        x2 *= mul;
        y2 *= mul;
        J0 *= mul;
        J1 *= mul;
    }

    // renormalises the boundaries still below the range; true while one is
    __device__ __forceinline__ bool fixup()
    {
        if (E1 != 0 && leg_fixup(x1, y1, E1))
            w1 = u1s;
        if (E2 != 0 && leg_fixup(x2, y2, E2))
            w2 = u2s;
        return (E1 | E2) != 0;
    }
};

// One degree of two adjacent cell rows r0 (above) and r1 (below) whose
// common boundary, r0's lower and r1's upper, is carried once, by r0
// (r1's boundary-2 state is not advanced): three boundary recurrences
// instead of four and one product w x of the common boundary for both
// integrals.  r0's value rounds as CellRec::step; r1's difference of
// boundary terms is formed from the rounded common product.
__device__ __forceinline__ void step_shared(CellRec &r0, CellRec &r1,
                                            double beta, double hb,
                                            double inv, double &v0,
                                            double &v1)
{
    const double q = r0.w1 * r0.x1;
    const double d0 = fma(r0.w2, r0.x2, -q);
    const double d1 = fma(-r1.w1, r1.x1, q);
    const double J0 = fma(hb, r0.J0, -(d0 * inv));
    const double J1 = fma(hb, r1.J0, -(d1 * inv));
    r0.J0 = r0.J1;
    r0.J1 = J0;
    r1.J0 = r1.J1;
    r1.J1 = J1;
    const double za = fma(r0.t1, r0.x1, -(beta * r0.y1));
    r0.y1 = r0.x1;
    r0.x1 = za;
    const double zb = fma(r0.t2, r0.x2, -(beta * r0.y2));
    r0.y2 = r0.x2;
    r0.x2 = zb;
    const double zc = fma(r1.t1, r1.x1, -(beta * r1.y1));
    r1.y1 = r1.x1;
    r1.x1 = zc;
    v0 = J0;
    v1 = J1;
}

// Seeds of order m >= 1 at one cell row: R~_mm at both boundaries and
// J~_mm = I_mm 2^g0 (I_mm in real units from imm).
__device__ __forceinline__ void cell_seed(CellRec &R, double sigma, int g0,
                                          double u1, double u2, long long m,
                                          double imm)
{
    leg_seed(sigma, u1, 1.0, false, m, 0, R.x1, R.E1);
    leg_seed(sigma, u2, 1.0, false, m, 0, R.x2, R.E2);
    R.y1 = R.y2 = 0.0;
    R.w1 = R.E1 == 0 ? R.u1s : 0.0;
    R.w2 = R.E2 == 0 ? R.u2s : 0.0;
    R.J0 = 0.0;
    R.J1 = scalbn(imm, g0);
}

// x^k for a non-negative integer k by binary powering (one rounding per
// multiplication; the radius ratios of the cells)
__device__ __forceinline__ double ipow(double x, long long k)
{
    double r = 1.0;
    while (k)
    {
        if (k & 1)
            r *= x;
        x *= x;
        k >>= 1;
    }
    return r;
}

// Longitude factors of order m for cells of width dlon
__device__ __forceinline__ void lon_factors(long long m, double dlon,
                                            double *sm, double *cm,
                                            double *fm)
{
    if (m == 0)
    {
        *sm = dlon;
        *cm = 0.0;
        *fm = dlon;
        return;
    }
    const double mr = (double)m;
    double s, c;
    sincos(mr * dlon, &s, &c);
    *sm = s / mr;
    *cm = (c - 1.0) / mr;
    const double m2 = 2.0 / mr;
    *fm = m2 * sin(dlon / m2);
}

} // namespace

// ---------------------------------------------------------------------------
// I_mm of every cell-row pair (sectorial integrals, sha_cell.c:586-660)
// ---------------------------------------------------------------------------
// Two steps.  k_cell_imm_q: one thread per (order, pair) evaluates
// q_m = (t2 P_mm(t2) - t1 P_mm(t1)) / (m + 1) from the sectorial seeds of
// leg.cuh (P_mm = S_m u^m, S_m = sqrt(3) prod d_k, src/leg/
// leg_func_prepare.c; below the double range it is zero, as CHarm's
// X-numbers convert).  k_cell_imm_rec: one thread per pair runs the
// recurrence over the orders, I_mm = g_m I_m-2,m-2 + q_m, from the closed
// forms of I_11 and I_22, in place.  imm is order-major ([m][pair]), so
// that the writes and the reads by the warps of one order are coalesced.
__global__ void k_cell_imm_q(CellArgs A)
{
    const int np = A.npairs;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= A.nmax * (long long)np)
        return;
    const long long m = 1 + idx / np;
    const int p = (int)(idx % np);
    const double t1 = A.geo[0 * np + p], u1 = A.geo[1 * np + p];
    const double t2 = A.geo[2 * np + p], u2 = A.geo[3 * np + p];
    const double sigma = A.sg[2 * m];
    const int g0 = (int)A.sg[2 * m + 1];
    double x1, x2;
    int e1, e2;
    leg_seed(sigma, u1, 1.0, false, m, 0, x1, e1);
    leg_seed(sigma, u2, 1.0, false, m, 0, x2, e2);
    const double p1 = scalbn(x1, e1 - g0), p2 = scalbn(x2, e2 - g0);
    A.imm[(size_t)m * np + p] = A.hn[m].y * (t2 * p2 - t1 * p1);
}

__global__ void k_cell_imm_rec(CellArgs A)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int np = A.npairs;
    if (p >= np)
        return;
    const long long N = A.nmax;
    const double ROOT3 = 1.73205080756887729353;
    const double PI_2 = 1.57079632679489661923;
    const double t1 = A.geo[0 * np + p], u1 = A.geo[1 * np + p];
    const double t2 = A.geo[2 * np + p], u2 = A.geo[3 * np + p];
    const double la1 = A.geo[6 * np + p], la2 = A.geo[7 * np + p];
    double *io = A.imm + p;
    io[0] = 0.0;
    // the closed forms of CHarm (shs_cell_kernel.c:229-262)
    double im2 = (ROOT3 / 2.0) * ((t2 * u2 - (PI_2 - la2)) -
                                  (t1 * u1 - (PI_2 - la1)));
    io[(size_t)np] = im2;
    if (N < 2)
        return;
    double im1 = (3.87298334620741688518 / 6.0) *
                 (t2 * (3.0 - t2 * t2) - t1 * (3.0 - t1 * t1));
    io[2 * (size_t)np] = im1;
    constexpr int B = 8;
    for (long long m0 = 3; m0 <= N; m0 += B)
    {
        double q[B], gv[B];
#pragma unroll
        for (int b = 0; b < B; b++)
        {
            const long long m = m0 + b;
            q[b] = m <= N ? io[(size_t)m * np] : 0.0;
            gv[b] = m <= N ? __ldg(&A.gm[m]) : 0.0;
        }
#pragma unroll
        for (int b = 0; b < B; b++)
        {
            const long long m = m0 + b;
            if (m > N)
                break;
            const double v = fma(gv[b], im2, q[b]);
            io[(size_t)m * np] = v;
            im2 = im1;
            im1 = v;
        }
    }
}

// ---------------------------------------------------------------------------
// Grid synthesis: lumped coefficients of every cell row and order
// ---------------------------------------------------------------------------
template <bool RR>
__global__ void __launch_bounds__(CELL_WARPS * 32) k_shs_cell(CellArgs A)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const unsigned lane = threadIdx.x & 31u;
    const unsigned warp = threadIdx.x >> 5;
    const Stage S = warp_stage(smem_raw + (size_t)warp * CELL_STAGE_BYTES);
    const long long N = A.nmax;
    const int np = A.npairs;

    for (;;)
    {
        unsigned long long item = 0;
        if (lane == 0)
            item = atomicAdd(A.counter, 1ull);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= (unsigned long long)A.nitems)
            break;
        const long long m = (long long)(item / (unsigned long long)A.ntiles);
        const int tile = (int)(item % (unsigned long long)A.ntiles);
        const int p = tile * 32 + (int)lane;
        const bool valid = p < np;
        CellRec R;
        R.t1 = valid ? A.geo[0 * np + p] : 0.0;
        const double u1 = valid ? A.geo[1 * np + p] : 1.0;
        R.t2 = valid ? A.geo[2 * np + p] : 0.0;
        const double u2 = valid ? A.geo[3 * np + p] : 1.0;
        const double rho = (RR && valid) ? A.geo[4 * np + p] : 1.0;
        R.u1s = u1 * u1;
        R.u2s = u2 * u2;
        // polar optimisation (src/misc/misc_polar_optimization_apply.c with
        // cos(latmin), shs_cell_grd.c:720-727): the order adds nothing
        const bool skip_lane =
            !valid || (A.polar_thr >= 0.0 &&
                       A.polar_thr < (double)m - (double)N * u1);
        const bool skip = __all_sync(0xffffffffu, skip_lane);
        double ae = 0.0, ao = 0.0, be = 0.0, bo = 0.0;
        const long long c0 = tri_col0(N, m);
        const long long ncol = N - m + 1;
        const int nchunks = (int)((ncol + LEG_CHUNK - 1) / LEG_CHUNK);
        double rn = RR ? ipow(rho, m + 1) : 1.0;   // (R/r)^(n+1)

        if (!skip && m == 0)
        {
            // zonal: un-normalised polynomials (shs_cell_kernel.c:97-175);
            // the sums take I_n0 / ct_n against ct_n C_n0
            double p0a = 1.0, p0b = 1.0, p1a = R.t1, p1b = R.t2;
            for (int j = 0; j < nchunks; j++)
            {
                const int cnt = (int)min((long long)LEG_CHUNK,
                                         ncol - (long long)j * LEG_CHUNK);
                stage_chunk(S, A, c0, m, j, cnt, lane);
                for (int i = 0; i < cnt; i++)
                {
                    const long long n = (long long)j * LEG_CHUNK + i;
                    double in0;
                    if (n == 0)
                        in0 = R.t2 - R.t1;
                    else
                    {
                        const double4 z = A.zn[n];
                        const double p2a = z.x * (R.t1 * p1a) - z.y * p0a;
                        const double p2b = z.x * (R.t2 * p1b) - z.y * p0b;
                        in0 = z.z * ((p2b - p0b) - (p2a - p0a));
                        p0a = p1a;
                        p1a = p2a;
                        p0b = p1b;
                        p1b = p2b;
                    }
                    const double v = (in0 / A.tc[c0 + n]) * rn;
                    if (RR)
                        rn *= rho;
                    const double2 c = S.cs[i];
                    if ((n & 1) == 0)
                        ae = fma(v, c.x, ae);
                    else
                        ao = fma(v, c.x, ao);
                }
            }
        }
        else if (!skip)
        {
            const double sigma = A.sg[2 * m];
            const int g0 = (int)A.sg[2 * m + 1];
            cell_seed(R, sigma, g0, u1, u2, m,
                      valid ? A.imm[(size_t)m * np + p] : 0.0);
            bool any_scaled = __any_sync(0xffffffffu, (R.E1 | R.E2) != 0);
            for (int j = 0; j < nchunks; j++)
            {
                const int cnt = (int)min((long long)LEG_CHUNK,
                                         ncol - (long long)j * LEG_CHUNK);
                stage_chunk(S, A, c0, m, j, cnt, lane);
                int i0 = 0;
                if (j == 0)
                {
                    // n = m: the sectorial integral
                    const double v = R.J1 * rn;
                    if (RR)
                        rn *= rho;
                    const double2 c = S.cs[0];
                    ae = fma(v, c.x, ae);
                    be = fma(v, c.y, be);
                    i0 = 1;
                }
                else
                    R.scale(A.tmul[(size_t)m * A.ldmul + j]);
                auto one = [&](int i, bool odd) {
                    const double beta = S.tb[i].x;
                    const double2 h = S.hn[i];
                    const double J = R.step(beta, h.x, h.y);
                    const double v = RR ? J * rn : J;
                    if (RR)
                        rn *= rho;
                    const double2 c = S.cs[i];
                    if (odd)
                    {
                        ao = fma(v, c.x, ao);
                        bo = fma(v, c.y, bo);
                    }
                    else
                    {
                        ae = fma(v, c.x, ae);
                        be = fma(v, c.y, be);
                    }
                };
                int i = i0;
                if (i & 1)
                {
                    one(i, true);
                    i++;
                }
#pragma unroll 4
                for (; i + 1 < cnt; i += 2)
                {
                    one(i, false);
                    one(i + 1, true);
                }
                if (i < cnt)
                    one(i, false);
                if (any_scaled)
                    any_scaled = __any_sync(0xffffffffu, R.fixup());
            }
        }
        if (skip_lane)
            ae = ao = be = bo = 0.0;
        if (valid)
        {
            double sm, cm, fm;
            lon_factors(m, A.dlon, &sm, &cm, &fm);
            const double sc = A.geo[5 * np + p];
            auto put = [&](int row, double a, double b) {
                double2 v;
                if (A.fft)
                {
                    const double c = m == 0 ? 1.0 : 0.5;
                    v.x = ((a * sm - b * cm) * c) * sc;
                    v.y = -((a * cm + b * sm) * c) * sc;
                }
                else
                {
                    v.x = (a * fm) * sc;
                    v.y = (b * fm) * sc;
                }
                A.out[(size_t)row * A.ldf + m] = v;
            };
            put(A.row_n[p], ae + ao, be + bo);
            if (A.row_s[p] >= 0)
                put(A.row_s[p], ae - ao, be - bo);
        }
    }
}

// ---------------------------------------------------------------------------
// Grid synthesis, two adjacent cell-row pairs per lane
// ---------------------------------------------------------------------------
// Rows aligned as the analysis requires them (latmin[i] == latmax[i + 1]):
// lane l of tile t takes the pairs 2l and 2l + 1 of the tile's 64, whose
// common boundary (the lower one of the first, the upper one of the second)
// is carried once (step_shared): per two pairs and degree, three boundary
// recurrences instead of four and one product w x for both integrals.  The
// rest is k_shs_cell's, row by row.
template <bool RR>
__global__ void __launch_bounds__(CELL_WARPS * 32) k_shs_cell2(CellArgs A)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const unsigned lane = threadIdx.x & 31u;
    const unsigned warp = threadIdx.x >> 5;
    const Stage S = warp_stage(smem_raw + (size_t)warp * CELL_STAGE_BYTES);
    const long long N = A.nmax;
    const int np = A.npairs;

    for (;;)
    {
        unsigned long long item = 0;
        if (lane == 0)
            item = atomicAdd(A.counter, 1ull);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= (unsigned long long)A.nitems)
            break;
        const long long m = (long long)(item / (unsigned long long)A.ntiles);
        const int tile = (int)(item % (unsigned long long)A.ntiles);
        CellRec R[2];
        int pk[2];
        bool valid[2], skip_k[2];
        double rho[2], rn[2], u1k[2], u2k[2];
        double ae[2] = {0.0, 0.0}, ao[2] = {0.0, 0.0};
        double be[2] = {0.0, 0.0}, bo[2] = {0.0, 0.0};
        bool skip_all = true;
#pragma unroll
        for (int k = 0; k < 2; k++)
        {
            const int p = tile * 64 + 2 * (int)lane + k;
            pk[k] = p;
            valid[k] = p < np;
            R[k].t1 = valid[k] ? A.geo[0 * np + p] : 0.0;
            u1k[k] = valid[k] ? A.geo[1 * np + p] : 1.0;
            R[k].t2 = valid[k] ? A.geo[2 * np + p] : 0.0;
            u2k[k] = valid[k] ? A.geo[3 * np + p] : 1.0;
            rho[k] = (RR && valid[k]) ? A.geo[4 * np + p] : 1.0;
            R[k].u1s = u1k[k] * u1k[k];
            R[k].u2s = u2k[k] * u2k[k];
            skip_k[k] = !valid[k] ||
                        (A.polar_thr >= 0.0 &&
                         A.polar_thr < (double)m - (double)N * u1k[k]);
            skip_all &= skip_k[k];
            rn[k] = RR ? ipow(rho[k], m + 1) : 1.0;
        }
        const bool skip = __all_sync(0xffffffffu, skip_all);
        const long long c0 = tri_col0(N, m);
        const long long ncol = N - m + 1;
        const int nchunks = (int)((ncol + LEG_CHUNK - 1) / LEG_CHUNK);

        if (!skip && m == 0)
        {
            // zonal: un-normalised polynomials (shs_cell_kernel.c:97-175),
            // row by row
            double p0a[2] = {1.0, 1.0}, p0b[2] = {1.0, 1.0};
            double p1a[2] = {R[0].t1, R[1].t1}, p1b[2] = {R[0].t2, R[1].t2};
            for (int j = 0; j < nchunks; j++)
            {
                const int cnt = (int)min((long long)LEG_CHUNK,
                                         ncol - (long long)j * LEG_CHUNK);
                stage_chunk(S, A, c0, m, j, cnt, lane);
                for (int i = 0; i < cnt; i++)
                {
                    const long long n = (long long)j * LEG_CHUNK + i;
                    const double tcn = A.tc[c0 + n];
                    const double2 c = S.cs[i];
#pragma unroll
                    for (int k = 0; k < 2; k++)
                    {
                        double in0;
                        if (n == 0)
                            in0 = R[k].t2 - R[k].t1;
                        else
                        {
                            const double4 z = A.zn[n];
                            const double p2a =
                                z.x * (R[k].t1 * p1a[k]) - z.y * p0a[k];
                            const double p2b =
                                z.x * (R[k].t2 * p1b[k]) - z.y * p0b[k];
                            in0 = z.z * ((p2b - p0b[k]) - (p2a - p0a[k]));
                            p0a[k] = p1a[k];
                            p1a[k] = p2a;
                            p0b[k] = p1b[k];
                            p1b[k] = p2b;
                        }
                        const double v = (in0 / tcn) * rn[k];
                        if (RR)
                            rn[k] *= rho[k];
                        if ((n & 1) == 0)
                            ae[k] = fma(v, c.x, ae[k]);
                        else
                            ao[k] = fma(v, c.x, ao[k]);
                    }
                }
            }
        }
        else if (!skip)
        {
            const double sigma = A.sg[2 * m];
            const int g0 = (int)A.sg[2 * m + 1];
            bool sc = false;
#pragma unroll
            for (int k = 0; k < 2; k++)
            {
                cell_seed(R[k], sigma, g0, u1k[k], u2k[k], m,
                          valid[k] ? A.imm[(size_t)m * np + pk[k]] : 0.0);
                sc |= (R[k].E1 | R[k].E2) != 0;
            }
            // the common boundary is renormalised through R[0]
            R[1].E2 = 0;
            bool any_scaled = __any_sync(0xffffffffu, sc);
            for (int j = 0; j < nchunks; j++)
            {
                const int cnt = (int)min((long long)LEG_CHUNK,
                                         ncol - (long long)j * LEG_CHUNK);
                stage_chunk(S, A, c0, m, j, cnt, lane);
                int i0 = 0;
                if (j == 0)
                {
                    // n = m: the sectorial integrals
                    const double2 c = S.cs[0];
#pragma unroll
                    for (int k = 0; k < 2; k++)
                    {
                        const double v = R[k].J1 * rn[k];
                        if (RR)
                            rn[k] *= rho[k];
                        ae[k] = fma(v, c.x, ae[k]);
                        be[k] = fma(v, c.y, be[k]);
                    }
                    i0 = 1;
                }
                else
                {
                    const double mul = A.tmul[(size_t)m * A.ldmul + j];
                    R[0].scale(mul);
                    R[1].scale(mul);
                }
                auto one = [&](int i, bool odd) {
                    const double beta = S.tb[i].x;
                    const double2 h = S.hn[i];
                    double v[2];
                    step_shared(R[0], R[1], beta, h.x, h.y, v[0], v[1]);
                    const double2 c = S.cs[i];
#pragma unroll
                    for (int k = 0; k < 2; k++)
                    {
                        const double w = RR ? v[k] * rn[k] : v[k];
                        if (RR)
                            rn[k] *= rho[k];
                        if (odd)
                        {
                            ao[k] = fma(w, c.x, ao[k]);
                            bo[k] = fma(w, c.y, bo[k]);
                        }
                        else
                        {
                            ae[k] = fma(w, c.x, ae[k]);
                            be[k] = fma(w, c.y, be[k]);
                        }
                    }
                };
                int i = i0;
                if (i & 1)
                {
                    one(i, true);
                    i++;
                }
#pragma unroll 2
                for (; i + 1 < cnt; i += 2)
                {
                    one(i, false);
                    one(i + 1, true);
                }
                if (i < cnt)
                    one(i, false);
                if (any_scaled)
                {
                    const bool s0 = R[0].fixup();
                    const bool s1 = R[1].fixup();
                    any_scaled = __any_sync(0xffffffffu, s0 || s1);
                }
            }
        }
        double sm, cm, fm;
        lon_factors(m, A.dlon, &sm, &cm, &fm);
#pragma unroll
        for (int k = 0; k < 2; k++)
        {
            if (skip_k[k])
                ae[k] = ao[k] = be[k] = bo[k] = 0.0;
            if (!valid[k])
                continue;
            const int p = pk[k];
            const double sc = A.geo[5 * np + p];
            auto put = [&](int row, double a, double b) {
                double2 v;
                if (A.fft)
                {
                    const double c = m == 0 ? 1.0 : 0.5;
                    v.x = ((a * sm - b * cm) * c) * sc;
                    v.y = -((a * cm + b * sm) * c) * sc;
                }
                else
                {
                    v.x = (a * fm) * sc;
                    v.y = (b * fm) * sc;
                }
                A.out[(size_t)row * A.ldf + m] = v;
            };
            put(A.row_n[p], ae[k] + ao[k], be[k] + bo[k]);
            if (A.row_s[p] >= 0)
                put(A.row_s[p], ae[k] - ao[k], be[k] - bo[k]);
        }
    }
}

// ---------------------------------------------------------------------------
// Grid analysis (approximate quadrature): partial sums per group of tiles
// ---------------------------------------------------------------------------
// Work item = (order m, group g of tiles of 32 K pairs); each lane carries K
// pairs of cell rows and forms, per degree, the sum over them of
// J~_n {amp, bmp}^(n+m parity).  Every 32 degrees the warp transposes its
// lane values through shared memory so that lane l holds the warp total of
// degree n0 + l, added to the group's partial column (the warp owns it);
// k_sha_reduce sums the groups in fixed order and applies ct_n, the
// 1 / (4 pi) r / mu factor and the rescaling.
template <int K, bool SH>
__global__ void __launch_bounds__(CELL_WARPS * 32, K == 1 ? 3 : 2)
    k_sha_cell(CellArgs A)
{
    static_assert(!SH || K == 2, "shared boundaries pair two rows");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const unsigned lane = threadIdx.x & 31u;
    const unsigned warp = threadIdx.x >> 5;
    unsigned char *wbase = smem_raw + (size_t)warp * CELL_SHA_WARP_BYTES;
    const Stage S = warp_stage_sha(wbase);
    double2 *red = reinterpret_cast<double2 *>(
        wbase + 2 * LEG_CHUNK * sizeof(double2));
    const long long N = A.nmax;
    const int np = A.npairs;
    const long long T = tri_size(N);

    for (;;)
    {
        unsigned long long item = 0;
        if (lane == 0)
            item = atomicAdd(A.counter, 1ull);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= (unsigned long long)A.nitems)
            break;
        const long long m = (long long)(item / (unsigned long long)A.ngroups);
        const int g = (int)(item % (unsigned long long)A.ngroups);
        const long long c0 = tri_col0(N, m);
        const long long ncol = N - m + 1;
        const int nchunks = (int)((ncol + LEG_CHUNK - 1) / LEG_CHUNK);
        double2 *col = A.part + (size_t)g * (size_t)T + c0;
        const int tile0 = g * A.tiles_per_group;
        const int tile1 = min(tile0 + A.tiles_per_group, A.ntiles);
        double sm, cm, fm;
        lon_factors(m, A.dlon, &sm, &cm, &fm);
        bool stored = false;

        for (int tile = tile0; tile < tile1; tile++)
        {
            CellRec R[K];
            double amp[K], amm[K], bmp[K], bmm[K];
            double p0a[K], p0b[K], p1a[K], p1b[K];
            bool all_skip = true, any_scaled = false;
#pragma unroll
            for (int k = 0; k < K; k++)
            {
                // with shared boundaries a lane takes two adjacent pairs
                const int p = SH ? tile * 64 + 2 * (int)lane + k
                                 : tile * (32 * K) + k * 32 + (int)lane;
                const bool valid = p < np;
                R[k].t1 = valid ? A.geo[0 * np + p] : 0.0;
                const double u1 = valid ? A.geo[1 * np + p] : 1.0;
                R[k].t2 = valid ? A.geo[2 * np + p] : 0.0;
                const double u2 = valid ? A.geo[3 * np + p] : 1.0;
                R[k].u1s = u1 * u1;
                R[k].u2s = u2 * u2;
                const bool skip_lane =
                    !valid || (A.polar_thr >= 0.0 &&
                               A.polar_thr < (double)m - (double)N * u1);
                all_skip &= skip_lane;
                // amplitudes of the order (sha_cell.c:790-840): the r2c
                // sums a = Re F, b = -Im F of the row and of its mirror,
                // combined with the longitude integrals
                amp[k] = amm[k] = bmp[k] = bmm[k] = 0.0;
                if (!skip_lane)
                {
                    const double2 Fn = A.F[(size_t)A.row_n[p] * A.ldF + m];
                    double a = Fn.x, b = -Fn.y, a2 = 0.0, b2 = 0.0;
                    if (A.row_s[p] >= 0)
                    {
                        const double2 Fs =
                            A.F[(size_t)A.row_s[p] * A.ldF + m];
                        a2 = Fs.x;
                        b2 = -Fs.y;
                    }
                    const double ap = a + a2, am = a - a2;
                    const double bp = b + b2, bm = b - b2;
                    if (m == 0)
                    {
                        amp[k] = ap * A.dlon;
                        amm[k] = am * A.dlon;
                    }
                    else
                    {
                        amp[k] = ap * sm + bp * cm;
                        amm[k] = am * sm + bm * cm;
                        bmp[k] = bp * sm - ap * cm;
                        bmm[k] = bm * sm - am * cm;
                    }
                }
                p0a[k] = p0b[k] = 1.0;
                p1a[k] = R[k].t1;
                p1b[k] = R[k].t2;
                if (m > 0)
                {
                    cell_seed(R[k], A.sg[2 * m], (int)A.sg[2 * m + 1], u1, u2,
                              m, valid ? A.imm[(size_t)m * np + p] : 0.0);
                    any_scaled |= (R[k].E1 | R[k].E2) != 0;
                    // state before degree m: (x, y) = (0, R~_mm) and
                    // J0 = -J~_mm, so that the step of degree m with the
                    // staged beta = -1, h beta = -1, 1/(n+1) = 0 yields R~_mm and
                    // J~_mm: every degree takes the same step
                    R[k].y1 = R[k].x1;
                    R[k].x1 = 0.0;
                    R[k].y2 = R[k].x2;
                    R[k].x2 = 0.0;
                    R[k].J0 = -R[k].J1;
                    R[k].J1 = 0.0;
                    // the common boundary is renormalised through r0
                    if (SH && k == 1)
                        R[k].E2 = 0;
                }
            }
            if (__all_sync(0xffffffffu, all_skip))
                continue;
            any_scaled = __any_sync(0xffffffffu, any_scaled);
            // lane partial sums of degree jj of a 32-degree block: row jj,
            // column lane of the swizzled transpose
            auto put = [&](int jj, double vc, double vs) {
                red[jj * 32 + ((int)lane ^ jj)] = make_double2(vc, vs);
            };
            // lane l: the warp total of degree n0 + l added to the group's
            // running column (loaded before the block, so that its latency
            // hides behind the block)
            auto flush = [&](long long i_l, double2 prev) {
                __syncwarp();
                const double2 *row = red + lane * 32;
                double oc0 = 0.0, os0 = 0.0, oc1 = 0.0, os1 = 0.0;
#pragma unroll
                for (int q = 0; q < 32; q += 2)
                {
                    const double2 a = row[q ^ (int)lane];
                    const double2 b = row[(q + 1) ^ (int)lane];
                    oc0 += a.x;
                    os0 += a.y;
                    oc1 += b.x;
                    os1 += b.y;
                }
                __syncwarp();
                const double outc = oc0 + oc1, outs = os0 + os1;
                if (i_l < ncol)
                    col[i_l] = stored ? make_double2(prev.x + outc,
                                                     prev.y + outs)
                                      : make_double2(outc, outs);
            };
            if (m == 0)
            {
                // zonal: un-normalised polynomials (sha_cell.c:880-960);
                // the partial sums carry I_n0 / ct_n (k_sha_reduce applies
                // ct_n)
                for (int j = 0; j < nchunks; j++)
                {
                    const int cnt = (int)min((long long)LEG_CHUNK,
                                             ncol - (long long)j * LEG_CHUNK);
                    for (int half = 0; half < 2; half++)
                    {
                        const int ib = 32 * half;
                        if (ib >= cnt)
                            break;
                        const long long i_l =
                            (long long)j * LEG_CHUNK + ib + lane;
                        double2 prev = make_double2(0.0, 0.0);
                        if (stored && i_l < ncol)
                            prev = col[i_l];
                        for (int jj = 0; jj < 32; jj++)
                        {
                            const long long kk =
                                (long long)j * LEG_CHUNK + ib + jj;
                            double vc = 0.0;
                            if (kk < ncol)
                            {
                                const double rct = 1.0 / A.tc[kk];
                                const double4 z =
                                    kk > 0 ? A.zn[kk]
                                           : make_double4(0.0, 0.0, 0.0, 0.0);
#pragma unroll
                                for (int k = 0; k < K; k++)
                                {
                                    double in0;
                                    if (kk == 0)
                                        in0 = R[k].t2 - R[k].t1;
                                    else
                                    {
                                        const double p2a =
                                            z.x * (R[k].t1 * p1a[k]) -
                                            z.y * p0a[k];
                                        const double p2b =
                                            z.x * (R[k].t2 * p1b[k]) -
                                            z.y * p0b[k];
                                        in0 = z.z * ((p2b - p0b[k]) -
                                                     (p2a - p0a[k]));
                                        p0a[k] = p1a[k];
                                        p1a[k] = p2a;
                                        p0b[k] = p1b[k];
                                        p1b[k] = p2b;
                                    }
                                    vc = fma(in0 * rct,
                                             (kk & 1) ? amm[k] : amp[k], vc);
                                }
                            }
                            put(jj, vc, 0.0);
                        }
                        flush(i_l, prev);
                    }
                }
                stored = true;
                continue;
            }
            for (int j = 0; j < nchunks; j++)
            {
                const int cnt = (int)min((long long)LEG_CHUNK,
                                         ncol - (long long)j * LEG_CHUNK);
                stage_chunk(S, A, c0, m, j, cnt, lane);
                if (j == 0)
                {
                    // the seed step (see above)
                    if (lane == 0)
                    {
                        S.tb[0].x = -1.0;
                        S.hn[0] = make_double2(-1.0, 0.0);   // h beta, 0
                    }
                    __syncwarp();
                }
                else
                {
                    const double mul = A.tmul[(size_t)m * A.ldmul + j];
#pragma unroll
                    for (int k = 0; k < K; k++)
                        R[k].scale(mul);
                }
                for (int half = 0; half < 2; half++)
                {
                    const int ib = 32 * half;
                    if (ib >= cnt)
                        break;
                    const long long i_l = (long long)j * LEG_CHUNK + ib + lane;
                    double2 prev = make_double2(0.0, 0.0);
                    if (stored && i_l < ncol)
                        prev = col[i_l];
                    // degrees beyond nmax read beta = h = 1/(n+1) = 0 and
                    // contribute J = 0
#pragma unroll 4
                    for (int jj = 0; jj < 32; jj++)
                    {
                        const int i = ib + jj;
                        const double beta = S.tb[i].x;
                        const double2 h = S.hn[i];
                        const double hb = h.x;
                        const bool odd = (jj & 1) != 0;
                        double vc = 0.0, vs = 0.0;
                        if constexpr (SH)
                        {
                            double v0, v1;
                            step_shared(R[0], R[K - 1], beta, hb, h.y, v0, v1);
                            vc = fma(v0, odd ? amm[0] : amp[0], vc);
                            vs = fma(v0, odd ? bmm[0] : bmp[0], vs);
                            vc = fma(v1, odd ? amm[K - 1] : amp[K - 1], vc);
                            vs = fma(v1, odd ? bmm[K - 1] : bmp[K - 1], vs);
                        }
                        else
                        {
#pragma unroll
                            for (int k = 0; k < K; k++)
                            {
                                const double v = R[k].step(beta, hb, h.y);
                                vc = fma(v, odd ? amm[k] : amp[k], vc);
                                vs = fma(v, odd ? bmm[k] : bmp[k], vs);
                            }
                        }
                        put(jj, vc, vs);
                    }
                    flush(i_l, prev);
                }
                if (any_scaled)
                {
                    bool still = false;
#pragma unroll
                    for (int k = 0; k < K; k++)
                        still |= R[k].fixup();
                    any_scaled = __any_sync(0xffffffffu, still);
                }
            }
            stored = true;
        }
        if (!stored)
            for (long long i = lane; i < ncol; i += 32)
                col[i] = make_double2(0.0, 0.0);
    }
}

// ---------------------------------------------------------------------------
// Scattered cells (src/shs/shs_cell_sctr.c)
// ---------------------------------------------------------------------------
// One warp per tile of 32 cells walks every order: I_mm follows the
// recurrence over the orders in registers (sectorial values from leg_seed,
// converted to real units), the degree loop is the grid kernel's for one
// row, and each order adds (a m2sm2dl) cos(m lonc) + (b m2sm2dl) sin(m lonc)
// with lonc the cell's central longitude.
template <bool RR>
__global__ void __launch_bounds__(CELL_WARPS * 32) k_shs_cell_sctr(CellArgs A)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const unsigned lane = threadIdx.x & 31u;
    const unsigned warp = threadIdx.x >> 5;
    const Stage S = warp_stage(smem_raw + (size_t)warp * CELL_STAGE_BYTES);
    const long long N = A.nmax;
    const int np = A.npairs;
    const double ROOT3 = 1.73205080756887729353;
    const double PI_2 = 1.57079632679489661923;

    for (;;)
    {
        unsigned long long item = 0;
        if (lane == 0)
            item = atomicAdd(A.counter, 1ull);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= (unsigned long long)A.nitems)
            break;
        const int p = (int)item * 32 + (int)lane;
        const bool valid = p < np;
        CellRec R;
        R.t1 = valid ? A.geo[0 * np + p] : 0.0;
        const double u1 = valid ? A.geo[1 * np + p] : 1.0;
        R.t2 = valid ? A.geo[2 * np + p] : 0.0;
        const double u2 = valid ? A.geo[3 * np + p] : 1.0;
        const double rho = (RR && valid) ? A.geo[4 * np + p] : 1.0;
        const double la1 = valid ? A.geo[6 * np + p] : 0.0;
        const double la2 = valid ? A.geo[7 * np + p] : 0.0;
        const double lsum = valid ? A.lonsum[p] : 0.0;   // lonmin + lonmax
        const double dl = valid ? A.dlonc[p] : 1.0;      // lonmax - lonmin
        R.u1s = u1 * u1;
        R.u2s = u2 * u2;
        double fi = 0.0;
        double ratiom = rho;                 // (R/r)^(m+1)
        double im2 = 0.0, im1 = 0.0;         // I_m-2,m-2, I_m-1,m-1
        bool done = !valid;                  // polar-optimised from here on

        for (long long m = 0; m <= N; m++, ratiom *= rho)
        {
            if (!done && A.polar_thr >= 0.0 &&
                A.polar_thr < (double)m - (double)N * u1)
                done = true;
            // I_mm of this order (the sequence runs for every cell)
            double imm = 0.0;
            double sigma = 0.0;
            int g0 = 0;
            if (m > 0)
            {
                sigma = A.sg[2 * m];
                g0 = (int)A.sg[2 * m + 1];
                leg_seed(sigma, u1, 1.0, false, m, 0, R.x1, R.E1);
                leg_seed(sigma, u2, 1.0, false, m, 0, R.x2, R.E2);
                // P_mm in real units (below the range: 0, as X-numbers)
                const double p1 = scalbn(R.x1, R.E1 - g0);
                const double p2 = scalbn(R.x2, R.E2 - g0);
                if (m == 1)
                    imm = (ROOT3 / 2.0) * ((R.t2 * u2 - (PI_2 - la2)) -
                                           (R.t1 * u1 - (PI_2 - la1)));
                else if (m == 2)
                    imm = (3.87298334620741688518 / 6.0) *
                          (R.t2 * (3.0 - R.t2 * R.t2) -
                           R.t1 * (3.0 - R.t1 * R.t1));
                else
                    imm = A.gm[m] * im2 +
                          (1.0 / (double)(m + 1)) * (R.t2 * p2 - R.t1 * p1);
                im2 = im1;
                im1 = imm;
            }
            if (__all_sync(0xffffffffu, done))
                continue;
            const long long c0 = tri_col0(N, m);
            const long long ncol = N - m + 1;
            const int nchunks = (int)((ncol + LEG_CHUNK - 1) / LEG_CHUNK);
            double a = 0.0, b = 0.0;
            double rn = RR ? ratiom : 1.0;
            if (m == 0)
            {
                double p0a = 1.0, p0b = 1.0, p1a = R.t1, p1b = R.t2;
                for (int j = 0; j < nchunks; j++)
                {
                    const int cnt = (int)min((long long)LEG_CHUNK,
                                             ncol - (long long)j * LEG_CHUNK);
                    stage_chunk(S, A, c0, m, j, cnt, lane);
                    for (int i = 0; i < cnt; i++)
                    {
                        const long long n = (long long)j * LEG_CHUNK + i;
                        double in0;
                        if (n == 0)
                            in0 = R.t2 - R.t1;
                        else
                        {
                            const double4 z = A.zn[n];
                            const double p2a = z.x * (R.t1 * p1a) - z.y * p0a;
                            const double p2b = z.x * (R.t2 * p1b) - z.y * p0b;
                            in0 = z.z * ((p2b - p0b) - (p2a - p0a));
                            p0a = p1a;
                            p1a = p2a;
                            p0b = p1b;
                            p1b = p2b;
                        }
                        const double v = (in0 / A.tc[c0 + n]) * rn;
                        if (RR)
                            rn *= rho;
                        a = fma(v, S.cs[i].x, a);
                    }
                }
            }
            else
            {
                R.y1 = R.y2 = 0.0;
                R.w1 = R.E1 == 0 ? R.u1s : 0.0;
                R.w2 = R.E2 == 0 ? R.u2s : 0.0;
                R.J0 = 0.0;
                R.J1 = scalbn(imm, g0);
                bool any_scaled = __any_sync(0xffffffffu, (R.E1 | R.E2) != 0);
                for (int j = 0; j < nchunks; j++)
                {
                    const int cnt = (int)min((long long)LEG_CHUNK,
                                             ncol - (long long)j * LEG_CHUNK);
                    stage_chunk(S, A, c0, m, j, cnt, lane);
                    int i = 0;
                    if (j == 0)
                    {
                        const double v = R.J1 * rn;
                        if (RR)
                            rn *= rho;
                        a = fma(v, S.cs[0].x, a);
                        b = fma(v, S.cs[0].y, b);
                        i = 1;
                    }
                    else
                        R.scale(A.tmul[(size_t)m * A.ldmul + j]);
#pragma unroll 4
                    for (; i < cnt; i++)
                    {
                        const double beta = S.tb[i].x;
                        const double2 h = S.hn[i];
                        const double J = R.step(beta, h.x, h.y);
                        const double v = RR ? J * rn : J;
                        if (RR)
                            rn *= rho;
                        const double2 c = S.cs[i];
                        a = fma(v, c.x, a);
                        b = fma(v, c.y, b);
                    }
                    if (any_scaled)
                        any_scaled = __any_sync(0xffffffffu, R.fixup());
                }
            }
            if (!done)
            {
                double fm;
                if (m == 0)
                    fm = dl;
                else
                {
                    const double m2 = 2.0 / (double)m;
                    fm = m2 * sin(dl / m2);
                }
                double sl, cl;
                sincos(((double)m / 2.0) * lsum, &sl, &cl);
                fi += (a * fm) * cl + (b * fm) * sl;
            }
        }
        if (valid)
        {
            const double dsigma = (R.t2 - R.t1) * dl;
            A.fout[p] = (fi / dsigma) * A.mur;
        }
    }
}

// ---------------------------------------------------------------------------
// Direct forward DFT of rows of any length (odd rows of cell grids, which
// the row transforms of rfft.cu serve in the inverse direction only)
// ---------------------------------------------------------------------------
// X[row][k] = sum_j x[row][j] exp(-2 pi i j k / L), k = 0..kmax, the
// unnormalised r2c of FFTW's convention.  One thread per (row, k); the
// phase advances by a rotation through 2 pi k / L and restarts from the
// exact angle of (j k mod L) every 64 samples.
__global__ void k_dft_rows_fwd(long long nrows, long long L, int kmax,
                               const double *__restrict__ x, long long ldx,
                               double2 *X, int ldX)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long K = (long long)kmax + 1;
    if (idx >= nrows * K)
        return;
    const long long row = idx / K;
    const long long k = idx % K;
    const double *xr = x + row * ldx;
    double s1, c1;
    sincospi(2.0 * (double)k / (double)L, &s1, &c1);
    double re = 0.0, im = 0.0;
    for (long long j0 = 0; j0 < L; j0 += 64)
    {
        double ss, cc;
        sincospi(2.0 * (double)((j0 * k) % L) / (double)L, &ss, &cc);
        const long long j1 = min(j0 + 64, L);
        for (long long j = j0; j < j1; j++)
        {
            const double v = xr[j];
            re = fma(v, cc, re);
            im = fma(-v, ss, im);
            const double cn = fma(cc, c1, -(ss * s1));
            ss = fma(ss, c1, cc * s1);
            cc = cn;
        }
    }
    X[row * ldX + k] = make_double2(re, im);
}

// ---------------------------------------------------------------------------
// Launch helpers
// ---------------------------------------------------------------------------
cudaError_t launch_dft_rows_fwd(long long nrows, long long L, int kmax,
                                const double *x, long long ldx, double2 *X,
                                int ldX, cudaStream_t st)
{
    const long long total = nrows * ((long long)kmax + 1);
    if (total <= 0)
        return cudaSuccess;
    const int threads = 128;
    k_dft_rows_fwd<<<(unsigned)((total + threads - 1) / threads), threads, 0,
                     st>>>(nrows, L, kmax, x, ldx, X, ldX);
    return cudaGetLastError();
}

cudaError_t launch_cell_imm(const CellArgs &A, cudaStream_t st)
{
    if (A.npairs <= 0 || A.nmax < 1)
        return cudaSuccess;
    const long long total = A.nmax * (long long)A.npairs;
    k_cell_imm_q<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(A);
    const int threads = 32;
    k_cell_imm_rec<<<(A.npairs + threads - 1) / threads, threads, 0, st>>>(
        A);
    return cudaGetLastError();
}

cudaError_t launch_shs_cell(const CellArgs &A, bool rr, bool shared,
                            int grid, cudaStream_t st)
{
    const size_t smem = CELL_WARPS * CELL_STAGE_BYTES;
    if (shared && rr)
        k_shs_cell2<true><<<grid, CELL_WARPS * 32, smem, st>>>(A);
    else if (shared)
        k_shs_cell2<false><<<grid, CELL_WARPS * 32, smem, st>>>(A);
    else if (rr)
        k_shs_cell<true><<<grid, CELL_WARPS * 32, smem, st>>>(A);
    else
        k_shs_cell<false><<<grid, CELL_WARPS * 32, smem, st>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_sha_cell(const CellArgs &A, int K, bool shared, int grid,
                            cudaStream_t st)
{
    const size_t smem = CELL_WARPS * CELL_SHA_WARP_BYTES;
    static bool attr_set = false;
    if (!attr_set)
    {
        for (const void *f : {(const void *)k_sha_cell<1, false>,
                              (const void *)k_sha_cell<2, false>,
                              (const void *)k_sha_cell<2, true>})
        {
            cudaError_t e = cudaFuncSetAttribute(
                f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess)
                return e;
        }
        attr_set = true;
    }
    if (K == 2 && shared)
        k_sha_cell<2, true><<<grid, CELL_WARPS * 32, smem, st>>>(A);
    else if (K == 2)
        k_sha_cell<2, false><<<grid, CELL_WARPS * 32, smem, st>>>(A);
    else
        k_sha_cell<1, false><<<grid, CELL_WARPS * 32, smem, st>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_shs_cell_sctr(const CellArgs &A, bool rr, int grid,
                                 cudaStream_t st)
{
    const size_t smem = CELL_WARPS * CELL_STAGE_BYTES;
    if (rr)
        k_shs_cell_sctr<true><<<grid, CELL_WARPS * 32, smem, st>>>(A);
    else
        k_shs_cell_sctr<false><<<grid, CELL_WARPS * 32, smem, st>>>(A);
    return cudaGetLastError();
}

} // namespace cb
