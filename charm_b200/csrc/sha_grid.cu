// Analysis on quadrature grids: the per-order Legendre contraction of
// CHarm's sha_point (src/sha/sha_point.c:713-980), after the r2c transform of
// the grid rows.
//
// Work item = (order m, group g of latitude tiles); one warp per item.  For
// each tile of 32*K latitude pairs the warp runs the rescaled recurrence of
// leg.cuh over n and forms, per degree, the lane partial sum over its K
// pairs of R~_n(t) * {a, b}^(n+m parity).  Every 32 degrees the warp
// transpose-reduce leaves lane l with the warp total of degree n0 + l,
// which is added to the group's partial column (plain read-modify-write:
// the warp owns it).  k_sha_reduce (tables.cu) sums the groups in a fixed
// order and applies ct_n, so results are deterministic.
//
// The same kernel computes the adjoint of the scattered-point synthesis
// (src/shs/shs_point_sctr.c:86-728) with respect to the coefficients: the
// "pairs" are then single points (no mirror, so both parities share one
// amplitude g_i (cos m lon_i, sin m lon_i)), and points off the sphere r = R
// fold (R/r)^(n+1) into the recurrence as the synthesis does.

#include <cstdint>

#include "common.cuh"
#include "kernels.h"
#include "leg.cuh"
#include "synth.cuh"

namespace cb
{

namespace
{

// per warp: two beta stages, two mbarriers (16 B), 32 x 33 partial sums
constexpr size_t SHA_WARP_SMEM =
    2 * LEG_CHUNK * sizeof(double2) + 16 + 32 * 33 * sizeof(double2);

struct PairA
{
    double ae, ao, be, bo;
};

__device__ __forceinline__ PairA load_pair_A(const ShaGridArgs &A, int p,
                                             long long m)
{
    PairA r{0.0, 0.0, 0.0, 0.0};
    if (p >= A.npairs)
        return r;
    int rn = A.row_n[p], rs = A.row_s[p];
    double2 Fn = A.F[(size_t)rn * A.ldF + m];
    double a = A.cw_n[p] * Fn.x;
    double b = -A.cw_n[p] * Fn.y;
    double a2 = 0.0, b2 = 0.0;
    if (rs >= 0)
    {
        double2 Fs = A.F[(size_t)rs * A.ldF + m];
        a2 = A.cw_s[p] * Fs.x;
        b2 = -A.cw_s[p] * Fs.y;
    }
    // sha_point.c:740-747 (symm = 1 when a mirror row exists)
    r.ae = a + a2;
    r.ao = a - a2;
    r.be = b + b2;
    r.bo = b - b2;
    return r;
}

} // namespace

// resident blocks per SM at which each tile width stays free of spills
// (measured with -Xptxas -v: K=8 246, K=6 215, K=4 166, K=2 128 registers)
constexpr int sha_min_blocks(int K) { return K >= 6 ? 2 : (K >= 4 ? 3 : 4); }

// amplitude source of k_sha_grid
enum
{
    SHA_SRC_GRID = 0,     // latitude pairs of a grid, r2c rows
    SHA_SRC_POINTS = 1,   // scattered points on the sphere r = R
    SHA_SRC_POINTS_R = 2  // scattered points with their own radii
};

// amplitudes of point p for order m: g_p (cos m lon_p, sin m lon_p), times
// `scale`
__device__ __forceinline__ PairA load_point_A(const ShaGridArgs &A, int p,
                                              long long m, double scale)
{
    PairA r{0.0, 0.0, 0.0, 0.0};
    if (p >= A.npairs)
        return r;
    double sm, cm;
    sincos_mlon((double)m, A.lon[p], &sm, &cm);
    const double g = A.g[p] * scale;
    r.ae = r.ao = g * cm;
    r.be = r.bo = g * sm;
    return r;
}

template <int K, int SRC>
__global__ void __launch_bounds__(128, sha_min_blocks(K)) k_sha_grid(ShaGridArgs A)
{
    constexpr bool PTS = SRC != SHA_SRC_GRID;
    constexpr bool RR = SRC == SHA_SRC_POINTS_R;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const unsigned lane = threadIdx.x & 31u;
    const unsigned warp = threadIdx.x >> 5;
    const size_t stage_bytes = LEG_CHUNK * sizeof(double2);
    unsigned char *wbase = smem_raw + (size_t)warp * SHA_WARP_SMEM;
    uint64_t *bar = reinterpret_cast<uint64_t *>(wbase + 2 * stage_bytes);
    double2 *red = reinterpret_cast<double2 *>(wbase + 2 * stage_bytes + 16);
    // stage s starts at wbase + s * stage_bytes; the mbarrier phases of
    // the two stages are bits 0 and 1 of `phases` (scalars, so that nothing
    // is indexed at run time and spilled to local memory)
    auto stg = [&](int s) {
        return reinterpret_cast<double2 *>(wbase + (size_t)s * stage_bytes);
    };
    if (lane == 0)
    {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
    }
    __syncwarp();
    unsigned phases = 0u;
    const long long N = A.nmax;
    const int np = A.npairs;
    bool failed = false;

    for (;;)
    {
        unsigned long long item = 0;
        if (lane == 0)
            item = atomicAdd(A.counter, 1ull);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= (unsigned long long)A.nitems)
            break;
        const long long m =
            A.m0 + (long long)(item / (unsigned long long)A.ngroups);
        const int g =
            A.group0 + (int)(item % (unsigned long long)A.ngroups);
        const long long c0 = tri_col0(N, m);
        const long long ncol = N - m + 1;
        const int nchunks = (int)((ncol + LEG_CHUNK - 1) / LEG_CHUNK);
        double2 *col = A.part + (size_t)g * (size_t)tri_size(N) + c0;
        const int tile0 = g * A.tiles_per_group;
        int tile1 = tile0 + A.tiles_per_group;
        if (tile1 > A.ntiles)
            tile1 = A.ntiles;
        const double sigma = A.sg[2 * m];
        bool stored = false;

        for (int tile = tile0; tile < tile1 && !failed; tile++)
        {
            double t[K], x[K], y[K], rho2[K];
            int E[K];
            PairA pa[K];
            bool skip = A.polar_thr >= 0.0;
#pragma unroll
            for (int k = 0; k < K; k++)
            {
                int p = tile * (32 * K) + k * 32 + (int)lane;
                bool valid = p < np;
                double u = 1.0, rh = 1.0;
                if (PTS)
                {
                    double tt = 0.0;
                    if (valid)
                        sincos(A.lat[p], &tt, &u);
                    if (RR && valid)
                        rh = A.R / A.r[p];
                    // (R/r)^(n+1) folded into the recurrence: t rho and
                    // beta rho^2, seed times rho^(m+1)
                    t[k] = RR ? tt * rh : tt;
                }
                else
                {
                    t[k] = valid ? A.t[p] : 0.0;
                    u = valid ? A.u[p] : 1.0;
                }
                rho2[k] = rh * rh;
                if (valid)
                    leg_seed(sigma, u, rh, RR, m, 0, x[k], E[k]);
                else
                {
                    x[k] = 0.0;
                    E[k] = 0;
                }
                // state (R~_n-1, R~_n-2) = (0, seed): the first step, with
                // beta = -1 at n = m (set in the staged table below),
                // yields the seed itself, so every degree takes the same
                // recurrence step
                y[k] = x[k];
                x[k] = 0.0;
                if (valid && !((double)m - (double)N * u > A.polar_thr))
                    skip = false;
                // scaled latitudes contribute nothing until they switch
                // off the sphere the sums read rho^2 R~ (see below), so
                // the amplitudes carry 1 / rho^2
                pa[k] = (E[k] != 0) ? PairA{0.0, 0.0, 0.0, 0.0}
                        : (PTS ? load_point_A(A, p, m, RR ? 1.0 / rho2[k] : 1.0)
                               : load_pair_A(A, p, m));
            }
            if (__all_sync(0xffffffffu, skip))
                continue;
            bool any_scaled = false;
#pragma unroll
            for (int k = 0; k < K; k++)
                any_scaled |= (E[k] != 0);
            any_scaled = __any_sync(0xffffffffu, any_scaled);

            auto issue = [&](int j, int s) {
                if (lane == 0)
                {
                    long long cnt = ncol - (long long)j * LEG_CHUNK;
                    if (cnt > LEG_CHUNK)
                        cnt = LEG_CHUNK;
                    unsigned bytes = (unsigned)(cnt * sizeof(double2));
                    mbar_arrive_expect_tx(&bar[s], bytes);
                    bulk_g2s(stg(s), A.tb + c0 + (long long)j * LEG_CHUNK,
                             bytes, &bar[s]);
                }
            };
            issue(0, 0);
            if (nchunks > 1)
                issue(1, 1);

            for (int j = 0; j < nchunks; j++)
            {
                const int s = j & 1;
                if (!mbar_wait_bounded(&bar[s], (phases >> s) & 1u, A.status))
                {
                    failed = true;
                    break;
                }
                phases ^= 1u << s;
                if (j > 0)
                {
                    const double mul = A.tmul[(size_t)m * A.ldmul + j];
#pragma unroll
                    for (int k = 0; k < K; k++)
                    {
                        x[k] *= mul;
                        y[k] *= mul;
                    }
                }
                long long cntl = ncol - (long long)j * LEG_CHUNK;
                const int cnt = cntl > LEG_CHUNK ? LEG_CHUNK : (int)cntl;
                double2 *stb = stg(s);
                // degrees beyond nmax read beta = 0 and contribute 0
                if (cnt < LEG_CHUNK)
                {
                    if ((int)lane >= cnt)
                        stb[lane] = make_double2(0.0, 0.0);
                    if ((int)lane + 32 >= cnt)
                        stb[lane + 32] = make_double2(0.0, 0.0);
                    __syncwarp();
                }
                if (j == 0)
                {
                    if (lane == 0)
                        stb[0].x = -1.0;
                    __syncwarp();
                }
#pragma unroll 1
                for (int half = 0; half < 2; half++)
                {
                    const long long n0 = m + (long long)j * LEG_CHUNK + 32 * half;
                    if (n0 > N)
                        break;
                    const double2 *blk = stb + 32 * half;
                    // the group's running sum of degree n0 + lane, loaded
                    // now so that its latency hides behind the block
                    const long long n = n0 + lane;
                    double2 prev = make_double2(0.0, 0.0);
                    if (stored && n <= N)
                        prev = col[n - m];
                    // lane partial sums of the 32 degrees: row jj, column
                    // lane of a 32 x 33 array (one pad column keeps both
                    // the row-wise stores and the column-wise read-back
                    // free of bank conflicts, with constant offsets)
                    double2 *redl = red + lane;
                    // accumulation of degree jj - 1 follows the recurrence
                    // step of degree jj (its value is then in y), so that
                    // each step's sums overlap the next step's products
                    auto accumulate = [&](const double *v, int row) {
                        double vc = 0.0, vs = 0.0;
#pragma unroll
                        for (int k = 0; k < K; k++)
                        {
                            if ((row & 1) == 0)
                            {
                                vc = fma(v[k], pa[k].ae, vc);
                                vs = fma(v[k], pa[k].be, vs);
                            }
                            else
                            {
                                vc = fma(v[k], pa[k].ao, vc);
                                vs = fma(v[k], pa[k].bo, vs);
                            }
                        }
                        redl[row * 33] = make_double2(vc, vs);
                    };
#pragma unroll
                    for (int jj = 0; jj < 32; jj++)
                    {
                        const double beta = blk[jj].x;
#pragma unroll
                        for (int k = 0; k < K; k++)
                        {
                            // off the sphere y holds rho^2 R~_n-2, so that
                            // the seed injection (beta = -1) stays exact
                            double z = fma(t[k], x[k], -(beta * y[k]));
                            y[k] = RR ? rho2[k] * x[k] : x[k];
                            x[k] = z;
                        }
                        if (jj > 0)
                            accumulate(y, jj - 1);
                    }
                    if (RR)
                    {
                        double xr[K];
#pragma unroll
                        for (int k = 0; k < K; k++)
                            xr[k] = rho2[k] * x[k];
                        accumulate(xr, 31);
                    }
                    else
                        accumulate(x, 31);
                    __syncwarp();
                    // lane l: warp total of degree n0 + l, fixed order
                    const double2 *row = red + lane * 33;
                    double oc0 = 0.0, os0 = 0.0, oc1 = 0.0, os1 = 0.0;
#pragma unroll
                    for (int q = 0; q < 32; q += 2)
                    {
                        double2 a = row[q];
                        double2 b = row[q + 1];
                        oc0 += a.x;
                        os0 += a.y;
                        oc1 += b.x;
                        os1 += b.y;
                    }
                    __syncwarp();
                    const double outc = oc0 + oc1, outs = os0 + os1;
                    if (n <= N)
                        col[n - m] = stored ? make_double2(prev.x + outc,
                                                           prev.y + outs)
                                            : make_double2(outc, outs);
                }
                if (any_scaled)
                {
                    bool still = false;
#pragma unroll
                    for (int k = 0; k < K; k++)
                    {
                        if (leg_fixup(x[k], y[k], E[k]))
                        {
                            int p = tile * (32 * K) + k * 32 + (int)lane;
                            pa[k] = PTS ? load_point_A(A, p, m,
                                                       RR ? 1.0 / rho2[k] : 1.0)
                                        : load_pair_A(A, p, m);
                        }
                        still |= (E[k] != 0);
                    }
                    any_scaled = __any_sync(0xffffffffu, still);
                }
                __syncwarp();
                if (j + 2 < nchunks)
                {
                    fence_proxy_async_smem();
                    issue(j + 2, s);
                }
            }
            stored = true;
        }
        if (failed)
            break;
        if (!stored)
        {
            for (long long n = m + lane; n <= N; n += 32)
                col[n - m] = make_double2(0.0, 0.0);
        }
    }
}

template <int SRC>
static cudaError_t launch_src(const ShaGridArgs &A, int K, int grid,
                              cudaStream_t st)
{
    const int warps = 4;
    const size_t smem = (size_t)warps * SHA_WARP_SMEM;
    // the dynamic shared memory exceeds the 48 KB default; set once
    static bool attr_set = false;
    if (!attr_set)
    {
        const void *fns[] = {(const void *)k_sha_grid<8, SRC>,
                             (const void *)k_sha_grid<6, SRC>,
                             (const void *)k_sha_grid<4, SRC>,
                             (const void *)k_sha_grid<2, SRC>,
                             (const void *)k_sha_grid<1, SRC>};
        for (const void *f : fns)
        {
            cudaError_t e = cudaFuncSetAttribute(
                f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess)
                return e;
        }
        attr_set = true;
    }
    if (K == 8)
        k_sha_grid<8, SRC><<<grid, warps * 32, smem, st>>>(A);
    else if (K == 6)
        k_sha_grid<6, SRC><<<grid, warps * 32, smem, st>>>(A);
    else if (K == 4)
        k_sha_grid<4, SRC><<<grid, warps * 32, smem, st>>>(A);
    else if (K == 2)
        k_sha_grid<2, SRC><<<grid, warps * 32, smem, st>>>(A);
    else
        k_sha_grid<1, SRC><<<grid, warps * 32, smem, st>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_sha_grid(const ShaGridArgs &A, int K, int grid,
                            cudaStream_t st)
{
    return launch_src<SHA_SRC_GRID>(A, K, grid, st);
}

cudaError_t launch_sha_points(const ShaGridArgs &A, int src, int K, int grid,
                              cudaStream_t st)
{
    if (src == SHA_SRC_POINTS_R)
        return launch_src<SHA_SRC_POINTS_R>(A, K, grid, st);
    if (src == SHA_SRC_POINTS)
        return launch_src<SHA_SRC_POINTS>(A, K, grid, st);
    return launch_src<SHA_SRC_GRID>(A, K, grid, st);
}

} // namespace cb
