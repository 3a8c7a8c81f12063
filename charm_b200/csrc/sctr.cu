// Synthesis at scattered points (CHarm src/shs/shs_point_sctr.c:86-728).
//
// Work item = tile of 32*K points; one warp per item.  The warp walks all
// orders m = 0..nmax: the sectorial seed follows CHarm's sequence
// (src/leg/leg_func_prepare.c) in registers, the degree loop streams the
// whole recurrence table and scaled coefficient triangle through a
// two-stage shared-memory ring filled by 1-D bulk copies and runs the
// rescaled recurrence of leg.cuh, and each order's lumped coefficients are
// folded into f += a_m cos(m lon) + b_m sin(m lon)
// (shs_point_sctr.c:599-641).  Every point is written exactly once.
#include <cstdint>

#include "common.cuh"
#include "kernels.h"
#include "leg.cuh"
#include "synth.cuh"

namespace cb
{

template <int KIND, int DL, int DR, int K, bool RR>
__global__ void __launch_bounds__(128) k_sctr(SctrArgs A)
{
    using Q = Qty<KIND, DL, DR>;
    constexpr int NQ = Q::NQ;
    constexpr int ND = Q::NEEDD;
    constexpr bool NEEDN = (ND > 0) || (KIND == 0 && DR > 0) || (KIND > 0);

    extern __shared__ __align__(128) unsigned char smem_raw[];
    const unsigned lane = threadIdx.x & 31u;
    const unsigned warp = threadIdx.x >> 5;
    const size_t stage_bytes = 2 * LEG_CHUNK * sizeof(double2);
    unsigned char *wbase =
        smem_raw + (size_t)warp * (2 * stage_bytes + 2 * sizeof(uint64_t));
    uint64_t *bar = reinterpret_cast<uint64_t *>(wbase + 2 * stage_bytes);
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
    const double BIG = 0x1p960, BIGI = 0x1p-960;
    const double BIGS = 0x1p480, BIGSI = 0x1p-480;
    const double ROOT3 = 1.73205080756887729353;
    const int dorder = KIND == 0 ? (DR + DL + A.dlon) : KIND;
    bool failed = false;

    for (;;)
    {
        unsigned long long item = 0;
        if (lane == 0)
            item = atomicAdd(A.counter, 1ull);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= (unsigned long long)A.ntiles)
            break;

        long long pk[K];
        double tq[K], tu[K], urr[K], u2r[K], uk[K], rho1[K], rho2[K], lon[K];
        double xs[K], rp[K];
        int ixs[K];
        double fa[NQ][K];
#pragma unroll
        for (int k = 0; k < K; k++)
        {
            long long p = (long long)item * (32 * K) + k * 32 + lane;
            pk[k] = p;
            bool valid = p < A.npoint;
            double la = valid ? A.lat[p] : 0.0;
            double t, u;
            sincos(la, &t, &u);
            double rh = (RR && valid) ? A.R / A.r[p] : 1.0;
            lon[k] = valid ? A.lon[p] : 0.0;
            uk[k] = u;
            tq[k] = RR ? t * rh : t;
            rho1[k] = rh;
            rho2[k] = rh * rh;
            double ur = 1.0 / u;
            tu[k] = t * ur;
            urr[k] = RR ? ur * rh : ur;
            u2r[k] = ur * ur;
            xs[k] = 1.0;
            ixs[k] = 0;
            // (R/r)^(1 + dorder) for m = 0 (src/shs/shs_rpows.c)
            double r0 = 1.0;
            for (int i = 0; i < 1 + dorder; i++)
                r0 *= rh;
            rp[k] = r0;
#pragma unroll
            for (int q = 0; q < NQ; q++)
                fa[q][k] = 0.0;
        }

        // chunk stream over the whole triangle, column by column
        long long im = 0;
        int ij = 0;                      // next chunk to issue
        auto ncol_of = [&](long long m) { return N - m + 1; };
        auto nch_of = [&](long long m) {
            return (int)((ncol_of(m) + LEG_CHUNK - 1) / LEG_CHUNK);
        };
        auto issue_next = [&](int s) {
            if (im > N)
                return;
            if (lane == 0)
            {
                long long off = tri_col0(N, im) + (long long)ij * LEG_CHUNK;
                long long cnt = ncol_of(im) - (long long)ij * LEG_CHUNK;
                if (cnt > LEG_CHUNK)
                    cnt = LEG_CHUNK;
                unsigned bytes = (unsigned)(cnt * sizeof(double2));
                mbar_arrive_expect_tx(&bar[s], 2 * bytes);
                bulk_g2s(stg(s), A.tb + off, bytes, &bar[s]);
                bulk_g2s(stg(s) + LEG_CHUNK, A.cs + off, bytes, &bar[s]);
            }
            if (++ij >= nch_of(im))
            {
                ij = 0;
                ++im;
            }
        };
        int consumed = 0;
        issue_next(0);
        issue_next(1);

        for (long long m = 0; m <= N && !failed; m++)
        {
            // sectorial seed of order m (leg_func_prepare.c:18-69) times the
            // chunk-0 power of two of the rescaled recurrence
            const int g0 = (int)A.sg[2 * m + 1];
            double x[K], y[K];
            int E[K];
            bool skip = A.polar_thr >= 0.0;
#pragma unroll
            for (int k = 0; k < K; k++)
            {
                if (m == 1)
                {
                    xs[k] = ROOT3 * uk[k];
                    ixs[k] = 0;
                }
                else if (m >= 2)
                {
                    double v = (A.dm[m - 1] * uk[k]) * xs[k];
                    double w = fabs(v);
                    if (w >= BIGS)
                    {
                        v *= BIGI;
                        ixs[k] += 1;
                    }
                    else if (w < BIGSI)
                    {
                        v *= BIG;
                        ixs[k] -= 1;
                    }
                    xs[k] = v;
                }
                if (m >= 1)
                    rp[k] *= rho1[k];
                x[k] = (m == 0) ? rp[k] : (RR ? xs[k] * rp[k] : xs[k]);
                E[k] = ((m == 0) ? 0 : 960 * ixs[k]) + g0;
                y[k] = 0.0;
                leg_seed_normalise(x[k], E[k]);
                if (pk[k] < A.npoint &&
                    !((double)m - (double)N * uk[k] > A.polar_thr))
                    skip = false;
            }
            skip = __all_sync(0xffffffffu, skip);
            bool any_scaled = false;
#pragma unroll
            for (int k = 0; k < K; k++)
                any_scaled |= (E[k] != 0);
            any_scaled = __any_sync(0xffffffffu, any_scaled);

            Acc<NQ, 1, K> acc;
            acc.zero();
            const double md = (double)m;
            const double m2 = md * md;
            const long long ncol = ncol_of(m);
            const int nch = nch_of(m);
            for (int j = 0; j < nch; j++)
            {
                const int s = consumed & 1;
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
                const double2 *stb = stg(s);
                const double2 *scs = stg(s) + LEG_CHUNK;
                const long long nbase = m + (long long)j * LEG_CHUNK;
                if (!skip)
                {
                    int i = 0;
                    if (j == 0)
                    {
                        // n = m
                        const double2 c = scs[0];
                        const double np1 = md + 1.0;
#pragma unroll
                        for (int k = 0; k < K; k++)
                        {
                            double p = x[k], dp = 0.0, ddp = 0.0;
                            if (ND >= 1)
                                dp = -((md * tu[k]) * p);
                            if (ND >= 2)
                                ddp = fma(tu[k], dp,
                                          fma(m2, u2r[k], -(md * (md + 1.0))) * p);
#pragma unroll
                            for (int q = 0; q < NQ; q++)
                            {
                                double v = Q::val(q, p, dp, ddp, np1);
                                acc.v[q][0][0][k] = fma(v, c.x, acc.v[q][0][0][k]);
                                acc.v[q][1][0][k] = fma(v, c.y, acc.v[q][1][0][k]);
                            }
                        }
                        // n = m + 1 (beta = 0)
                        if (cnt > 1)
                        {
                            const double et = stb[1].y;
                            const double2 c1 = scs[1];
                            const double nd = md + 1.0, np2 = nd + 1.0;
#pragma unroll
                            for (int k = 0; k < K; k++)
                            {
                                double xo = x[k];
                                double z = tq[k] * xo;
                                y[k] = xo;
                                x[k] = z;
                                double dp = 0.0, ddp = 0.0;
                                if (ND >= 1)
                                    dp = (m == 0)
                                             ? (uk[k] * rho1[k]) * xo
                                             : fma(et * urr[k], xo, -((nd * tu[k]) * z));
                                if (ND >= 2)
                                    ddp = (m == 0) ? -z
                                                   : fma(tu[k], dp,
                                                         fma(m2, u2r[k], -(nd * np2)) * z);
#pragma unroll
                                for (int q = 0; q < NQ; q++)
                                {
                                    double v = Q::val(q, z, dp, ddp, np2);
                                    acc.v[q][0][0][k] = fma(v, c1.x, acc.v[q][0][0][k]);
                                    acc.v[q][1][0][k] = fma(v, c1.y, acc.v[q][1][0][k]);
                                }
                            }
                        }
                        i = 2;
                    }
#pragma unroll 4
                    for (; i < cnt; i++)
                    {
                        const double2 tbv = stb[i];
                        const double2 c = scs[i];
                        const double nd = NEEDN ? (double)(nbase + i) : 0.0;
                        const double np1 = nd + 1.0;
#pragma unroll
                        for (int k = 0; k < K; k++)
                        {
                            const double xo = x[k];
                            const double by = RR ? tbv.x * (rho2[k] * y[k])
                                                 : tbv.x * y[k];
                            const double z = fma(tq[k], xo, -by);
                            y[k] = xo;
                            x[k] = z;
                            double dp = 0.0, ddp = 0.0;
                            if (ND >= 1)
                                dp = fma(tbv.y * urr[k], xo, -((nd * tu[k]) * z));
                            if (ND >= 2)
                                ddp = fma(tu[k], dp,
                                          fma(m2, u2r[k], -(nd * np1)) * z);
#pragma unroll
                            for (int q = 0; q < NQ; q++)
                            {
                                const double v = (KIND == 0 && DL == 0 && DR == 0)
                                                     ? z
                                                     : Q::val(q, z, dp, ddp, np1);
                                acc.v[q][0][0][k] = fma(v, c.x, acc.v[q][0][0][k]);
                                acc.v[q][1][0][k] = fma(v, c.y, acc.v[q][1][0][k]);
                            }
                        }
                    }
                    if (any_scaled)
                    {
                        bool still = false;
#pragma unroll
                        for (int k = 0; k < K; k++)
                        {
                            if (leg_fixup(x[k], y[k], E[k]))
                                acc.zero_k(k);
                            still |= (E[k] != 0);
                        }
                        any_scaled = __any_sync(0xffffffffu, still);
                    }
                }
                __syncwarp();
                ++consumed;
                fence_proxy_async_smem();
                issue_next(s);
            }
            if (failed || skip)
                continue;
#pragma unroll
            for (int k = 0; k < K; k++)
            {
                if (E[k] != 0)
                    acc.zero_k(k);
                double a[NQ], b[NQ];
#pragma unroll
                for (int q = 0; q < NQ; q++)
                {
                    a[q] = acc.v[q][0][0][k];
                    b[q] = acc.v[q][1][0][k];
                }
                double ur = 1.0 / uk[k];
                lumped_post<KIND, DR, NQ>(a, b, md, ur, ur * ur, tu[k], A.dlon);
                double sm, cm;
                sincos_mlon(md, lon[k], &sm, &cm);
#pragma unroll
                for (int q = 0; q < NQ; q++)
                    fa[q][k] = fma(a[q], cm, fma(b[q], sm, fa[q][k]));
            }
        }
        if (failed)
            break;
#pragma unroll
        for (int k = 0; k < K; k++)
        {
            if (pk[k] >= A.npoint)
                continue;
#pragma unroll
            for (int q = 0; q < NQ; q++)
                A.f[(size_t)q * A.npoint + pk[k]] = A.mur * fa[q][k];
        }
    }
}

template <int KIND, int DL, int DR, int K, bool RR>
static cudaError_t launch_s1(const SctrArgs &A, int grid, cudaStream_t st)
{
    const int warps = 4;
    size_t smem = (size_t)warps *
                  (2 * 2 * LEG_CHUNK * sizeof(double2) + 2 * sizeof(uint64_t));
    k_sctr<KIND, DL, DR, K, RR><<<grid, warps * 32, smem, st>>>(A);
    return cudaGetLastError();
}

template <int KIND, int DL, int DR, bool RR>
static cudaError_t launch_sk(const SctrArgs &A, int K, int grid,
                             cudaStream_t st)
{
    if (K == 4)
        return launch_s1<KIND, DL, DR, 4, RR>(A, grid, st);
    if (K == 2)
        return launch_s1<KIND, DL, DR, 2, RR>(A, grid, st);
    return launch_s1<KIND, DL, DR, 1, RR>(A, grid, st);
}

template <bool RR>
static cudaError_t launch_srr(const SctrArgs &A, int kgrad, int dr, int dlat,
                              int K, int grid, cudaStream_t st)
{
    if (kgrad == 1)
        return launch_sk<1, 1, 0, RR>(A, K, grid, st);
    if (kgrad == 2)
        return launch_sk<2, 2, 0, RR>(A, K, grid, st);
    if (dlat == 0 && dr == 0)
        return launch_sk<0, 0, 0, RR>(A, K, grid, st);
    if (dlat == 0 && dr == 1)
        return launch_sk<0, 0, 1, RR>(A, K, grid, st);
    if (dlat == 0 && dr == 2)
        return launch_sk<0, 0, 2, RR>(A, K, grid, st);
    if (dlat == 1 && dr == 0)
        return launch_sk<0, 1, 0, RR>(A, K, grid, st);
    if (dlat == 1 && dr == 1)
        return launch_sk<0, 1, 1, RR>(A, K, grid, st);
    if (dlat == 2 && dr == 0)
        return launch_sk<0, 2, 0, RR>(A, K, grid, st);
    return cudaErrorInvalidValue;
}

cudaError_t launch_sctr(const SctrArgs &A, int kgrad, int dr, int dlat,
                        bool rr, int K, int grid, cudaStream_t st)
{
    return rr ? launch_srr<true>(A, kgrad, dr, dlat, K, grid, st)
              : launch_srr<false>(A, kgrad, dr, dlat, K, grid, st);
}

} // namespace cb
