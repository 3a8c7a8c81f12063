// Synthesis of lumped coefficients on grids (CHarm's shs_point_kernel,
// src/shs/shs_point_kernel.c:745-2010, as driven by
// src/shs/shs_point_grd.c:598-1018).
//
// Work item = (order m, tile of 32*K latitude pairs); one warp per item,
// handed out by an atomic counter in order of decreasing cost (ascending
// m).  Each lane carries K latitude pairs.  The degree loop streams the
// recurrence table (beta_n, e_n/a_n) and the scaled coefficients
// (ct_n C_nm, ct_n S_nm) through a two-stage shared-memory ring filled by
// 1-D bulk copies (TMA) completed on mbarriers, and runs the rescaled
// recurrence of leg.cuh: per degree and latitude one DMUL and three DFMA
// for the potential.  The north/south symmetry
// P_nm(-t) = (-1)^(n+m) P_nm(t) is used by keeping even and odd (n+m)
// partial sums; the parity of every step is a compile-time constant.
#include <cstdint>
#include <type_traits>

#include "common.cuh"
#include "kernels.h"
#include "leg.cuh"
#include "synth.cuh"

namespace cb
{

template <int KIND, int DL, int DR, int K, bool RR>
__global__ void __launch_bounds__(128) k_shs_grid(ShsGridArgs A)
{
    using Q = Qty<KIND, DL, DR>;
    constexpr int NQ = Q::NQ;
    constexpr int ND = Q::NEEDD;
    constexpr bool NEEDN = (ND > 0) || (KIND == 0 && DR > 0) || (KIND > 0);
    constexpr int dorder_c = KIND == 0 ? -1 : KIND;

    extern __shared__ __align__(128) unsigned char smem_raw[];
    const unsigned lane = threadIdx.x & 31u;
    const unsigned warp = threadIdx.x >> 5;
    // per warp: 2 stages x (tb, cs) x LEG_CHUNK double2, then 2 mbarriers
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
    const int np = A.npairs;
    const int dorder = dorder_c >= 0 ? dorder_c : (DR + DL + A.dlon);

    for (;;)
    {
        unsigned long long item = 0;
        if (lane == 0)
            item = atomicAdd(A.counter, 1ull);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= (unsigned long long)A.nitems)
            break;
        // batched sets: find the set of this item (items of set j start at
        // sets[j].item0), its degree, coefficients and output
        long long Nset = N;
        const double2 *csp = A.cs;
        double2 *outp = A.out;
        double mur = A.mur, polar_thr = A.polar_thr;
        unsigned long long local = item;
        if (A.nsets > 0)
        {
            int lo = 0, hi = A.nsets - 1;
            while (lo < hi)
            {
                int mid = (lo + hi + 1) >> 1;
                if ((unsigned long long)A.sets[mid].item0 <= item)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            const BatchSet &bs = A.sets[lo];
            Nset = bs.nmax;
            csp = bs.cs;
            outp = bs.out;
            mur = bs.mur;
            polar_thr = bs.polar_thr;
            local = item - (unsigned long long)bs.item0;
        }
        const long long m =
            A.m0 + (long long)(local / (unsigned long long)A.ntiles);
        const int tile =
            A.tile0 + (int)(local % (unsigned long long)A.ntiles);
        const double sigma = A.sg[2 * m];

        // ---- geometry and seeds of this lane's latitude pairs ----------
        int pk[K];
        double tq[K], tu[K], urr[K], u2r[K], uk[K], rho1[K], rho2[K];
        double x[K], y[K];
        int E[K];
        bool polar_skip = polar_thr >= 0.0;
#pragma unroll
        for (int k = 0; k < K; k++)
        {
            int p = tile * (32 * K) + k * 32 + (int)lane;
            pk[k] = p;
            bool valid = p < np;
            double t = valid ? A.t[p] : 0.0;
            double u = valid ? A.u[p] : 1.0;
            double rh = (RR && valid) ? A.rho[p] : 1.0;
            uk[k] = u;
            tq[k] = RR ? t * rh : t;
            rho1[k] = rh;
            rho2[k] = rh * rh;
            double ur = 1.0 / u;
            tu[k] = t * ur;
            urr[k] = RR ? ur * rh : ur;
            u2r[k] = ur * ur;
            y[k] = 0.0;
            if (valid)
                leg_seed(sigma, u, rh, RR, m, dorder, x[k], E[k]);
            else
            {
                x[k] = 0.0;
                E[k] = 0;
            }
            if (valid && !((double)m - (double)Nset * u > polar_thr))
                polar_skip = false;
        }
        polar_skip = __all_sync(0xffffffffu, polar_skip);

        Acc<NQ, 2, K> acc;
        acc.zero();

        if (!polar_skip)
        {
            // table offsets of the degree-N triangle; a set of lower degree
            // (coefficients in the same layout) stops at its own nmax
            const long long c0 = tri_col0(N, m);
            const long long ncol = Nset - m + 1;
            const int nchunks = (int)((ncol + LEG_CHUNK - 1) / LEG_CHUNK);
            auto issue = [&](int j, int s) {
                if (lane == 0)
                {
                    long long off = c0 + (long long)j * LEG_CHUNK;
                    long long cnt = ncol - (long long)j * LEG_CHUNK;
                    if (cnt > LEG_CHUNK)
                        cnt = LEG_CHUNK;
                    unsigned bytes = (unsigned)(cnt * sizeof(double2));
                    mbar_arrive_expect_tx(&bar[s], 2 * bytes);
                    bulk_g2s(stg(s), A.tb + off, bytes, &bar[s]);
                    bulk_g2s(stg(s) + LEG_CHUNK, csp + off, bytes, &bar[s]);
                }
            };
            issue(0, 0);
            if (nchunks > 1)
                issue(1, 1);

            bool any_scaled = false;
#pragma unroll
            for (int k = 0; k < K; k++)
                any_scaled |= (E[k] != 0);
            any_scaled = __any_sync(0xffffffffu, any_scaled);
            const double md = (double)m;
            const double m2 = md * md;

            if (!mbar_wait_bounded(&bar[0], (phases >> 0) & 1u, A.status))
                break;
            phases ^= 1u << 0;

            // ---- n = m (sectorial, even) --------------------------------
            {
                const double2 c = stg(0)[LEG_CHUNK];
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
            }
            // ---- n = m + 1 (odd; beta = 0, R_m+1 = t R_m) ---------------
            if (ncol > 1)
            {
                const double et = stg(0)[1].y;
                const double2 c = stg(0)[LEG_CHUNK + 1];
                const double nd = md + 1.0, np1 = nd + 1.0;
#pragma unroll
                for (int k = 0; k < K; k++)
                {
                    double xo = x[k];
                    double z = tq[k] * xo;
                    y[k] = xo;
                    x[k] = z;
                    double dp = 0.0, ddp = 0.0;
                    if (ND >= 1)
                        dp = (m == 0) ? (uk[k] * rho1[k]) * xo
                                      : fma(et * urr[k], xo, -((nd * tu[k]) * z));
                    if (ND >= 2)
                        ddp = (m == 0) ? -z
                                       : fma(tu[k], dp,
                                             fma(m2, u2r[k], -(nd * np1)) * z);
#pragma unroll
                    for (int q = 0; q < NQ; q++)
                    {
                        double v = Q::val(q, z, dp, ddp, np1);
                        acc.v[q][0][1][k] = fma(v, c.x, acc.v[q][0][1][k]);
                        acc.v[q][1][1][k] = fma(v, c.y, acc.v[q][1][1][k]);
                    }
                }
            }

            // ---- n = m + 2 .. N -----------------------------------------
            bool ok = true;
            for (int j = 0; j < nchunks; j++)
            {
                const int s = j & 1;
                if (j > 0)
                {
                    if (!mbar_wait_bounded(&bar[s], (phases >> s) & 1u, A.status))
                    {
                        ok = false;
                        break;
                    }
                    phases ^= 1u << s;
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

                auto step = [&](auto parc, int i) {
                    constexpr int PAR = decltype(parc)::value;
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
                            const double v =
                                (KIND == 0 && DL == 0 && DR == 0)
                                    ? z
                                    : Q::val(q, z, dp, ddp, np1);
                            acc.v[q][0][PAR][k] =
                                fma(v, c.x, acc.v[q][0][PAR][k]);
                            acc.v[q][1][PAR][k] =
                                fma(v, c.y, acc.v[q][1][PAR][k]);
                        }
                    }
                };
                const std::integral_constant<int, 0> EVEN{};
                const std::integral_constant<int, 1> ODD{};
                int i = (j == 0) ? 2 : 0;
                if (cnt == LEG_CHUNK && j > 0)
                {
#pragma unroll 8
                    for (int pp = 0; pp < LEG_CHUNK / 2; pp++)
                    {
                        step(EVEN, 2 * pp);
                        step(ODD, 2 * pp + 1);
                    }
                }
                else
                {
#pragma unroll 2
                    for (; i + 1 < cnt; i += 2)
                    {
                        step(EVEN, i);
                        step(ODD, i + 1);
                    }
                    if (i < cnt)
                        step(EVEN, i);
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
                __syncwarp();
                if (j + 2 < nchunks)
                {
                    fence_proxy_async_smem();
                    issue(j + 2, s);
                }
            }
            if (!ok)
                break;
            // latitudes that never left the scaled range contribute nothing
#pragma unroll
            for (int k = 0; k < K; k++)
                if (E[k] != 0)
                    acc.zero_k(k);
        }

        // ---- lumped coefficients: parity combination, derivative
        //      post-processing (shs_point_kernel.c:1643-1946), packing ----
        const double md = (double)m;
        const double cpack = A.fft_pack ? (m == 0 ? 1.0 : 0.5) : 1.0;
        const double sgnb = A.fft_pack ? -1.0 : 1.0;
#pragma unroll
        for (int k = 0; k < K; k++)
        {
            int p = pk[k];
            if (p >= np)
                continue;
            double ur = 1.0 / uk[k];
            double u2 = ur * ur;
#pragma unroll
            for (int h = 0; h < 2; h++)
            {
                int row = h == 0 ? A.row_n[p] : A.row_s[p];
                if (row < 0 || row >= A.nlat)
                    continue;
                double tuh = h == 0 ? tu[k] : -tu[k];
                double a[NQ], b[NQ];
#pragma unroll
                for (int q = 0; q < NQ; q++)
                {
                    double sg = (double)Q::parity(q);
                    double ev_c = acc.v[q][0][0][k], od_c = acc.v[q][0][1][k];
                    double ev_s = acc.v[q][1][0][k], od_s = acc.v[q][1][1][k];
                    a[q] = h == 0 ? ev_c + od_c : sg * (ev_c - od_c);
                    b[q] = h == 0 ? ev_s + od_s : sg * (ev_s - od_s);
                }
                lumped_post<KIND, DR, NQ>(a, b, md, ur, u2, tuh, A.dlon);
#pragma unroll
                for (int q = 0; q < NQ; q++)
                {
                    size_t o = ((size_t)q * A.nlat + row) * (size_t)A.ldf + m;
                    outp[o] = make_double2(cpack * mur * a[q],
                                           sgnb * (cpack * mur * b[q]));
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Longitude sums where FFT does not apply (CHarm's PSLR path,
// src/shs/shs_grd_lr.c, shs_grd_lr2.c): f[q][i][j] = sum_m a cos(m lon_j) +
// b sin(m lon_j).
// ---------------------------------------------------------------------------
__global__ void k_lon_direct(int npar, int nlat, int nlon, long long nmax,
                             const double2 *__restrict__ lc, int ldf,
                             const double *__restrict__ lon, double *f)
{
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long total = (long long)npar * nlat * nlon;
    if (idx >= total)
        return;
    int j = (int)(idx % nlon);
    long long qi = idx / nlon;
    const double2 *row = lc + qi * ldf;
    double lj = lon[j];
    // cos(m lon), sin(m lon) by rotation through lon from one order to the
    // next -- the recurrence over the orders that CHarm's PSLR path runs
    // over the longitudes (src/shs/shs_grd_lr.c, shs_grd_lr2.c: 2 cos(m
    // dlon) d_j-1 - d_j-2) -- restarted from the exact angle
    // (sincos_mlon) every 64 orders, so that the rounding of the rotations
    // cannot accumulate over more than 64 steps
    double s1, c1;
    sincos(lj, &s1, &c1);
    double acc = 0.0;
    for (long long m0 = 0; m0 <= nmax; m0 += 64)
    {
        double ss, cc;
        sincos_mlon((double)m0, lj, &ss, &cc);
        const long long m1 = m0 + 63 < nmax ? m0 + 63 : nmax;
        for (long long m = m0; m <= m1; m++)
        {
            const double2 v = row[m];
            acc = fma(v.x, cc, fma(v.y, ss, acc));
            const double cn = fma(cc, c1, -(ss * s1));
            ss = fma(ss, c1, cc * s1);
            cc = cn;
        }
    }
    f[idx] = acc;
}

// ---------------------------------------------------------------------------
// Launch helpers
// ---------------------------------------------------------------------------
template <int KIND, int DL, int DR, int K, bool RR>
static cudaError_t launch_one(const ShsGridArgs &A, int grid,
                              cudaStream_t st)
{
    const int warps = 4;
    size_t smem = (size_t)warps *
                  (2 * 2 * LEG_CHUNK * sizeof(double2) + 2 * sizeof(uint64_t));
    k_shs_grid<KIND, DL, DR, K, RR><<<grid, warps * 32, smem, st>>>(A);
    return cudaGetLastError();
}

template <int KIND, int DL, int DR, bool RR>
static cudaError_t launch_k(const ShsGridArgs &A, int K, int grid,
                            cudaStream_t st)
{
    if (K == 4)
        return launch_one<KIND, DL, DR, 4, RR>(A, grid, st);
    if (K == 2)
        return launch_one<KIND, DL, DR, 2, RR>(A, grid, st);
    return launch_one<KIND, DL, DR, 1, RR>(A, grid, st);
}

template <bool RR>
static cudaError_t launch_rr(const ShsGridArgs &A, int kgrad, int dr,
                             int dlat, int K, int grid, cudaStream_t st)
{
    if (kgrad == 1)
        return launch_k<1, 1, 0, RR>(A, K, grid, st);
    if (kgrad == 2)
        return launch_k<2, 2, 0, RR>(A, K, grid, st);
    if (dlat == 0 && dr == 0)
        return launch_k<0, 0, 0, RR>(A, K, grid, st);
    if (dlat == 0 && dr == 1)
        return launch_k<0, 0, 1, RR>(A, K, grid, st);
    if (dlat == 0 && dr == 2)
        return launch_k<0, 0, 2, RR>(A, K, grid, st);
    if (dlat == 1 && dr == 0)
        return launch_k<0, 1, 0, RR>(A, K, grid, st);
    if (dlat == 1 && dr == 1)
        return launch_k<0, 1, 1, RR>(A, K, grid, st);
    if (dlat == 2 && dr == 0)
        return launch_k<0, 2, 0, RR>(A, K, grid, st);
    return cudaErrorInvalidValue;
}

cudaError_t launch_shs_grid(const ShsGridArgs &A, int kgrad, int dr,
                            int dlat, bool rr, int K, int grid,
                            cudaStream_t st)
{
    return rr ? launch_rr<true>(A, kgrad, dr, dlat, K, grid, st)
              : launch_rr<false>(A, kgrad, dr, dlat, K, grid, st);
}

cudaError_t launch_lon_direct(int npar, int nlat, int nlon, long long nmax,
                              const double2 *lc, int ldf, const double *lon,
                              double *f, cudaStream_t st)
{
    long long total = (long long)npar * nlat * nlon;
    int blocks = (int)((total + 255) / 256);
    k_lon_direct<<<blocks, 256, 0, st>>>(npar, nlat, nlon, nmax, lc, ldf, lon,
                                         f);
    return cudaGetLastError();
}

} // namespace cb
