// Synthesis of lumped coefficients on grids (CHarm's shs_point_kernel for
// grids, src/shs/shs_point_kernel.c:745-2010, driven as in
// src/shs/shs_point_grd.c:598-1018), plus the tables it reads.
//
// Work item = (order m, tile of 32*K latitude pairs); one warp per item,
// items handed out by an atomic counter in order of decreasing cost
// (ascending m).  Each lane carries K latitude pairs.  The degree loop
// streams the recurrence coefficients (a_nm, b_nm), the coefficients
// (C_nm, S_nm) and, for derivatives, (e_nm, n) through a two-stage
// shared-memory ring filled by 1-D bulk copies (TMA) on mbarriers.  The
// north/south symmetry P_nm(-t) = (-1)^(n+m) P_nm(t) is used by keeping
// separate even and odd (n+m) partial sums.
#include <cstdint>

#include "common.cuh"
#include "kernels.h"
#include "leg.cuh"
#include "synth.cuh"

namespace cb
{

// ---------------------------------------------------------------------------
// Tables
// ---------------------------------------------------------------------------

// (a_nm, b_nm) for all 0 <= m <= n <= nmax, order-major; a_mm = b_mm = 0 and
// b_m+1,m = 0 (src/leg/leg_func_anm_bnm.c:14-65).  r, ri are sqrt(k),
// 1/sqrt(k) (leg_func_r_ri.c).
__global__ void k_table_ab(long long nmax, const double *__restrict__ r,
                           const double *__restrict__ ri, double2 *ab)
{
    long long m = blockIdx.x;
    if (m > nmax)
        return;
    long long c0 = tri_col0(nmax, m);
    for (long long n = m + threadIdx.x; n <= nmax; n += blockDim.x)
    {
        double a = 0.0, b = 0.0;
        if (n == m + 1)
            a = r[2 * m + 3];
        else if (n >= m + 2)
        {
            double w = r[2 * n + 1] * ri[n - m] * ri[n + m];
            a = r[2 * n - 1] * w;
            b = r[n - m - 1] * r[n + m - 1] * ri[2 * n - 3] * w;
        }
        ab[c0 + n - m] = make_double2(a, b);
    }
}

// (e_nm, n) for the latitude derivatives (src/leg/leg_func_enm.c:14-55).
__global__ void k_table_en(long long nmax, const double *__restrict__ r,
                           const double *__restrict__ ri, double2 *en)
{
    long long m = blockIdx.x;
    if (m > nmax)
        return;
    long long c0 = tri_col0(nmax, m);
    for (long long n = m + threadIdx.x; n <= nmax; n += blockDim.x)
    {
        double e = 0.0;
        if (n > m)
            e = r[2 * n + 1] * r[n - m] * r[n + m] * ri[2 * n - 1];
        en[c0 + n - m] = make_double2(e, (double)n);
    }
}

// Interleaves the caller's C, S triangles (degree shc_nmax) into (C, S)
// pairs of the degree-nmax triangle.  S_n0 is forced to zero: CHarm never
// reads it (shs_point_kernel.c:1014-1248 uses only C for m = 0).
__global__ void k_interleave_cs(long long nmax, long long shc_nmax,
                                const double *__restrict__ c,
                                const double *__restrict__ s, double2 *cs)
{
    long long m = blockIdx.x;
    if (m > nmax)
        return;
    long long c0 = tri_col0(nmax, m);
    long long s0 = tri_col0(shc_nmax, m);
    for (long long n = m + threadIdx.x; n <= nmax; n += blockDim.x)
        cs[c0 + n - m] = make_double2(c[s0 + n - m], m == 0 ? 0.0 : s[s0 + n - m]);
}

// Sectorial seeds of every latitude pair, src/leg/leg_func_prepare.c:18-69
// with the radial factor (R/r)^(m+1+dorder) (src/shs/shs_rpows.c) folded in:
// psx[m*np + p] * 2^pse[m*np + p] = P_mm(u_p) * rho_p^(m+1+dorder).
// The mantissa sequence is CHarm's (same products, same X-number
// renormalisation), so the seeds agree with CHarm bit for bit when rho = 1.
__global__ void k_sectorial(long long nmax, int np,
                            const double *__restrict__ u,
                            const double *__restrict__ rho, int use_rho,
                            int dorder, const double *__restrict__ dm,
                            double *psx, int *pse)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np)
        return;
    const double BIG = 0x1p960, BIGI = 0x1p-960;
    const double BIGS = 0x1p480, BIGSI = 0x1p-480;
    const double ROOT3 = 1.73205080756887729353;
    double up = u[p];
    double rh = use_rho ? rho[p] : 1.0;
    double rp = 1.0;
    for (int i = 0; i < 1 + dorder; i++)
        rp *= rh;
    psx[p] = rp;
    pse[p] = 0;
    if (nmax == 0)
        return;
    double x = ROOT3 * up;
    int ix = 0;
    rp *= rh;
    psx[(size_t)np + p] = use_rho ? x * rp : x;
    pse[(size_t)np + p] = 0;
    for (long long m = 2; m <= nmax; m++)
    {
        x = (dm[m - 1] * up) * x;
        double w = fabs(x);
        if (w >= BIGS)
        {
            x *= BIGI;
            ix += 1;
        }
        else if (w < BIGSI)
        {
            x *= BIG;
            ix -= 1;
        }
        rp *= rh;
        psx[(size_t)m * np + p] = use_rho ? x * rp : x;
        pse[(size_t)m * np + p] = 960 * ix;
    }
}

// ---------------------------------------------------------------------------
// Synthesis kernel
// ---------------------------------------------------------------------------
struct StageView
{
    double2 *ab;
    double2 *cs;
    double2 *en;
};

template <int KIND, int DL, int DR, int K, bool RR>
__global__ void __launch_bounds__(128)
k_shs_grid(ShsGridArgs A)
{
    using Q = Qty<KIND, DL, DR>;
    constexpr int NQ = Q::NQ;
    constexpr int ND = Q::NEEDD;
    constexpr int NSLOT = ND > 0 ? 3 : 2;

    extern __shared__ __align__(128) unsigned char smem_raw[];
    const unsigned lane = threadIdx.x & 31u;
    const unsigned warp = threadIdx.x >> 5;
    // per warp: 2 stages x NSLOT x LEG_CHUNK double2, then 2 mbarriers
    const size_t stage_bytes = (size_t)NSLOT * LEG_CHUNK * sizeof(double2);
    unsigned char *wbase =
        smem_raw + (size_t)warp * (2 * stage_bytes + 2 * sizeof(uint64_t));
    uint64_t *bar = reinterpret_cast<uint64_t *>(wbase + 2 * stage_bytes);
    StageView st[2];
#pragma unroll
    for (int s = 0; s < 2; s++)
    {
        double2 *b = reinterpret_cast<double2 *>(wbase + s * stage_bytes);
        st[s].ab = b;
        st[s].cs = b + LEG_CHUNK;
        st[s].en = b + 2 * LEG_CHUNK;
    }
    if (lane == 0)
    {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
    }
    __syncwarp();
    unsigned phase[2] = {0u, 0u};

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

        // ---- geometry of this lane's latitude pairs --------------------
        int pk[K];
        double tq[K], tu[K], urr[K], u2r[K], uk[K], rho1[K], rho2[K];
        double x[K], y[K];
        int E[K];
        bool polar_skip = A.polar_thr >= 0.0;
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
            x[k] = valid ? A.psx[(size_t)m * np + p] : 0.0;
            E[k] = valid ? A.pse[(size_t)m * np + p] : 0;
            y[k] = 0.0;
            if (valid && !((double)m - (double)N * u > A.polar_thr))
                polar_skip = false;
        }
        polar_skip = __all_sync(0xffffffffu, polar_skip);

        Acc<NQ, 2, K> acc;
        acc.zero();

        if (!polar_skip)
        {
            const long long c0 = tri_col0(N, m);
            const long long ncol = N - m + 1;
            const int nchunks = (int)((ncol + LEG_CHUNK - 1) / LEG_CHUNK);
            auto issue = [&](int j, int s) {
                if (lane == 0)
                {
                    long long off = c0 + (long long)j * LEG_CHUNK;
                    long long cnt = ncol - (long long)j * LEG_CHUNK;
                    if (cnt > LEG_CHUNK)
                        cnt = LEG_CHUNK;
                    unsigned bytes = (unsigned)(cnt * sizeof(double2));
                    mbar_arrive_expect_tx(&bar[s], bytes * NSLOT);
                    bulk_g2s(st[s].ab, A.ab + off, bytes, &bar[s]);
                    bulk_g2s(st[s].cs, A.cs + off, bytes, &bar[s]);
                    if (ND > 0)
                        bulk_g2s(st[s].en, A.en + off, bytes, &bar[s]);
                }
            };
            issue(0, 0);
            if (nchunks > 1)
                issue(1, 1);

            // seeds: renormalise, unscaled latitudes start contributing now
#pragma unroll
            for (int k = 0; k < K; k++)
                leg_seed_normalise(x[k], E[k]);
            bool any_scaled = false;
#pragma unroll
            for (int k = 0; k < K; k++)
                any_scaled |= (E[k] != 0);
            any_scaled = __any_sync(0xffffffffu, any_scaled);

            const double md = (double)m;
            const double m2 = md * md;

            if (!mbar_wait_bounded(&bar[0], phase[0], A.status))
                break;
            phase[0] ^= 1u;

            // ---- n = m (sectorial, even) ----------------------------------
            {
                double2 c = st[0].cs[0];
                double np1 = md + 1.0;
#pragma unroll
                for (int k = 0; k < K; k++)
                {
                    double p = x[k];
                    double dp = 0.0, ddp = 0.0;
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
            // ---- n = m + 1 (odd, b = 0) -----------------------------------
            if (ncol > 1)
            {
                double a = st[0].ab[1].x;
                double2 c = st[0].cs[1];
                double e = ND > 0 ? st[0].en[1].x : 0.0;
                double nd = md + 1.0;
                double np1 = nd + 1.0;
#pragma unroll
                for (int k = 0; k < K; k++)
                {
                    double xo = x[k];
                    double z = (a * tq[k]) * xo;
                    y[k] = xo;
                    x[k] = z;
                    double dp = 0.0, ddp = 0.0;
                    if (ND >= 1)
                    {
                        if (m == 0)
                            dp = (1.73205080756887729353 * uk[k]) *
                                 (RR ? rho1[k] * xo : xo);
                        else
                            dp = fma(e * urr[k], xo, -((nd * tu[k]) * z));
                    }
                    if (ND >= 2)
                    {
                        if (m == 0)
                            ddp = -z;
                        else
                            ddp = fma(tu[k], dp,
                                      fma(m2, u2r[k], -(nd * np1)) * z);
                    }
#pragma unroll
                    for (int q = 0; q < NQ; q++)
                    {
                        double v = Q::val(q, z, dp, ddp, np1);
                        acc.v[q][0][1][k] = fma(v, c.x, acc.v[q][0][1][k]);
                        acc.v[q][1][1][k] = fma(v, c.y, acc.v[q][1][1][k]);
                    }
                }
            }

            // ---- n = m + 2 .. N --------------------------------------------
            int since_fix = 2;
            bool ok = true;
            for (int j = 0; j < nchunks; j++)
            {
                const int s = j & 1;
                if (j > 0)
                {
                    if (!mbar_wait_bounded(&bar[s], phase[s], A.status))
                    {
                        ok = false;
                        break;
                    }
                    phase[s] ^= 1u;
                }
                long long cntl = ncol - (long long)j * LEG_CHUNK;
                const int cnt = cntl > LEG_CHUNK ? LEG_CHUNK : (int)cntl;
                const double2 *sab = st[s].ab;
                const double2 *scs = st[s].cs;
                const double2 *sen = st[s].en;
                int i = (j == 0) ? 2 : 0;
                for (; i < cnt; i += 2)
                {
                    // two degrees per iteration: even then odd parity
#pragma unroll
                    for (int par = 0; par < 2; par++)
                    {
                        if (par == 1 && i + 1 >= cnt)
                            break;
                        double2 ab = sab[i + par];
                        double2 c = scs[i + par];
                        double2 en = ND > 0 ? sen[i + par]
                                            : make_double2(0.0, 0.0);
                        double nd = ND > 0 ? en.y
                                           : (double)(m + (long long)j * LEG_CHUNK + i + par);
                        double np1 = nd + 1.0;
#pragma unroll
                        for (int k = 0; k < K; k++)
                        {
                            double xo = x[k];
                            double by = RR ? ab.y * (rho2[k] * y[k])
                                           : ab.y * y[k];
                            double z = fma(ab.x * tq[k], xo, -by);
                            y[k] = xo;
                            x[k] = z;
                            double dp = 0.0, ddp = 0.0;
                            if (ND >= 1)
                                dp = fma(en.x * urr[k], xo,
                                         -((nd * tu[k]) * z));
                            if (ND >= 2)
                                ddp = fma(tu[k], dp,
                                          fma(m2, u2r[k], -(nd * np1)) * z);
#pragma unroll
                            for (int q = 0; q < NQ; q++)
                            {
                                double v = (KIND == 0 && DL == 0 && DR == 0)
                                               ? z
                                               : Q::val(q, z, dp, ddp, np1);
                                acc.v[q][0][par][k] =
                                    fma(v, c.x, acc.v[q][0][par][k]);
                                acc.v[q][1][par][k] =
                                    fma(v, c.y, acc.v[q][1][par][k]);
                            }
                        }
                    }
                    since_fix += 2;
                    if (any_scaled && since_fix >= LEG_FIX_EVERY)
                    {
                        since_fix = 0;
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
                    double sg = (h == 0) ? 1.0 : (double)Q::parity(q);
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
                    A.out[o] = make_double2(cpack * A.mur * a[q],
                                            sgnb * (cpack * A.mur * b[q]));
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Longitude sums where FFT does not apply (CHarm's PSLR path,
// src/shs/shs_grd_lr.c, shs_grd_lr2.c): f[q][i][j] = sum_m a cos(m lon_j) +
// b sin(m lon_j), with the angle m*lon_j formed exactly (two-product) before
// the sine and cosine.
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
    double acc = 0.0;
    for (long long m = 0; m <= nmax; m++)
    {
        double ss, cc;
        sincos_mlon((double)m, lj, &ss, &cc);
        double2 v = row[m];
        acc = fma(v.x, cc, fma(v.y, ss, acc));
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
    constexpr int ND = Qty<KIND, DL, DR>::NEEDD;
    constexpr int NSLOT = ND > 0 ? 3 : 2;
    const int warps = 4;
    size_t smem = (size_t)warps *
                  (2 * NSLOT * LEG_CHUNK * sizeof(double2) + 2 * sizeof(uint64_t));
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

cudaError_t launch_tables(long long nmax, const double *r, const double *ri,
                          double2 *ab, double2 *en, cudaStream_t st)
{
    int blocks = (int)(nmax + 1);
    k_table_ab<<<blocks, 128, 0, st>>>(nmax, r, ri, ab);
    if (en)
        k_table_en<<<blocks, 128, 0, st>>>(nmax, r, ri, en);
    return cudaGetLastError();
}

cudaError_t launch_interleave(long long nmax, long long shc_nmax,
                              const double *c, const double *s, double2 *cs,
                              cudaStream_t st)
{
    k_interleave_cs<<<(int)(nmax + 1), 128, 0, st>>>(nmax, shc_nmax, c, s, cs);
    return cudaGetLastError();
}

cudaError_t launch_sectorial(long long nmax, int np, const double *u,
                             const double *rho, int use_rho, int dorder,
                             const double *dm, double *psx, int *pse,
                             cudaStream_t st)
{
    k_sectorial<<<(np + 127) / 128, 128, 0, st>>>(nmax, np, u, rho, use_rho,
                                                   dorder, dm, psx, pse);
    return cudaGetLastError();
}

cudaError_t launch_lon_direct(int npar, int nlat, int nlon, long long nmax,
                              const double2 *lc, int ldf, const double *lon,
                              double *f, cudaStream_t st)
{
    long long total = (long long)npar * nlat * nlon;
    int blocks = (int)((total + 255) / 256);
    k_lon_direct<<<blocks, 256, 0, st>>>(npar, nlat, nlon, nmax, lc, ldf, lon, f);
    return cudaGetLastError();
}

} // namespace cb
