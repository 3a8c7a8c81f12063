// Batched grid synthesis with the degree sums on the tensor cores
// (split precision: exact INT8 digit products, recombined in FP64).
//
// For one order m and a tile of 128 latitude pairs the lumped coefficients
// of all sets of a batch are a product of two matrices,
//     a_s(lat) = sum_n  A[lat][n] B[n][s],
//     A[lat][n] = P_nm(t_lat) (R/r)^(n+1)   (the Legendre block),
//     B[n][s]   = C_nm or S_nm of set s    (32 columns: 16 sets x C, S),
// with the even and odd (n - m) degrees summed separately for the north /
// south symmetry (CHarm's shs_point_kernel, src/shs/shs_point_kernel.c:
// 745-2010, forms the same sums one lane at a time).
//
// Precision.  Both operands become integers on fixed-point grids:
//     A_int = round(A 2^(51 - eA)),  2^eA a bound of |A| on that latitude,
//     B_int = round(B 2^(54 - eB)),  2^eB > max_n |B| of that column,
// each written in base 256 with seven digits: A_int in two's complement
// (digits 0..5 unsigned, the top digit signed), taken straight from the
// mantissa of x c~_n + 1.5 2^52 (one FMA on the recurrence value x already
// carrying 2^(51 - eA), no conversion instruction); B_int with balanced
// digits in [-128, 127] (the bytes of
// B_int + sum_i 128 256^i, minus 128), so that every dropped product has
// zero mean.  The digit products a_i b_j are exact in the INT32
// accumulators of tcgen05.mma kind::i8; products of level s = i + j are
// summed in one accumulator and weighted by 256^s in FP64 afterwards.
// Levels below 5 are dropped: they hold about 2^-53 of a typical term.
// 34 digit pairs per degree tile and parity, issued as 7 MMAs (one per
// Legendre digit against the stack of coefficient digits it meets, N =
// 64..224); 8 levels x 2 parities x 32 columns = all 512 TMEM columns.
//
// The fixed-point grid of the Legendre values of each (order, latitude) is
// chosen from a bound of |P_nm| (k_tc_seeds); a value outside it sets
// DEV_ERR_TC_RANGE and the call fails.
//
// Pipeline per CTA (one latitude pair per TMEM lane; warp roles at
// k_shs_tc): the coefficient digit tiles and the recurrence tables of a
// 64-degree chunk arrive by bulk copies, three chunks ahead of the MMAs
// (four stages, streamed across work items); 128 threads run the rescaled
// recurrence of leg.cuh in FP64, cut the values into digits and store them
// as the K-major operand tiles (two stages); a producer lane issues the 14
// MMAs of the chunk and commits them to an mbarrier, so the tensor cores
// work on chunk j while the threads prepare chunk j + 1; epilogue warps
// drain an item's accumulators while the next item is prepared.
#include <cstdint>
#include <type_traits>

#include "common.cuh"
#include "kernels.h"
#include "leg.cuh"
#include "synth.cuh"

namespace cb
{

namespace
{

constexpr int TC_M = 128;          // latitude pairs per item = TMEM lanes
constexpr int TC_COLS = 32;        // accumulator columns
constexpr int TC_D = 7;            // digits per operand
constexpr int TC_LMIN = 5;         // lowest product level kept
constexpr int TC_NLEV = 2 * TC_D - 1 - TC_LMIN;        // 8
static_assert(TC_NLEV == 8, "the epilogue groups the levels 3 + 3 + 2");
constexpr int TC_ATILE = TC_M * 32;                    // bytes
constexpr int TC_BTILE = TC_COLS * 32;                 // bytes
constexpr int TC_ASTAGE = 2 * TC_D * TC_ATILE;         // 57344
constexpr int TC_BSTAGE = 2 * TC_D * TC_BTILE;         // 14336
constexpr int TC_CH = 64;                              // degrees per chunk
constexpr int TC_NB = 4;           // coefficient / table stages
// the producer loads chunk g + TC_AHEAD + 1 once the MMAs of chunk g - 1
// (the last user of that stage) are complete
constexpr int TC_AHEAD = TC_NB - 2;
constexpr unsigned TC_TMEM_COLS = 512;
// offset of the balanced digits of the coefficients: sum_{i<7} 128 256^i
constexpr unsigned long long TC_BIAS = 0x0080808080808080ull;
// x + 1.5 2^52 holds round(x) in its low mantissa bits for |x| < 2^51:
// bits = 0x4338000000000000 + round(x) (two's complement)
constexpr double TC_MAGIC = 6755399441055744.0;

// byte offset of (row r, byte k) in a [rows x 32 B] K-major operand tile
// without swizzle: 8-row x 16-byte core matrices, the two K halves of a
// row group 128 B apart (leading byte offset), row groups 256 B apart
// (stride byte offset)
__host__ __device__ __forceinline__ int tc_tile_off(int r, int k)
{
    return (r >> 3) * 256 + (k >> 4) * 128 + (r & 7) * 16 + (k & 15);
}

// shared-memory matrix descriptor of such a tile (sm_100 layout: start
// address, LBO and SBO in 16-byte units, version 1, no swizzle)
__device__ __forceinline__ uint64_t tc_sdesc(uint32_t addr)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) |
           ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(256u >> 4) << 32) |
           ((uint64_t)1 << 46);
}

// instruction descriptors: D int32, B signed 8-bit, A unsigned (digits
// 0..5 of the Legendre values) or signed (their top digit), both K-major,
// M = 128, N = TC_COLS
// (N in bits 17..22, in units of 8)
constexpr uint32_t TC_IDESC_U = (2u << 4) | (0u << 7) | (1u << 10) |
                                ((uint32_t)(TC_M >> 4) << 24);
constexpr uint32_t TC_IDESC_S = TC_IDESC_U | (1u << 7);

__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b,
                                       uint32_t idesc, uint32_t acc)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
                 ::"r"(d), "l"(a), "l"(b), "r"(idesc), "r"(acc)
                 : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::"
                 "cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before()
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_after()
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 8 consecutive accumulator columns of this warp's 32 lanes
__device__ __forceinline__ void tc_ld8(uint32_t taddr, int (&v)[8])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]),
                   "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(taddr));
}

// 2 consecutive accumulator columns of this warp's 32 lanes (the column
// offset is even)
__device__ __forceinline__ void tc_ld2(uint32_t taddr, int (&v)[2])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];"
                 : "=r"(v[0]), "=r"(v[1])
                 : "r"(taddr));
}

__device__ __forceinline__ void tc_wait_ld()
{
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// zeros into 16 consecutive accumulator columns of this warp's 32 lanes
__device__ __forceinline__ void tc_st_zero16(uint32_t taddr)
{
    const unsigned z = 0u;
    asm volatile("tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
                 "{%1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, "
                 "%1, %1};" ::"r"(taddr), "r"(z)
                 : "memory");
}

// zeros into 2 consecutive accumulator columns (even offset)
__device__ __forceinline__ void tc_st_zero2(uint32_t taddr)
{
    const unsigned z = 0u;
    asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %1};"
                 ::"r"(taddr), "r"(z)
                 : "memory");
}

__device__ __forceinline__ void tc_wait_st()
{
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// exact int64 -> double for |u| < 2^51 with one integer add and one DADD:
// the bits 0x4338000000000000 + u are 1.5 2^52 + u
__device__ __forceinline__ double l2d_exact(long long u)
{
    return __longlong_as_double(u + 0x4338000000000000LL) - TC_MAGIC;
}

// 2^e for |e| < 1000 (exact)
__device__ __forceinline__ double pow2i(int e)
{
    return __hiloint2double((e + 1023) << 20, 0);
}

// Bytes d of four 64-bit words v0..v3 (as lo / hi halves) gathered into
// one word per digit: w[d] = {v0.b_d, v1.b_d, v2.b_d, v3.b_d}.
__device__ __forceinline__ void tc_transpose4(const unsigned (&lo)[4],
                                              const unsigned (&hi)[4],
                                              unsigned (&w)[TC_D])
{
    unsigned a = __byte_perm(lo[0], lo[1], 0x5140);
    unsigned b = __byte_perm(lo[0], lo[1], 0x7362);
    unsigned c = __byte_perm(lo[2], lo[3], 0x5140);
    unsigned d = __byte_perm(lo[2], lo[3], 0x7362);
    w[0] = __byte_perm(a, c, 0x5410);
    w[1] = __byte_perm(a, c, 0x7632);
    w[2] = __byte_perm(b, d, 0x5410);
    w[3] = __byte_perm(b, d, 0x7632);
    unsigned e = __byte_perm(hi[0], hi[1], 0x5140);
    unsigned f = __byte_perm(hi[0], hi[1], 0x7362);
    unsigned g = __byte_perm(hi[2], hi[3], 0x5140);
    unsigned h = __byte_perm(hi[2], hi[3], 0x7362);
    w[4] = __byte_perm(e, g, 0x5410);
    w[5] = __byte_perm(e, g, 0x7632);
    w[6] = __byte_perm(f, h, 0x5410);
}

} // namespace

// ---------------------------------------------------------------------------
// Preparation of the coefficient operand
// ---------------------------------------------------------------------------
// Column exponents: ecol[m][c] with 2^ecol > max_n |B[n][c]| (0 for an
// all-zero column).  One block per order m, one warp per set.
__global__ void k_tc_colexp(ShsTcPrep P)
{
    const long long m = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (m > P.nmax || warp >= 16)
        return;
    double mc = 0.0, ms = 0.0;
    if (warp < P.nsets && m <= P.set_nmax[warp])
    {
        const long long s0 = tri_col0(P.shc_nmax[warp], m);
        const double *c = P.c[warp] + s0 - m;
        const double *s = P.s[warp] + s0 - m;
        for (long long n = m + lane; n <= P.set_nmax[warp]; n += 32)
        {
            mc = fmax(mc, fabs(c[n]));
            if (m > 0)
                ms = fmax(ms, fabs(s[n]));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        mc = fmax(mc, __shfl_xor_sync(0xffffffffu, mc, o));
        ms = fmax(ms, __shfl_xor_sync(0xffffffffu, ms, o));
    }
    if (lane == 0)
    {
        // columns below 2^-900 are scaled as if of that size (their digits
        // vanish); the range keeps every power of two of the kernels normal
        const int ec = mc > 0.0 ? max(expo_of(mc) + 1, -900) : 0;
        const int es = ms > 0.0 ? max(expo_of(ms) + 1, -900) : 0;
        P.ecol[m * TC_COLS + 2 * warp] = ec;
        P.ecol[m * TC_COLS + 2 * warp + 1] = es;
        if (!isfinite(mc) || !isfinite(ms))
            atomicOr(P.status, DEV_ERR_BAD_ARGS);
    }
}

// The coefficient families of the gradients.  With A_n = P_nm (R/r)^(n+1)
// the Legendre operand and X = C or S of one set, the potential, grad1 and
// grad2 need, per latitude, the sums over n of A_n times
//   f = 0: X_n,  1: n X_n,  2: n (n + 1) X_n,
//   f = 3: e_(n+1) X_(n+1),  4: n e_(n+1) X_(n+1),
// e_n = sqrt((n - m)(n + m)(2n + 1) / (2n - 1)) (src/leg/leg_func_enm.c):
// cos(lat) dP_n/dlat = e_n P_n-1 - n sin(lat) P_n shifts the first term to
// the Legendre index n - 1 (families 3, 4), and the Legendre equation
// d2P_n/dlat2 = tan(lat) dP_n/dlat - (n (n + 1) - m^2 / cos^2(lat)) P_n
// gives the second derivatives -- the per-degree relations CHarm's
// kernels (src/shs/shs_point_kernel.c:1639-1946) and shs_grid.cu use.
// src[n] = X_nm, nset the set's degree.
__device__ __forceinline__ double tc_family(int f, long long m, long long n,
                                            const double *src, long long nset)
{
    const double nd = (double)n;
    if (f <= 2)
    {
        if (n > nset)
            return 0.0;
        const double x = src[n];
        return f == 0 ? x : (f == 1 ? nd * x : (nd * (nd + 1.0)) * x);
    }
    const long long n1 = n + 1;
    if (n1 > nset)
        return 0.0;
    const double n1d = (double)n1, md = (double)m;
    const double e = sqrt(((n1d - md) * (n1d + md)) * (2.0 * n1d + 1.0) /
                          (2.0 * n1d - 1.0));
    const double x = e * src[n1];
    return f == 3 ? x : nd * x;
}

// Column exponents of the gradient families: column 10 set + 2 f + (C, S),
// one warp per column.
__global__ void k_tc_colexp_grad(ShsTcPrep P)
{
    const long long m = blockIdx.x;
    const int col = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (m > P.nmax)
        return;
    const int set = col / (2 * SHS_TC_FAMILIES);
    const int f = (col % (2 * SHS_TC_FAMILIES)) >> 1;
    const bool is_s = col & 1;
    double mx = 0.0;
    if (set < P.nsets && m <= P.set_nmax[set] && !(is_s && m == 0))
    {
        const long long s0 = tri_col0(P.shc_nmax[set], m);
        const double *src = (is_s ? P.s[set] : P.c[set]) + s0 - m;
        for (long long n = m + lane; n <= P.set_nmax[set]; n += 32)
            mx = fmax(mx, fabs(tc_family(f, m, n, src, P.set_nmax[set])));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0)
    {
        P.ecol[m * TC_COLS + col] = mx > 0.0 ? max(expo_of(mx) + 1, -900) : 0;
        if (!isfinite(mx))
            atomicOr(P.status, DEV_ERR_BAD_ARGS);
    }
}

// Digit tiles of every (order, chunk): [parity][digit][32 columns x 32 B].
// One block per order, thread = (parity, column, 16-degree half).
__global__ void __launch_bounds__(128) k_tc_bdigits(ShsTcPrep P)
{
    const long long m = blockIdx.x;
    if (m > P.nmax)
        return;
    const int t = threadIdx.x;
    const int p = t >> 6, col = (t >> 1) & 31, h = t & 1;
    // potential: columns (C, S) per set; gradients: 10 per set
    const int set = P.grad ? col / (2 * SHS_TC_FAMILIES) : (col >> 1);
    const int fam = P.grad ? (col % (2 * SHS_TC_FAMILIES)) >> 1 : 0;
    const bool is_s = col & 1;
    const bool active = set < P.nsets && m <= P.set_nmax[set] &&
                        !(is_s && m == 0);
    const double *src = nullptr;
    long long nset = -1;
    if (active)
    {
        const long long s0 = tri_col0(P.shc_nmax[set], m);
        src = (is_s ? P.s[set] : P.c[set]) + s0 - m;
        nset = P.set_nmax[set];
    }
    const double sc = pow2i(54 - P.ecol[m * TC_COLS + col]);
    const long long nch = (P.nmax - m + TC_CH) / TC_CH;
    unsigned char *base = P.bdig + (size_t)P.chunk0[m] * TC_BSTAGE;
    for (long long j = 0; j < nch; j++)
    {
        unsigned w[TC_D][4];
#pragma unroll
        for (int q = 0; q < 4; q++)
        {
            unsigned lo[4], hi[4];
#pragma unroll
            for (int b = 0; b < 4; b++)
            {
                const int k = 16 * h + 4 * q + b;
                const long long n = m + j * TC_CH + 2 * k + p;
                double v =
                    (n <= nset) ? tc_family(fam, m, n, src, nset) * sc : 0.0;
                unsigned long long y =
                    (unsigned long long)__double2ll_rn(v) + TC_BIAS;
                lo[b] = (unsigned)y;
                hi[b] = (unsigned)(y >> 32);
            }
            unsigned wd[TC_D];
            tc_transpose4(lo, hi, wd);
#pragma unroll
            for (int d = 0; d < TC_D; d++)
                w[d][q] = wd[d] ^ 0x80808080u;
        }
        unsigned char *ch = base + (size_t)j * TC_BSTAGE;
#pragma unroll
        for (int d = 0; d < TC_D; d++)
        {
            uint4 *dst = reinterpret_cast<uint4 *>(
                ch + (p * TC_D + d) * TC_BTILE + tc_tile_off(col, 16 * h));
            *dst = make_uint4(w[d][0], w[d][1], w[d][2], w[d][3]);
        }
    }
}

// beta_n and ct_n of every order in rows of ldmul * 64 entries, zero
// beyond the order's last degree: each chunk's slice is one 16-byte aligned
// bulk copy, and the padding makes the tail of the last chunk contribute
// nothing without a test per degree.  ct is stored by parity within each
// chunk (the 32 even-(n - m) degrees, then the 32 odd ones).
__global__ void k_tc_ctab(long long nmax, int ld, const double2 *__restrict__ tb,
                          const double *__restrict__ tc, double *btp,
                          double *ctp)
{
    const long long m = blockIdx.x;
    if (m > nmax)
        return;
    const long long c0 = tri_col0(nmax, m);
    const long long ncol = nmax - m + 1;
    for (long long i = threadIdx.x; i < ld; i += blockDim.x)
    {
        btp[m * ld + i] = i < ncol ? tb[c0 + i].x : 0.0;
        // ct in [chunk][parity][32] order: degree offset 64 j + 2 k + p
        const long long r = i & 63;
        const long long src = (i - r) + 2 * (r & 31) + (r >> 5);
        ctp[m * ld + i] = src < ncol ? tc[c0 + src] : 0.0;
    }
}

// Seeds of every (order, latitude pair), once per call: the sectorial value
// R~_mm (leg.cuh), its binary exponent E while below the double range, and
// the exponent eA of the fixed-point grid of that latitude and order, i.e.
// 2^eA > min(sqrt(2N + 1), 6 (m + 1)^(1/4) / sqrt(cos lat)) (times (R/r)^(N+1)
// below the sphere): |P_nm| <= sqrt(2n + 1) holds for the geodetic
// normalisation, and sqrt(cos lat) |P_nm| stays below 4.2 (m + 1)^(1/4) for
// all n, m <= 2190 (evaluated on 190 latitudes).  Values in range are
// stored already multiplied by 2^(51 - eA).
template <bool RR>
__global__ void k_tc_seeds(ShsTcArgs A, double *seed_x, int2 *seed_e)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long np = A.npairs;
    if (idx >= (A.nmax + 1) * np)
        return;
    const long long m = idx / np;
    const int p = (int)(idx % np);
    const double u = A.u[p];
    const double rh = RR ? A.rho[p] : 1.0;
    double x;
    int E;
    leg_seed(A.sg[2 * m], u, rh, RR, m, 0, x, E);
    double bnd = sqrt(2.0 * (double)A.nmax + 1.0);
    if (u > 0.0)
        bnd = fmin(bnd, 6.0 * sqrt(sqrt((double)m + 1.0)) / sqrt(u));
    if (RR && rh > 1.0)
        bnd *= pow(rh, (double)(A.nmax + 1));
    const int eA = expo_of(bnd) + 1;
    if (E == 0)
        x *= pow2i(51 - eA);
    seed_x[idx] = x;
    seed_e[idx] = make_int2(E, eA);
}

// ---------------------------------------------------------------------------
// The contraction kernel
// ---------------------------------------------------------------------------
// Warp roles (13 warps):
//   0..3  preparation: one latitude pair per thread (TMEM lane 32 w + l);
//         per chunk the recurrence on 64 degrees, fixed point, digits into
//         A stage g % 2, then an arrival on bar_a;
//   4     producer (lane 0): bulk loads TC_AHEAD + 1 chunks ahead of the
//         MMAs, the 14 MMAs of each chunk once bar_a completes, a commit per
//         chunk (bar_m: its stages are free again) and per work item
//         (bar_acc: the accumulators hold the item's sums);
//   5..12 epilogue: after bar_acc, read the accumulators (warp w: lanes of
//         quarter w % 4, half of the columns), recombine, write, clear them
//         and arrive on bar_free, which the producer waits for before the
//         next item's first MMA.
// The preparation of the next item runs while the tensor cores finish an
// item and the epilogue drains it.  Every wait is bounded; a wait that gives
// up raises the CTA's abort flag, which every loop reads, so all roles
// reach the final barrier.
constexpr int TC_PREP = 128;
constexpr int TC_THREADS = 13 * 32;
constexpr int TC_RING = 8;          // work items in flight (ring of ids)

// barrier among the preparation threads (id 1) with an OR of a predicate
__device__ __forceinline__ bool tc_prep_or(bool v)
{
    unsigned r;
    asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\t"
                 "barrier.red.or.pred q, 1, 128, p;\n\tselp.u32 %0, 1, 0, q;\n\t}"
                 : "=r"(r)
                 : "r"((unsigned)v)
                 : "memory");
    return r != 0;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("{\n\t.reg .b64 st;\n\t"
                 "mbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

template <bool RR, bool GRAD>
__global__ void __launch_bounds__(TC_THREADS, 1) k_shs_tc(ShsTcArgs A)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char *sA = smem_raw;                         // 2 stages
    unsigned char *sB = sA + 2 * TC_ASTAGE;               // TC_NB stages
    double *sBt = reinterpret_cast<double *>(sB + TC_NB * TC_BSTAGE);
    double *sCt = sBt + TC_NB * TC_CH;
    double *sZero = sCt + TC_NB * TC_CH;                  // ct of no latitude
    uint64_t *bar_b = reinterpret_cast<uint64_t *>(sZero + TC_CH);
    uint64_t *bar_m = bar_b + TC_NB;                      // 2
    uint64_t *bar_a = bar_m + 2;                          // 2
    uint64_t *bar_acc = bar_a + 2;
    uint64_t *bar_free = bar_acc + 1;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar_free + 1);
    volatile int *sAbort = reinterpret_cast<volatile int *>(tslot + 1);
    // work items in order of issue, written by the producer when its load
    // cursor reaches them (several chunks before anyone reads them)
    volatile unsigned long long *sQ =
        reinterpret_cast<volatile unsigned long long *>(tslot + 4);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32"
                     " [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(TC_TMEM_COLS)
                     : "memory");
        asm volatile(
            "tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::
                : "memory");
    }
    if (tid < TC_CH)
        sZero[tid] = 0.0;
    if (tid == 0)
    {
        for (int i = 0; i < TC_NB; i++)
            mbar_init(&bar_b[i], 1);
        for (int i = 0; i < 2; i++)
        {
            mbar_init(&bar_m[i], 1);
            mbar_init(&bar_a[i], TC_PREP);
        }
        mbar_init(bar_acc, 1);
        mbar_init(bar_free, 8 * 32);
        fence_mbar_init();
        *sAbort = 0;
    }
    // degrees of this launch's sets (<= the tables' A.nmax): work items,
    // chunks and digit tiles stop here
    const long long N = A.nmax_sets;
    const int np = A.npairs;

    // ---- load cursor (producer lane 0) ----
    unsigned long long lk = 0;
    long long lm = 0, lj = 0, lnch = 0;
    bool lend = false;
    auto fetch_item = [&]() {
        const unsigned long long it = atomicAdd(A.counter, 1ull);
        sQ[lk % TC_RING] = it;
        if (it >= (unsigned long long)A.nitems)
        {
            lend = true;
            return;
        }
        lm = (long long)(it / (unsigned long long)A.ntiles);
        lj = 0;
        lnch = (N - lm + TC_CH) / TC_CH;
    };
    // loads chunk gg; the id of the next item is published before the
    // arrival on this chunk's barrier (release), so a thread that has
    // waited for the last chunk of an item also sees the next item's id
    auto issue_next = [&](unsigned long long gg) {
        if (lend)
            return;
        const long long cm = lm, cj = lj;
        if (++lj == lnch)
        {
            ++lk;
            fetch_item();
        }
        const int s = (int)(gg % TC_NB);
        const long long trow = cm * (long long)A.ldmul * TC_CH + cj * TC_CH;
        mbar_arrive_expect_tx(&bar_b[s],
                              TC_BSTAGE + 2 * TC_CH * sizeof(double));
        bulk_g2s(sB + s * TC_BSTAGE,
                 A.bdig + ((size_t)A.chunk0[cm] + (size_t)cj) * TC_BSTAGE,
                 TC_BSTAGE, &bar_b[s]);
        bulk_g2s(sBt + s * TC_CH, A.btp + trow, TC_CH * sizeof(double),
                 &bar_b[s]);
        bulk_g2s(sCt + s * TC_CH, A.ctp + trow, TC_CH * sizeof(double),
                 &bar_b[s]);
    };
    if (warp == 4 && lane == 0)
    {
        fetch_item();
        for (int a = 0; a <= TC_AHEAD; a++)
            issue_next((unsigned long long)a);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    if (warp < 4)
    {
        // ================= preparation =================
        const int row = tid;
        unsigned long long g = 0;
        unsigned range_err = 0u;
        // seed, exponents and geometry of an item's latitude pair
        double nx_x = 0.0, nx_t = 0.0, nx_rh = 1.0;
        int2 nx_e = make_int2(0, 0);
        bool have_next = false;
        auto load_seed = [&](unsigned long long it) {
            const long long mm = (long long)(it / (unsigned long long)A.ntiles);
            const int pp = (int)(it % (unsigned long long)A.ntiles) * TC_M + row;
            nx_x = 0.0;
            nx_t = 0.0;
            nx_rh = 1.0;
            nx_e = make_int2(0, 0);
            if (pp < np)
            {
                const long long i = mm * (long long)np + pp;
                nx_x = A.seed_x[i];
                nx_e = A.seed_e[i];
                nx_t = A.t[pp];
                if (RR)
                    nx_rh = A.rho[pp];
            }
        };
        for (unsigned long long k = 0;; k++)
        {
            // the same id for all 128 threads (written before the barrier
            // arrival they all waited for); aborts are decided together at
            // the end of an item
            const unsigned long long item = sQ[k % TC_RING];
            if (item >= (unsigned long long)A.nitems)
                break;
            const long long m =
                (long long)(item / (unsigned long long)A.ntiles);
            const int tile = (int)(item % (unsigned long long)A.ntiles);
            const int p = tile * TC_M + row;
            const bool valid = p < np;
            // this item's seed (prefetched during the previous item's last
            // chunk, or loaded now for the first item)
            if (!have_next)
                load_seed(item);
            const double tq = RR ? nx_t * nx_rh : nx_t;
            const double rho2 = nx_rh * nx_rh;
            double x = nx_x, y = 0.0;
            int E = nx_e.x;
            const int eA = nx_e.y;
            have_next = false;
            const double rs = pow2i(51 - eA);
            const long long ncol = N - m + 1;
            const int nch = (int)((ncol + TC_CH - 1) / TC_CH);
            double mul_next = 1.0;
            bool bad = false;
            for (int j = 0; j < nch; j++, g++)
            {
                const int sa = (int)(g & 1), sb = (int)(g % TC_NB);
                // after a wait gave up, the rest of the item only keeps
                // the barrier sequence of the preparation threads
                bool wok = !bad &&
                           (g < 2 ||
                            mbar_wait_bounded(&bar_m[sa],
                                              (unsigned)(((g - 2) >> 1) & 1),
                                              A.status));
                wok = wok && mbar_wait_bounded(&bar_b[sb],
                                               (unsigned)((g / TC_NB) & 1),
                                               A.status);
                if (j > 0)
                {
                    x *= mul_next;
                    y *= mul_next;
                }
                if (j + 1 < nch)
                    mul_next = A.tmul[m * A.ldmul + j + 1];
                else if (wok)
                {
                    // the next item's id was published before this chunk's
                    // load barrier: fetch its seeds while this chunk runs
                    const unsigned long long nit = sQ[(k + 1) % TC_RING];
                    if (nit < (unsigned long long)A.nitems)
                    {
                        load_seed(nit);
                        have_next = true;
                    }
                }
                unsigned char *at = sA + sa * TC_ASTAGE;
                const double2 *bt2 =
                    reinterpret_cast<const double2 *>(sBt + sb * TC_CH);
                // lanes below the double range (or past the grid): ct = 0
                const double2 *ct2 = reinterpret_cast<const double2 *>(
                    (valid && E == 0) ? sCt + sb * TC_CH : sZero);
                unsigned ov = 0u;
                auto prep = [&](auto first_c) {
                    constexpr bool FIRST = decltype(first_c)::value;
#pragma unroll 1
                    for (int hh = 0; hh < 2; hh++)
                    {
                        unsigned wE[TC_D][4], wO[TC_D][4];
#pragma unroll
                        for (int q = 0; q < 4; q++)
                        {
                            unsigned loE[4], hiE[4], loO[4], hiO[4];
                            double2 bp[4], cpE[2], cpO[2];
#pragma unroll
                            for (int kk = 0; kk < 4; kk++)
                                bp[kk] = bt2[16 * hh + 4 * q + kk];
                            cpE[0] = ct2[8 * hh + 2 * q];
                            cpE[1] = ct2[8 * hh + 2 * q + 1];
                            cpO[0] = ct2[16 + 8 * hh + 2 * q];
                            cpO[1] = ct2[16 + 8 * hh + 2 * q + 1];
#pragma unroll
                            for (int b = 0; b < 8; b++)
                            {
                                const double beta =
                                    (b & 1) ? bp[b >> 1].y : bp[b >> 1].x;
                                if (!(FIRST && q == 0 && b == 0 && hh == 0))
                                {
                                    const double by = RR ? beta * (rho2 * y)
                                                         : beta * y;
                                    const double z = fma(tq, x, -by);
                                    y = x;
                                    x = z;
                                }
                                const int kv = b >> 1;
                                const double2 c2 =
                                    (b & 1) ? cpO[kv >> 1] : cpE[kv >> 1];
                                const double ctn = (kv & 1) ? c2.y : c2.x;
                                // round(x ct) in two's complement from the
                                // mantissa of x ct + 1.5 2^52; the exponent
                                // field checks |x ct| < 2^51
                                const double tv = fma(x, ctn, TC_MAGIC);
                                const unsigned hw =
                                    (unsigned)__double2hiint(tv);
                                const unsigned lo =
                                    (unsigned)__double2loint(tv);
                                ov |= hw ^ 0x43300000u;
                                const unsigned hi = hw - 0x43380000u;
                                if (b & 1)
                                {
                                    loO[kv] = lo;
                                    hiO[kv] = hi;
                                }
                                else
                                {
                                    loE[kv] = lo;
                                    hiE[kv] = hi;
                                }
                            }
                            unsigned wd[TC_D];
                            tc_transpose4(loE, hiE, wd);
#pragma unroll
                            for (int d = 0; d < TC_D; d++)
                                wE[d][q] = wd[d];
                            tc_transpose4(loO, hiO, wd);
#pragma unroll
                            for (int d = 0; d < TC_D; d++)
                                wO[d][q] = wd[d];
                        }
                        const int off = tc_tile_off(row, 16 * hh);
#pragma unroll
                        for (int d = 0; d < TC_D; d++)
                        {
                            *reinterpret_cast<uint4 *>(at + d * TC_ATILE +
                                                       off) =
                                make_uint4(wE[d][0], wE[d][1], wE[d][2],
                                           wE[d][3]);
                            *reinterpret_cast<uint4 *>(
                                at + (TC_D + d) * TC_ATILE + off) =
                                make_uint4(wO[d][0], wO[d][1], wO[d][2],
                                           wO[d][3]);
                        }
                    }
                };
                if (wok && !bad)
                {
                    if (j == 0)
                        prep(std::integral_constant<bool, true>{});
                    else
                        prep(std::integral_constant<bool, false>{});
                }
                else
                {
                    bad = true;
                    *sAbort = 1;
                }
                range_err |= ov >> 20;
                // scaled lanes renormalise on their own (no barrier: a
                // lane's state does not depend on the others')
                if (valid && E != 0 && leg_fixup(x, y, E))
                {
                    x *= rs;
                    y *= rs;
                }
                fence_proxy_async_smem();
                mbar_arrive(&bar_a[sa]);
            }
            // a uniform decision to stop (a wait of some thread gave up)
            if (tc_prep_or(bad || *sAbort))
                break;
        }
        if (range_err)
            atomicOr(A.status, DEV_ERR_TC_RANGE);
    }
    else if (warp == 4)
    {
        // ================= producer =================
        if (lane == 0)
        {
            unsigned long long g = 0;
            for (unsigned long long k = 0;; k++)
            {
                const unsigned long long item = sQ[k % TC_RING];
                if (item >= (unsigned long long)A.nitems || *sAbort)
                    break;
                const long long m =
                    (long long)(item / (unsigned long long)A.ntiles);
                const int nch = (int)((N - m + TC_CH) / TC_CH);
                bool ok = true;
                for (int j = 0; j < nch && ok; j++, g++)
                {
                    const int sa = (int)(g & 1), sb = (int)(g % TC_NB);
                    ok = mbar_wait_bounded(&bar_a[sa],
                                           (unsigned)((g >> 1) & 1),
                                           A.status) &&
                         mbar_wait_bounded(&bar_b[sb],
                                           (unsigned)((g / TC_NB) & 1),
                                           A.status);
                    // the accumulators are free (cleared by the epilogue of
                    // the previous item, or at the start)
                    if (ok && j == 0)
                        ok = mbar_wait_bounded(bar_free, (unsigned)(k & 1),
                                               A.status);
                    if (!ok || *sAbort)
                    {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint64_t da0 =
                        tc_sdesc(smem_u32(sA + sa * TC_ASTAGE));
                    const uint64_t db0 =
                        tc_sdesc(smem_u32(sB + sb * TC_BSTAGE));
#pragma unroll
                    for (int pp = 0; pp < 2; pp++)
#pragma unroll
                        for (int ia = 0; ia < TC_D; ia++)
                        {
                            // Legendre digit ia against the stack of
                            // coefficient digits jb >= j0: block jb lands in
                            // the accumulator of level ia + jb - TC_LMIN
                            const int j0 = ia < TC_LMIN ? TC_LMIN - ia : 0;
                            const int n = TC_COLS * (TC_D - j0);
                            const uint64_t da =
                                da0 + (uint64_t)(((pp * TC_D + ia) *
                                                  TC_ATILE) >>
                                                 4);
                            const uint64_t db =
                                db0 + (uint64_t)(((pp * TC_D + j0) *
                                                  TC_BTILE) >>
                                                 4);
                            const uint32_t d =
                                tmem + (uint32_t)((pp * TC_NLEV + ia + j0 -
                                                   TC_LMIN) *
                                                  TC_COLS);
                            const uint32_t idesc =
                                (ia == TC_D - 1 ? TC_IDESC_S : TC_IDESC_U) |
                                ((uint32_t)(n >> 3) << 17);
                            tc_mma(d, da, db, idesc, 1u);
                        }
                    tc_commit(&bar_m[sa]);
                    if (j == nch - 1)
                        tc_commit(bar_acc);
                    // chunk g + TC_AHEAD + 1 goes to the stage of chunk
                    // g - 1, whose MMAs are the latest on that barrier
                    if (g >= 1 &&
                        !mbar_wait_bounded(&bar_m[(g - 1) & 1],
                                           (unsigned)(((g - 1) >> 1) & 1),
                                           A.status))
                    {
                        ok = false;
                        break;
                    }
                    issue_next(g + TC_AHEAD + 1);
                }
                if (!ok)
                {
                    *sAbort = 1;
                    break;
                }
            }
            // the last commit: all MMAs of this CTA are complete before the
            // accumulators are released
            if (g > 0)
                mbar_wait_bounded(&bar_m[(g - 1) & 1],
                                  (unsigned)(((g - 1) >> 1) & 1), A.status);
        }
        __syncwarp();
    }
    else
    {
        // ================= epilogue =================
        const int quarter = warp & 3;
        const int half = (warp - 5) >> 2;                 // columns half
        const int row = quarter * 32 + lane;
        const uint32_t lane_base = tmem + ((uint32_t)(quarter * 32) << 16);
        // clear this warp's half of the accumulator columns
        auto clear = [&]() {
            const uint32_t hb = lane_base + (uint32_t)(half * 16);
#pragma unroll 1
            for (int pl = 0; pl < 2 * TC_NLEV; pl++)
                tc_st_zero16(hb + (uint32_t)(pl * TC_COLS));
            tc_wait_st();
        };
        clear();
        tc_fence_before();
        mbar_arrive(bar_free);
        for (unsigned long long k = 0;; k++)
        {
            const unsigned long long item = sQ[k % TC_RING];
            if (__any_sync(0xffffffffu,
                           item >= (unsigned long long)A.nitems || *sAbort))
                break;
            // the item's rows, grid exponent and column exponents (lane
            // l: column l), loaded while the tensor cores finish its sums
            const long long m =
                (long long)(item / (unsigned long long)A.ntiles);
            const int tile = (int)(item % (unsigned long long)A.ntiles);
            const int p = tile * TC_M + row;
            const bool valid = p < np;
            int rown = -1, rows = -1, eA = 0;
            if (valid)
            {
                rown = A.row_n[p];
                rows = A.row_s[p];
                eA = A.seed_e[m * (long long)np + p].y;
            }
            const int ecl = __ldg(&A.ecol[m * TC_COLS + lane]);
            bool eok = mbar_wait_bounded(bar_acc, (unsigned)(k & 1),
                                         A.status);
            eok = __all_sync(0xffffffffu, eok);
            if (!eok)
            {
                *sAbort = 1;
                break;
            }
            tc_fence_after();
            const double cpack = m == 0 ? 1.0 : 0.5;
            const double rsi = pow2i(eA - 105);
            if constexpr (GRAD)
            {
                // potential, grad1 and grad2 from the five families of
                // each set (tc_family): half 0 of the warps takes sets 0 and
                // 2, half 1 set 1
                const double t = valid ? A.t[p] : 0.0;
                const double u = valid ? A.u[p] : 1.0;
                const double rho = (RR && valid) ? A.rho[p] : 1.0;
                const double ur = u > 0.0 ? 1.0 / u : 0.0;
                const double u2 = ur * ur;
                const double md = (double)m;
                const size_t qs = (size_t)A.nlat * (size_t)A.ldf;
#pragma unroll 1
                for (int set = half; set < A.nsets; set += 2)
                {
                    // [parity][family][C, S], scaled to the coefficients
                    double V[2][SHS_TC_FAMILIES][2];
#pragma unroll 1
                    for (int f = 0; f < SHS_TC_FAMILIES; f++)
                    {
                        const int col = 2 * SHS_TC_FAMILIES * set + 2 * f;
#pragma unroll
                        for (int pp = 0; pp < 2; pp++)
                        {
                            int v[TC_NLEV][2];
#pragma unroll
                            for (int L = 0; L < TC_NLEV; L++)
                                tc_ld2(lane_base +
                                           (uint32_t)((pp * TC_NLEV + L) *
                                                          TC_COLS +
                                                      col),
                                       v[L]);
                            tc_wait_ld();
#pragma unroll
                            for (int cs = 0; cs < 2; cs++)
                            {
                                const long long u0 =
                                    (long long)v[0][cs] +
                                    (long long)v[1][cs] * 256LL +
                                    (long long)v[2][cs] * 65536LL;
                                const long long u1 =
                                    (long long)v[3][cs] +
                                    (long long)v[4][cs] * 256LL +
                                    (long long)v[5][cs] * 65536LL;
                                const long long uu2 =
                                    (long long)v[6][cs] +
                                    (long long)v[7][cs] * 256LL;
                                V[pp][f][cs] = fma(
                                    l2d_exact(uu2), pow2i(8 * (6 + TC_LMIN)),
                                    fma(l2d_exact(u1),
                                        pow2i(8 * (3 + TC_LMIN)),
                                        l2d_exact(u0) * pow2i(8 * TC_LMIN)));
                            }
                        }
                        const int ec = __shfl_sync(0xffffffffu, ecl, col);
                        const int es = __shfl_sync(0xffffffffu, ecl, col + 1);
                        const double fc = pow2i(ec) * rsi;
                        const double fs = pow2i(es) * rsi;
#pragma unroll
                        for (int pp = 0; pp < 2; pp++)
                        {
                            V[pp][f][0] *= fc;
                            V[pp][f][1] *= fs;
                        }
                    }
                    // this warp is the only reader of the set's columns
                    // (for its lanes): zero them for the next item
#pragma unroll 1
                    for (int pl = 0; pl < 2 * TC_NLEV; pl++)
#pragma unroll
                        for (int f = 0; f < SHS_TC_FAMILIES; f++)
                            tc_st_zero2(lane_base +
                                        (uint32_t)(pl * TC_COLS +
                                                   2 * SHS_TC_FAMILIES * set +
                                                   2 * f));
                    if (!valid)
                        continue;
                    const double mur0 = A.mur[set];
                    const double mur1 = mur0 / A.Rref;
                    const double mur2 = mur1 / A.Rref;
                    double2 *o = A.out[set];
#pragma unroll 1
                    for (int hh = 0; hh < 2; hh++)
                    {
                        const int row = hh == 0 ? rown : rows;
                        if (row < 0 || row >= A.nlat)
                            continue;
                        // the families at this latitude: P_n(-t) =
                        // (-1)^(n - m) P_n(t) for the southern member
                        const double sg = hh == 0 ? 1.0 : -1.0;
                        const double tt = hh == 0 ? t : -t;
                        double a2[6], b2[6];
#pragma unroll
                        for (int cs = 0; cs < 2; cs++)
                        {
                            const double f0 = V[0][0][cs] + sg * V[1][0][cs];
                            const double fn = V[0][1][cs] + sg * V[1][1][cs];
                            const double fnn = V[0][2][cs] + sg * V[1][2][cs];
                            const double fe = V[0][3][cs] + sg * V[1][3][cs];
                            const double fke = V[0][4][cs] + sg * V[1][4][cs];
                            const double dp = (rho * fe - tt * fn) * ur;
                            double *q = cs == 0 ? a2 : b2;
                            q[0] = f0;                       // P
                            q[1] = fn + f0;                  // (n + 1) P
                            q[2] = dp;                       // dP
                            q[3] = fnn + 2.0 * (fn + f0);    // (n+1)(n+2) P
                            q[4] = (rho * (fke + 2.0 * fe) - tt * fnn) * ur;
                            q[5] = fma(tt * ur, dp,
                                       fma(md * md, u2 * f0, -fnn));   // ddP
                        }
                        const size_t at = (size_t)row * A.ldf + m;
                        const double w0 = cpack * mur0;
                        o[at] = make_double2(w0 * a2[0], -(w0 * b2[0]));
                        // grad1: (R/r)^(n+2), order l, r, p
                        double a1[3], b1[3];
#pragma unroll
                        for (int q = 0; q < 3; q++)
                        {
                            a1[q] = rho * a2[q];
                            b1[q] = rho * b2[q];
                        }
                        lumped_post<1, 0, 3>(a1, b1, md, ur, u2, tt * ur, 0);
                        const double w1 = cpack * mur1;
#pragma unroll
                        for (int q = 0; q < 3; q++)
                            o[(1 + q) * qs + at] =
                                make_double2(w1 * a1[q], -(w1 * b1[q]));
                        // grad2: (R/r)^(n+3), order ll lr lp rr rp pp
                        const double r2 = rho * rho;
#pragma unroll
                        for (int q = 0; q < 6; q++)
                        {
                            a2[q] *= r2;
                            b2[q] *= r2;
                        }
                        lumped_post<2, 0, 6>(a2, b2, md, ur, u2, tt * ur, 0);
                        const double w2 = cpack * mur2;
#pragma unroll
                        for (int q = 0; q < 6; q++)
                            o[(4 + q) * qs + at] =
                                make_double2(w2 * a2[q], -(w2 * b2[q]));
                    }
                }
                // the columns this warp read are zero again: release them
                tc_wait_st();
                tc_fence_before();
                mbar_arrive(bar_free);
            }
            else
            {
#pragma unroll 1
            for (int cb = 2 * half; cb < 2 * half + 2; cb++)
            {
                double tot[2][8];
#pragma unroll
                for (int pp = 0; pp < 2; pp++)
                {
                    int v[TC_NLEV][8];
#pragma unroll
                    for (int L = 0; L < TC_NLEV; L++)
                        tc_ld8(lane_base +
                                   (uint32_t)((pp * TC_NLEV + L) * TC_COLS +
                                              cb * 8),
                               v[L]);
                    tc_wait_ld();
#pragma unroll
                    for (int c = 0; c < 8; c++)
                    {
                        // levels 0..2, 3..5 and 6..7 combined exactly in
                        // 64-bit integers (|v| < 2^31: every group stays
                        // below 2^48), then two FMAs
                        const long long u0 = (long long)v[0][c] +
                                             (long long)v[1][c] * 256LL +
                                             (long long)v[2][c] * 65536LL;
                        const long long u1 = (long long)v[3][c] +
                                             (long long)v[4][c] * 256LL +
                                             (long long)v[5][c] * 65536LL;
                        const long long u2 = (long long)v[6][c] +
                                             (long long)v[7][c] * 256LL;
                        tot[pp][c] =
                            fma(l2d_exact(u2), pow2i(8 * (6 + TC_LMIN)),
                                fma(l2d_exact(u1), pow2i(8 * (3 + TC_LMIN)),
                                    l2d_exact(u0) * pow2i(8 * TC_LMIN)));
                    }
                }
                if (cb == 2 * half + 1)
                {
                    // every accumulator of this warp has been read: clear
                    // and release them before the item's outputs are written
                    clear();
                    tc_fence_before();
                    mbar_arrive(bar_free);
                }
                int ecv[4], esv[4];
#pragma unroll
                for (int kk = 0; kk < 4; kk++)
                {
                    ecv[kk] = __shfl_sync(0xffffffffu, ecl, 8 * cb + 2 * kk);
                    esv[kk] =
                        __shfl_sync(0xffffffffu, ecl, 8 * cb + 2 * kk + 1);
                }
                if (valid)
                {
#pragma unroll
                    for (int kk = 0; kk < 4; kk++)
                    {
                        const int set = cb * 4 + kk;
                        if (set >= A.nsets)
                            break;
                        const int ec = ecv[kk];
                        const int es = esv[kk];
                        const double fc = pow2i(ec) * rsi;
                        const double fs = pow2i(es) * rsi;
                        const double wgt = cpack * A.mur[set];
                        double2 *o = A.out[set];
                        if (rown >= 0 && rown < A.nlat)
                            o[(size_t)rown * A.ldf + m] = make_double2(
                                wgt * ((tot[0][2 * kk] + tot[1][2 * kk]) * fc),
                                -(wgt * ((tot[0][2 * kk + 1] +
                                          tot[1][2 * kk + 1]) *
                                         fs)));
                        if (rows >= 0 && rows < A.nlat)
                            o[(size_t)rows * A.ldf + m] = make_double2(
                                wgt * ((tot[0][2 * kk] - tot[1][2 * kk]) * fc),
                                -(wgt * ((tot[0][2 * kk + 1] -
                                          tot[1][2 * kk + 1]) *
                                         fs)));
                    }
                }
            }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
    {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     ::"r"(tmem), "r"(TC_TMEM_COLS)
                     : "memory");
    }
}

size_t shs_tc_smem_bytes()
{
    return 2 * TC_ASTAGE + TC_NB * TC_BSTAGE +
           (2 * TC_NB + 1) * TC_CH * sizeof(double) +
           (TC_NB + 6) * sizeof(uint64_t) + 4 * sizeof(uint32_t) +
           8 * sizeof(unsigned long long) + 64;
}

size_t shs_tc_chunk_bytes()
{
    return TC_BSTAGE;
}

cudaError_t launch_tc_ctab(long long nmax, int ld, const double2 *tb,
                           const double *tc, double *btp, double *ctp,
                           cudaStream_t st)
{
    k_tc_ctab<<<(unsigned)(nmax + 1), 128, 0, st>>>(nmax, ld, tb, tc, btp,
                                                    ctp);
    return cudaGetLastError();
}

cudaError_t launch_tc_seeds(const ShsTcArgs &A, bool rr, double *seed_x,
                            int2 *seed_e, cudaStream_t st)
{
    const long long n = (A.nmax + 1) * (long long)A.npairs;
    const unsigned blocks = (unsigned)((n + 255) / 256);
    if (rr)
        k_tc_seeds<true><<<blocks, 256, 0, st>>>(A, seed_x, seed_e);
    else
        k_tc_seeds<false><<<blocks, 256, 0, st>>>(A, seed_x, seed_e);
    return cudaGetLastError();
}

cudaError_t launch_tc_prep(const ShsTcPrep &P, cudaStream_t st)
{
    if (P.grad)
        k_tc_colexp_grad<<<(unsigned)(P.nmax + 1), 32 * TC_COLS, 0, st>>>(P);
    else
        k_tc_colexp<<<(unsigned)(P.nmax + 1), 512, 0, st>>>(P);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return e;
    k_tc_bdigits<<<(unsigned)(P.nmax + 1), 128, 0, st>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_shs_tc(const ShsTcArgs &A, bool rr, int grid,
                          cudaStream_t st)
{
    const size_t smem = shs_tc_smem_bytes();
    auto go = [&](auto kern) {
        cudaError_t e = cudaFuncSetAttribute(
            kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess)
            return e;
        kern<<<grid, TC_THREADS, smem, st>>>(A);
        return cudaGetLastError();
    };
    if (A.grad)
        return rr ? go(k_shs_tc<true, true>) : go(k_shs_tc<false, true>);
    return rr ? go(k_shs_tc<true, false>) : go(k_shs_tc<false, false>);
}

} // namespace cb
