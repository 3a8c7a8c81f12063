// Longitude transforms of whole grid rows in shared memory (one CTA, or a
// cluster of CTAs, per row).
//
// CHarm hands every grid row to FFTW: a c2r transform of the lumped
// coefficients in synthesis (src/shs/shs_grd_fft.c) and an r2c transform of
// the row in analysis (src/sha/sha_point.c, FFTW_FORWARD of the real row).
// Grid rows of the quadrature grids have an even length L = 2H whose half
// length H is often not smooth (GL: H = nmax + 1, e.g. 2191 = 7 * 313), so a
// library FFT falls back to slow multi-pass algorithms.  Here one CTA owns a
// row and does everything in shared memory:
//
//   * real <-> complex of half length: z_j = x_2j + i x_2j+1 and
//       X_k = (Z_k + conj Z_H-k)/2 - (i/2) e^(-i pi k/H) (Z_k - conj Z_H-k);
//   * the complex length-H DFT either directly (H = 2^a 3^b) or by
//     Bluestein's chirp-z algorithm (Bluestein 1970): with
//     w_n = exp(-i pi n^2 / H),  DFT(z)_k = w_k sum_j (z_j w_j) conj(w_k-j),
//     a circular convolution of length M >= 2H - 1, M = 2^a 3^b, evaluated
//     as FFT_M, a pointwise product with the precomputed FFT_M of the chirp,
//     and a second FFT_M (conjugated in and out, which inverts it);
//   * FFT_M by in-place Stockham autosort passes (radix 8, 4, 2 and 3 in
//     the run-time plans; 16, 16, 18 for M = 4608 and 16, 16, 9, 4 for
//     M = 9216 in the compile-time ones): every thread holds V values
//     across the barrier that separates the loads of a pass from its
//     stores, so one buffer of M values suffices.  The first pass reads its
//     inputs straight from global memory (with the chirp applied; the zero
//     half of the chirped sequence is skipped), and the last pass of the
//     first FFT applies the pointwise product as it stores.  In synthesis
//     the last pass of the second FFT writes the row itself.  Element i
//     lives at i + i/8 in shared memory, which spreads the strided stores
//     of the first pass over the banks;
//   * rows of length 4L whose spectra stop below L (DH2 synthesis): two
//     complex DFTs of length L per row, each computing every other pair of
//     the row (k_rfft_inv4, two CTAs per row);
//   * rows of odd length L (custom grids, synthesis only): one complex DFT
//     of length L by Bluestein, the row being its real part
//     (k_rfft_inv_odd);
//   * transform lengths beyond one CTA's shared memory (M > 9216, e.g. the
//     21602-point rows of the nmax 10800 GL grid, M = 24576): a cluster of
//     C = 2..16 CTAs per row, each holding M / C values, with a radix-C
//     step across the CTAs on either side of the per-CTA FFTs, read
//     through distributed shared memory (k_rfftc_fwd / k_rfftc_inv).
//
// Both directions are unnormalised, as FFTW's and CHarm's: the synthesis
// output is sum_k X_k e^(+2 pi i k n / L) over the Hermitian spectrum, and
// the analysis output is X_k = sum_n x_n e^(-2 pi i k n / L), k <= kmax.
#include <cstdint>
#include <type_traits>

#include <cooperative_groups.h>

#include "common.cuh"
#include "kernels.h"

namespace cb
{

namespace
{

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}

__device__ __forceinline__ double2 conj2(double2 a)
{
    return make_double2(a.x, -a.y);
}

__device__ __forceinline__ double2 add2(double2 a, double2 b)
{
    return make_double2(a.x + b.x, a.y + b.y);
}

__device__ __forceinline__ double2 sub2(double2 a, double2 b)
{
    return make_double2(a.x - b.x, a.y - b.y);
}

// -i a
__device__ __forceinline__ double2 mul_mi(double2 a)
{
    return make_double2(a.y, -a.x);
}

// shared-memory position of element i
__device__ __forceinline__ int pidx(int i)
{
    return i + (i >> 3);
}

constexpr double RSQRT2 = 0.70710678118654752440;
constexpr double SQRT3_2 = 0.86602540378443864676;

// In-register forward DFTs, X_k = sum_r v_r exp(-2 pi i r k / R).
__device__ __forceinline__ void dft2(double2 *v)
{
    double2 a = v[0], b = v[1];
    v[0] = add2(a, b);
    v[1] = sub2(a, b);
}

__device__ __forceinline__ void dft4(double2 &a0, double2 &a1, double2 &a2,
                                     double2 &a3)
{
    double2 t0 = add2(a0, a2), t1 = sub2(a0, a2);
    double2 t2 = add2(a1, a3), t3 = mul_mi(sub2(a1, a3));
    a0 = add2(t0, t2);
    a2 = sub2(t0, t2);
    a1 = add2(t1, t3);
    a3 = sub2(t1, t3);
}

__device__ __forceinline__ void dft8(double2 *v)
{
    // even / odd halves, then one radix-2 step with W8^k
    double2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    double2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4(e0, e1, e2, e3);
    dft4(o0, o1, o2, o3);
    double2 w1 = make_double2((o1.x + o1.y) * RSQRT2, (o1.y - o1.x) * RSQRT2);
    double2 w2 = mul_mi(o2);
    double2 w3 = make_double2((o3.y - o3.x) * RSQRT2, -(o3.x + o3.y) * RSQRT2);
    v[0] = add2(e0, o0);
    v[4] = sub2(e0, o0);
    v[1] = add2(e1, w1);
    v[5] = sub2(e1, w1);
    v[2] = add2(e2, w2);
    v[6] = sub2(e2, w2);
    v[3] = add2(e3, w3);
    v[7] = sub2(e3, w3);
}

__device__ __forceinline__ void dft3(double2 *v)
{
    double2 t = add2(v[1], v[2]);
    double2 d = sub2(v[1], v[2]);
    double2 h = make_double2(fma(-0.5, t.x, v[0].x), fma(-0.5, t.y, v[0].y));
    double2 q = mul_mi(make_double2(SQRT3_2 * d.x, SQRT3_2 * d.y));
    v[0] = add2(v[0], t);
    v[1] = add2(h, q);
    v[2] = sub2(h, q);
}

// cos and sin of pi/8, 2 pi/9, 4 pi/9, 8 pi/9
constexpr double C16 = 0.92387953251128675613;
constexpr double S16 = 0.38268343236508977173;
constexpr double C9A = 0.76604444311897803520;
constexpr double S9A = 0.64278760968653932632;
constexpr double C9B = 0.17364817766693034885;
constexpr double S9B = 0.98480775301220805936;
constexpr double C9D = -0.93969262078590838405;
constexpr double S9D = 0.34202014332566873304;

// 16 = 4 x 4 (n = 4 n1 + n2, k = k1 + 4 k2): DFTs of length 4 over n1,
// twiddles exp(-2 pi i n2 k1 / 16), DFTs of length 4 over n2.  HZ: the
// inputs v[8..15] are zero and are not read (the zero-padded half of a
// Bluestein sequence).
template <bool HZ>
__device__ __forceinline__ void dft16(double2 *v)
{
    double2 a[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++)
    {
        if constexpr (HZ)
        {
            const double2 x0 = v[n2], x1 = v[4 + n2];
            a[n2][0] = add2(x0, x1);
            a[n2][1] = add2(x0, mul_mi(x1));
            a[n2][2] = sub2(x0, x1);
            a[n2][3] = sub2(x0, mul_mi(x1));
        }
        else
        {
            a[n2][0] = v[n2];
            a[n2][1] = v[4 + n2];
            a[n2][2] = v[8 + n2];
            a[n2][3] = v[12 + n2];
            dft4(a[n2][0], a[n2][1], a[n2][2], a[n2][3]);
        }
    }
    a[1][1] = cmul(a[1][1], make_double2(C16, -S16));
    a[1][2] = make_double2((a[1][2].x + a[1][2].y) * RSQRT2,
                           (a[1][2].y - a[1][2].x) * RSQRT2);
    a[1][3] = cmul(a[1][3], make_double2(S16, -C16));
    a[2][1] = make_double2((a[2][1].x + a[2][1].y) * RSQRT2,
                           (a[2][1].y - a[2][1].x) * RSQRT2);
    a[2][2] = mul_mi(a[2][2]);
    a[2][3] = make_double2((a[2][3].y - a[2][3].x) * RSQRT2,
                           -(a[2][3].x + a[2][3].y) * RSQRT2);
    a[3][1] = cmul(a[3][1], make_double2(S16, -C16));
    a[3][2] = make_double2((a[3][2].y - a[3][2].x) * RSQRT2,
                           -(a[3][2].x + a[3][2].y) * RSQRT2);
    a[3][3] = cmul(a[3][3], make_double2(-C16, S16));
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++)
    {
        dft4(a[0][k1], a[1][k1], a[2][k1], a[3][k1]);
        v[k1] = a[0][k1];
        v[k1 + 4] = a[1][k1];
        v[k1 + 8] = a[2][k1];
        v[k1 + 12] = a[3][k1];
    }
}

// 9 = 3 x 3 (n = 3 n1 + n2, k = k1 + 3 k2), twiddles exp(-2 pi i n2 k1 / 9)
__device__ __forceinline__ void dft9(double2 *v)
{
    double2 a[3][3];
#pragma unroll
    for (int n2 = 0; n2 < 3; n2++)
    {
        a[n2][0] = v[n2];
        a[n2][1] = v[3 + n2];
        a[n2][2] = v[6 + n2];
        dft3(a[n2]);
    }
    a[1][1] = cmul(a[1][1], make_double2(C9A, -S9A));
    a[1][2] = cmul(a[1][2], make_double2(C9B, -S9B));
    a[2][1] = cmul(a[2][1], make_double2(C9B, -S9B));
    a[2][2] = cmul(a[2][2], make_double2(C9D, -S9D));
#pragma unroll
    for (int k1 = 0; k1 < 3; k1++)
    {
        double2 b[3] = {a[0][k1], a[1][k1], a[2][k1]};
        dft3(b);
        v[k1] = b[0];
        v[k1 + 3] = b[1];
        v[k1 + 6] = b[2];
    }
}

// 18 = 2 x 9 by the prime-factor (Good-Thomas) map, no twiddles: input
// n = (9 n1 + 2 n2) mod 18, output k = (9 k1 + 10 k2) mod 18
__device__ __forceinline__ void dft18(double2 *v)
{
    double2 e[9], o[9];
#pragma unroll
    for (int n2 = 0; n2 < 9; n2++)
    {
        e[n2] = v[(2 * n2) % 18];
        o[n2] = v[(9 + 2 * n2) % 18];
    }
    dft9(e);
    dft9(o);
#pragma unroll
    for (int k2 = 0; k2 < 9; k2++)
    {
        v[(10 * k2) % 18] = add2(e[k2], o[k2]);
        v[(9 + 10 * k2) % 18] = sub2(e[k2], o[k2]);
    }
}

template <int R, bool HZ = false>
__device__ __forceinline__ void dft(double2 *v)
{
    if constexpr (R == 2)
        dft2(v);
    else if constexpr (R == 3)
        dft3(v);
    else if constexpr (R == 4)
        dft4(v[0], v[1], v[2], v[3]);
    else if constexpr (R == 8)
        dft8(v);
    else if constexpr (R == 9)
        dft9(v);
    else if constexpr (R == 16)
        dft16<HZ>(v);
    else
    {
        static_assert(R == 18, "radix");
        dft18(v);
    }
}

// w[r] = w[1]^r for r = 2..R-1: w[2^a] = w[2^(a-1)]^2 and
// w[2^a + b] = w[2^a] w[b] (b < 2^a), at most log2 R + 1 products deep
constexpr int hibit(int r)
{
    int h = 1;
    while (2 * h <= r)
        h *= 2;
    return h;
}

template <int R>
__device__ __forceinline__ void twiddle_powers(double2 *w)
{
#pragma unroll
    for (int r = 2; r < R; r++)
    {
        if (r == hibit(r))
            w[r] = cmul(w[r / 2], w[r / 2]);
        else
            w[r] = cmul(w[hibit(r)], w[r - hibit(r)]);
    }
}

// Input of the first pass: element i of the sequence to transform.
struct SrcSmem
{
    const double2 *s;
    __device__ __forceinline__ double2 operator()(int i) const
    {
        return s[pidx(i)];
    }
};

// j div Ns and j mod Ns (one division by the run-time stride)
__device__ __forceinline__ void divmod_ns(int j, int Ns, int &q, int &k)
{
    k = j % Ns;
    q = (j - k) / Ns;
}

// One Stockham pass of radix R over s[0..M): butterfly j reads element
// j + r M/R (twiddled by exp(-2 pi i (j mod Ns) r / (Ns R))) and writes its
// R outputs to elements (j - j mod Ns) R + j mod Ns + r Ns.  The first pass
// (Ns = 1, no twiddles) reads through `src`; a non-null `bh` multiplies the
// stored outputs by bh and conjugates them.  Plans have 64 | M and start
// with two radix-8 passes, so M/R and every Ns > 1 are multiples of 8: the
// padded positions of a butterfly's elements are then a base plus a
// constant stride (r (M/R + M/8R) for loads, r (Ns + Ns/8) for stores, and
// r for the first pass's stores, whose bases are multiples of 8).
template <int R, int V, class Src>
__device__ __forceinline__ void stockham_pass(double2 *s,
                                              const double2 *__restrict__ tw,
                                              int M, int Ns, int tid, int T,
                                              bool first, const Src &src,
                                              const double2 *__restrict__ bh)
{
    constexpr int BPT = (V + R - 1) / R;
    const int nb = M / R;
    const int step = M / (Ns * R);
    const int ld_stride = nb + (nb >> 3);
    const int st_stride = (Ns == 1) ? 1 : Ns + (Ns >> 3);
    double2 v[BPT][R];
    if (first)
    {
#pragma unroll
        for (int c = 0; c < BPT; c++)
        {
            const int j = tid + c * T;
            if (j < nb)
            {
#pragma unroll
                for (int r = 0; r < R; r++)
                    v[c][r] = src(j + r * nb);
                dft<R>(v[c]);
            }
        }
    }
    else
    {
#pragma unroll
        for (int c = 0; c < BPT; c++)
        {
            const int j = tid + c * T;
            if (j < nb)
            {
                int q, k;
                divmod_ns(j, Ns, q, k);
                // one table twiddle per butterfly, its powers by products
                double2 wp[R];
                wp[1] = __ldg(&tw[k * step]);
                twiddle_powers<R>(wp);
                const int b = pidx(j);
                v[c][0] = s[b];
#pragma unroll
                for (int r = 1; r < R; r++)
                    v[c][r] = cmul(s[b + r * ld_stride], wp[r]);
                dft<R>(v[c]);
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < BPT; c++)
    {
        const int j = tid + c * T;
        if (j < nb)
        {
            int q, k;
            divmod_ns(j, Ns, q, k);
            const int d = q * Ns * R + k;
            const int b = pidx(d);
            if (bh)
            {
#pragma unroll
                for (int r = 0; r < R; r++)
                    s[b + r * st_stride] =
                        conj2(cmul(v[c][r], __ldg(&bh[d + r * Ns])));
            }
            else
            {
#pragma unroll
                for (int r = 0; r < R; r++)
                    s[b + r * st_stride] = v[c][r];
            }
        }
    }
    __syncthreads();
}

// Forward FFT of length M = 8^n8 4^n4 2^n2 3^n3 (passes in that order) of
// the sequence src(0..M), result in s (natural order).  One loop per radix
// keeps every pass's registers separate.
template <int V, class Src>
__device__ __forceinline__ void fft_m(double2 *s,
                                      const double2 *__restrict__ tw, int M,
                                      int4 np, int tid, int T, const Src &src,
                                      const double2 *__restrict__ bh_last)
{
    const int last = np.x + np.y + np.z + np.w - 1;
    int Ns = 1, p = 0;
    for (int i = 0; i < np.x; i++, p++, Ns *= 8)
        stockham_pass<8, V>(s, tw, M, Ns, tid, T, p == 0, src,
                            p == last ? bh_last : nullptr);
    for (int i = 0; i < np.y; i++, p++, Ns *= 4)
        stockham_pass<4, V>(s, tw, M, Ns, tid, T, p == 0, src,
                            p == last ? bh_last : nullptr);
    for (int i = 0; i < np.z; i++, p++, Ns *= 2)
        stockham_pass<2, V>(s, tw, M, Ns, tid, T, p == 0, src,
                            p == last ? bh_last : nullptr);
    for (int i = 0; i < np.w; i++, p++, Ns *= 3)
        stockham_pass<3, V>(s, tw, M, Ns, tid, T, p == 0, src,
                            p == last ? bh_last : nullptr);
}

// ---- the same transform with the whole plan known at compile time ----
// (the lengths the grids of nmax about 2160..2190 use: M = 4608, 9216).
// Radices, strides, thread counts and butterfly ranges become constants,
// so the index arithmetic of every pass folds away, and the larger
// radices cut the number of barrier-separated passes through shared
// memory: 4608 = 16 16 18 (three passes instead of five),
// 9216 = 16 16 9 4 (four instead of six).  The first pass has radix 16
// and every later stride is a multiple of 8, as the padded addressing
// needs.
// Compile-time plans: the radices of FFT_M pass by pass (the grids' common
// Bluestein lengths: GL rows of nmax 360, 540, 900, 1260, 1620, 1980, 2190
// and their neighbours, DH2 rows of nmax 2190, the nmax 10800 clusters).  The first is 16
// (the zero half of a chirped sequence is skipped there), the last even
// (the half-output passes), and every pass keeps M / R and the stride a
// multiple of 8 (the padded layout).
constexpr int ct_npass(int M)
{
    return (M == 9216 || M == 6144 || M == 3072 || M == 3456) ? 4 : 3;
}

constexpr int ct_radix(int M, int p)
{
    if (M == 4608)
        return p < 2 ? 16 : 18;
    if (M == 6144)   // the per-CTA length of the nmax 10800 cluster plan
        return p < 2 ? 16 : (p == 2 ? 8 : 3);
    if (M == 768)
        return p == 1 ? 3 : 16;
    if (M == 3072)
        return p == 1 ? 3 : (p == 2 ? 4 : 16);
    if (M == 3456)
        return p == 0 ? 16 : (p == 1 ? 3 : (p == 2 ? 9 : 8));
    if (M == 1152)
        return p == 0 ? 16 : (p == 1 ? 4 : 18);
    if (M == 2048)
        return p < 2 ? 16 : 8;
    if (M == 4096)
        return 16;
    return p < 2 ? 16 : (p == 2 ? 9 : 4);   // 9216
}

constexpr int ct_ns(int M, int p)
{
    int ns = 1;
    for (int i = 0; i < p; i++)
        ns *= ct_radix(M, i);
    return ns;
}

// read-only load that stays after the barrier before it (a volatile asm is
// not moved across the barrier's), so the twiddles of later passes are
// not hoisted into registers ahead of time
__device__ __forceinline__ double2 ld_tw(const double2 *p)
{
    double2 v;
    asm volatile("ld.global.nc.v2.f64 {%0, %1}, [%2];"
                 : "=d"(v.x), "=d"(v.y)
                 : "l"(p));
    return v;
}

// HZ (first pass of a Bluestein sequence only): elements M/2.. are zero
// (M >= 2H), so a butterfly's upper R/2 inputs are neither read nor added.
// HO (last pass of Bluestein's second FFT only): outputs M/2.. are never
// read (H <= M/2), so they are neither computed nor stored.
template <int R, int V, int M, int NS, bool FIRST, bool BH, bool HZ,
          bool HO = false, class Src>
__device__ __forceinline__ void stockham_ct(double2 *s,
                                            const double2 *__restrict__ tw,
                                            int tid, const Src &src,
                                            const double2 *__restrict__ bh)
{
    constexpr int T = M / V;
    constexpr int BPT = (V + R - 1) / R;
    constexpr int nb = M / R;
    constexpr int step = M / (NS * R);
    constexpr int ld_stride = nb + (nb >> 3);
    static_assert(nb % 8 == 0 && (NS == 1 || NS % 8 == 0), "padding");
    static_assert(!FIRST || R % 8 == 0, "first pass radix");
    static_assert(!HZ || (FIRST && R == 16), "zero half");
    static_assert(!HO || (NS * R == M && R % 2 == 0 && !BH), "half output");
    // padded offset of a butterfly's output r from its first one: the
    // first pass writes R consecutive elements from a multiple of 8
    auto st_off = [](int r) {
        return NS == 1 ? r + (r >> 3) : r * (NS + (NS >> 3));
    };
    double2 v[BPT][R];
#pragma unroll
    for (int c = 0; c < BPT; c++)
    {
        const int j = tid + c * T;
        if (j < nb)
        {
            if constexpr (FIRST)
            {
#pragma unroll
                for (int r = 0; r < (HZ ? R / 2 : R); r++)
                    v[c][r] = src(j + r * nb);
            }
            else
            {
                const int k = j % NS;
                double2 wp[R];
                wp[1] = ld_tw(&tw[k * step]);
                twiddle_powers<R>(wp);
                const int b = pidx(j);
                v[c][0] = s[b];
#pragma unroll
                for (int r = 1; r < R; r++)
                    v[c][r] = cmul(s[b + r * ld_stride], wp[r]);
            }
            dft<R, HZ>(v[c]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < BPT; c++)
    {
        const int j = tid + c * T;
        if (j < nb)
        {
            const int k = j % NS;
            const int d = (j / NS) * NS * R + k;
            const int b = pidx(d);
            if constexpr (BH)
            {
#pragma unroll
                for (int r = 0; r < R; r++)
                    s[b + st_off(r)] =
                        conj2(cmul(v[c][r], ld_tw(&bh[d + r * NS])));
            }
            else
            {
#pragma unroll
                for (int r = 0; r < (HO ? R / 2 : R); r++)
                    s[b + st_off(r)] = v[c][r];
            }
        }
    }
    __syncthreads();
}

// passes P..PEND-1 of FFT_M (compile-time plan); the FFT's last pass
// multiplies by bh when given; HZ: the upper half of the input sequence
// is zero; HO: only the lower half of the output is wanted
template <int V, int M, int P, bool HZ, int PEND = ct_npass(M),
          bool HO = false, class Src>
__device__ __forceinline__ void fft_ct(double2 *s,
                                       const double2 *__restrict__ tw, int tid,
                                       const Src &src,
                                       const double2 *__restrict__ bh_last)
{
    if constexpr (P < PEND)
    {
        constexpr int R = ct_radix(M, P);
        constexpr int NS = ct_ns(M, P);
        constexpr bool Z = HZ && P == 0;
        if constexpr (P == ct_npass(M) - 1)
        {
            if (bh_last)
                stockham_ct<R, V, M, NS, P == 0, true, Z>(s, tw, tid, src,
                                                          bh_last);
            else
                stockham_ct<R, V, M, NS, P == 0, false, Z, HO>(
                    s, tw, tid, src, nullptr);
        }
        else
            stockham_ct<R, V, M, NS, P == 0, false, Z>(s, tw, tid, src,
                                                       nullptr);
        fft_ct<V, M, P + 1, HZ, PEND, HO>(s, tw, tid, src, bh_last);
    }
}

// The last pass of the second FFT_M of Bluestein's algorithm (compile-time
// plan, even last radix) handed straight to its consumer: output
// k = j + r M/R of butterfly j goes to out(k, value) for k < H <= M/2.
// Nothing is stored in shared memory, so the pass needs no barrier.
template <int V, int M, class Out>
__device__ __forceinline__ void fft_ct_last_out(const double2 *s,
                                                const double2 *__restrict__ tw,
                                                int tid, int H, const Out &out)
{
    constexpr int P = ct_npass(M) - 1;
    constexpr int R = ct_radix(M, P);
    constexpr int NS = ct_ns(M, P);
    static_assert(NS * R == M && R % 2 == 0, "last pass");
    constexpr int T = M / V;
    constexpr int BPT = (V + R - 1) / R;
    constexpr int ld_stride = NS + (NS >> 3);
#pragma unroll 1
    for (int c = 0; c < BPT; c++)
    {
        const int j = tid + c * T;
        if (j < NS)
        {
            double2 wp[R], v[R];
            wp[1] = ld_tw(&tw[j]);
            twiddle_powers<R>(wp);
            const int b = pidx(j);
            v[0] = s[b];
#pragma unroll
            for (int r = 1; r < R; r++)
                v[r] = cmul(s[b + r * ld_stride], wp[r]);
            dft<R>(v);
            // H <= M/2: the outputs of the upper half are never used
#pragma unroll
            for (int r = 0; r < R / 2; r++)
                if (j + r * NS < H)
                    out(j + r * NS, v[r]);
        }
    }
}

// Complex DFT of length H of the sequence z(0..H), zero-padded to M when
// Bluestein is used; `pre` returns z_j already multiplied by the chirp
// (Bluestein) and 0 for j >= H.  On return the DFT value k is dft_h_out(k).
template <int V, int MC, class Pre>
__device__ __forceinline__ void dft_h(double2 *s, const RfftArgs &A, int tid,
                                      int T, const Pre &pre)
{
    if constexpr (MC > 0)
    {
        // plan fixed at compile time (A.M == MC, Bluestein)
        fft_ct<V, MC, 0, true>(s, A.tw, tid, pre, A.bh);
        fft_ct<V, MC, 0, false, ct_npass(MC), true>(s, A.tw, tid, SrcSmem{s},
                                                    nullptr);
    }
    else
    {
        if (A.direct)
        {
            fft_m<V>(s, A.tw, A.M, A.npass, tid, T, pre, nullptr);
            return;
        }
        fft_m<V>(s, A.tw, A.M, A.npass, tid, T, pre, A.bh);
        fft_m<V>(s, A.tw, A.M, A.npass, tid, T, SrcSmem{s}, nullptr);
    }
}

// value k (< H) of the length-H DFT after dft_h
__device__ __forceinline__ double2 dft_h_out(const double2 *s,
                                             const RfftArgs &A, int k)
{
    if (A.direct)
        return s[pidx(k)];
    return cmul(__ldg(&A.w[k]), conj2(s[pidx(k)]));
}

// Analysis input: z_j = x_2j + i x_2j+1 times the chirp.
struct SrcRow
{
    const double2 *x2;
    const double2 *w;
    int H;
    __device__ __forceinline__ double2 operator()(int i) const
    {
        if (i >= H)
            return make_double2(0.0, 0.0);
        double2 z = x2[i];
        return w ? cmul(z, __ldg(&w[i])) : z;
    }
};

// Analysis input from float rows (the single-precision mode)
struct SrcRowF
{
    const float2 *x2;
    const double2 *w;
    int H;
    __device__ __forceinline__ double2 operator()(int i) const
    {
        if (i >= H)
            return make_double2(0.0, 0.0);
        const float2 f = x2[i];
        double2 z = make_double2((double)f.x, (double)f.y);
        return w ? cmul(z, __ldg(&w[i])) : z;
    }
};

// Synthesis input: conj Z_k times the chirp, with
// Z_k = (X_k + conj X_H-k) + i e^(i pi k/H) (X_k - conj X_H-k) and X_k = 0
// above kmax (the inverse DFT is conj(DFT(conj Z))).
struct SrcSpectrum
{
    const double2 *X;
    const double2 *w;
    const double2 *ht;
    int H, kmax;
    __device__ __forceinline__ double2 operator()(int k) const
    {
        if (k >= H)
            return make_double2(0.0, 0.0);
        const int kh = H - k;
        double2 xk = k <= kmax ? X[k] : make_double2(0.0, 0.0);
        double2 xh = kh <= kmax ? conj2(X[kh]) : make_double2(0.0, 0.0);
        double2 e = cmul(conj2(__ldg(&ht[k])), sub2(xk, xh));
        double2 zc = make_double2(xk.x + xh.x - e.y, -(xk.y + xh.y + e.x));
        return w ? cmul(zc, __ldg(&w[k])) : zc;
    }
};

// Synthesis input of the quarter-length transform.  A row of length 4H
// whose spectrum X stops below H gives, with a = X_k, b = conj X_H-k and
// o = exp(2 pi i k / 4H),
//   V_0[k] = (a + b) + i o (a - i b),
//   V_1[k] = o^2 (a - b) + i o^3 (a + i b),
// and the inverse DFT of length H of V_rho holds the pairs
// (x_4q+2rho, x_4q+2rho+1) of the row (the four residues of the row index
// mod 4, paired into two complex sequences).  Returns conj V_rho[k] times
// the chirp, as SrcSpectrum.
struct SrcQuarter
{
    const double2 *X;
    const double2 *w;
    const double2 *w4;
    int H, kmax, rho;
    __device__ __forceinline__ double2 operator()(int k) const
    {
        if (k >= H)
            return make_double2(0.0, 0.0);
        const int kh = H - k;
        const double2 a = k <= kmax ? X[k] : make_double2(0.0, 0.0);
        const double2 b =
            (k >= 1 && kh <= kmax) ? conj2(X[kh]) : make_double2(0.0, 0.0);
        const double2 o = __ldg(&w4[k]);
        double2 v;
        if (rho == 0)
        {
            const double2 t = cmul(o, add2(a, mul_mi(b)));
            v = make_double2(a.x + b.x - t.y, a.y + b.y + t.x);
        }
        else
        {
            const double2 o2 = cmul(o, o);
            const double2 o3 = cmul(o2, o);
            const double2 u = cmul(o2, sub2(a, b));
            const double2 t = cmul(o3, sub2(a, mul_mi(b)));
            v = make_double2(u.x - t.y, u.y + t.x);
        }
        return cmul(conj2(v), __ldg(&w[k]));
    }
};

// Bluestein kernel b_n = conj w_|n| on the circle of length M
struct SrcKernel
{
    const double2 *w;
    int H, M;
    __device__ __forceinline__ double2 operator()(int n) const
    {
        if (n < H)
            return conj2(w[n]);
        if (n > M - H)
            return conj2(w[M - n]);
        return make_double2(0.0, 0.0);
    }
};

// Synthesis input of a row of odd length L: the Hermitian extension Y of
// the spectrum (Y_k = X_k for k <= (L - 1)/2, conj X_L-k above, zero above
// kmax, the imaginary part of X_0 ignored), conjugated and chirped; the row
// is the real part of the inverse DFT of length H = L.
struct SrcSpectrumOdd
{
    const double2 *X;
    const double2 *w;
    int H, kmax;
    __device__ __forceinline__ double2 operator()(int k) const
    {
        if (k >= H)
            return make_double2(0.0, 0.0);
        double2 y = make_double2(0.0, 0.0);
        if (2 * k < H)
        {
            if (k <= kmax)
                y = X[k];
            if (k == 0)
                y.y = 0.0;
        }
        else if (H - k <= kmax)
            y = conj2(X[H - k]);
        return cmul(conj2(y), __ldg(&w[k]));
    }
};

// ---- transforms longer than one CTA's shared memory ----
// A cluster of C CTAs owns a row; CTA q holds Mc = M / C values.  FFT_M of
// a sequence a is computed as
//   y_q[i] = w_M^(i q) sum_k a[i + k Mc] w_C^(k q)    (radix-C decimation
//            in frequency across the CTAs, folded into the loads of the
//            first local pass), then FFT_Mc(y_q)[l] = FFT_M(a)[C l + q],
// so every CTA holds one residue class of the spectrum, in which the
// pointwise product of Bluestein's algorithm needs no exchange.  The second
// FFT_M takes its input by residue classes (decimation in time): each CTA
// transforms its class, U_q = FFT_Mc, and
//   v_t = sum_q w_M^(q t) U_q[t mod Mc]
// is gathered through distributed shared memory for the outputs t a CTA
// writes.

// Input of the first local pass of CTA q: a = src(0..M) vanishes from nz
// on, so blocks k with k Mc >= nz are not read.
template <class Src>
struct SrcClusterDif
{
    Src src;
    const double2 *twM;
    int q, C, Mc, M, nz;
    __device__ __forceinline__ double2 operator()(int i) const
    {
        // i < Mc and q < C, C a power of two: k q mod C is a mask and
        // i q < Mc C = M needs no reduction
        double2 acc = src(i);
        for (int k = 1; k < C && k * Mc < nz; k++)
        {
            const int kq = (k * q) & (C - 1);
            acc = add2(acc, cmul(src(i + k * Mc), __ldg(&twM[kq * Mc])));
        }
        if (q == 0)
            return acc;
        return cmul(acc, __ldg(&twM[i * q]));
    }
};

// v_t of the second FFT_M (t < M) from the residue transforms U_q held in
// the shared memory of the cluster's CTAs.
__device__ __forceinline__ double2 cluster_v(
    const cooperative_groups::cluster_group &cl, double2 *s,
    const double2 *__restrict__ twM, int C, int Mc, int M, int t)
{
    const int pj = pidx(t % Mc);
    double2 acc = *cl.map_shared_rank(s + pj, 0);
    // e = qq t mod M by repeated addition (t < M)
    int e = 0;
    for (int qq = 1; qq < C; qq++)
    {
        e += t;
        if (e >= M)
            e -= M;
        const double2 u = *cl.map_shared_rank(s + pj, qq);
        acc = add2(acc, cmul(u, __ldg(&twM[e])));
    }
    return acc;
}

} // namespace

// Register cap NR: M / 16 <= 576 threads of 96 registers with V = 16 values
// per thread (five warps on one scheduler's 16384 registers; two CTAs of
// 288 threads per SM up to M = 4608).
#define RFFT_BOUNDS(NR) __maxnreg__(NR)

// Analysis direction: real rows x[row][0..L) -> X[row][0..kmax]; one CTA
// per row (a loop over rows would let the compiler hoist every pass's
// twiddles out of it and run out of registers).
template <int V, int NR, bool F32, int MC>
__global__ void RFFT_BOUNDS(NR) k_rfft_fwd(RfftArgs A)
{
    extern __shared__ __align__(16) double2 s[];
    const int tid = threadIdx.x, T = blockDim.x;
    const int H = A.H;
    const long long row = blockIdx.x;
    if constexpr (F32)
    {
        const float *xf = reinterpret_cast<const float *>(A.x);
        SrcRowF src{reinterpret_cast<const float2 *>(xf + row * A.ldx),
                    A.direct ? nullptr : A.w, H};
        dft_h<V, MC>(s, A, tid, T, src);
    }
    else
    {
        SrcRow src{reinterpret_cast<const double2 *>(A.x + row * A.ldx),
                   A.direct ? nullptr : A.w, H};
        dft_h<V, MC>(s, A, tid, T, src);
    }
    double2 *X = A.X + row * A.ldX;
    for (int k = tid; k <= A.kmax; k += T)
    {
        const int ka = (k == H) ? 0 : k;
        const int kb = (k == 0) ? 0 : H - k;
        double2 zk = dft_h_out(s, A, ka);
        double2 zh = conj2(dft_h_out(s, A, kb));
        double2 e = cmul(__ldg(&A.ht[k]), sub2(zk, zh));
        double2 sm = add2(zk, zh);
        X[k] = make_double2(0.5 * (sm.x + e.y), 0.5 * (sm.y - e.x));
    }
}

// Synthesis direction: X[row][0..kmax] (zero above) -> real rows x[row].
// Output of the synthesis direction: x_2k + i x_2k+1 = conj of DFT value
// k, which Bluestein's algorithm gives as w_k conj(second FFT output k).
template <bool F32>
struct OutRow
{
    void *x2;
    const double2 *w;
    __device__ __forceinline__ void operator()(int k, double2 v) const
    {
        const double2 z = cmul(__ldg(&w[k]), conj2(v));
        if constexpr (F32)
            reinterpret_cast<float2 *>(x2)[k] =
                make_float2((float)z.x, (float)-z.y);
        else
            reinterpret_cast<double2 *>(x2)[k] = conj2(z);
    }
};

template <int V, int NR, bool F32, int MC>
__global__ void RFFT_BOUNDS(NR) k_rfft_inv(RfftArgs A)
{
    extern __shared__ __align__(16) double2 s[];
    const int tid = threadIdx.x, T = blockDim.x;
    const long long row = blockIdx.x;
    SrcSpectrum src{A.X + row * A.ldX, A.direct ? nullptr : A.w, A.ht, A.H,
                    A.kmax};
    if constexpr (MC > 0)
    {
        // Bluestein with the second FFT's last pass writing the row
        void *x2 = F32 ? (void *)(reinterpret_cast<float *>(A.x) +
                                  row * A.ldx)
                       : (void *)(A.x + row * A.ldx);
        fft_ct<V, MC, 0, true>(s, A.tw, tid, src, A.bh);
        fft_ct<V, MC, 0, false, ct_npass(MC) - 1>(s, A.tw, tid, SrcSmem{s},
                                                  nullptr);
        fft_ct_last_out<V, MC>(s, A.tw, tid, A.H, OutRow<F32>{x2, A.w});
        return;
    }
    dft_h<V, MC>(s, A, tid, T, src);
    if constexpr (F32)
    {
        float *xf = reinterpret_cast<float *>(A.x);
        float2 *x2 = reinterpret_cast<float2 *>(xf + row * A.ldx);
        for (int j = tid; j < A.H; j += T)
        {
            const double2 z = conj2(dft_h_out(s, A, j));
            x2[j] = make_float2((float)z.x, (float)z.y);
        }
    }
    else
    {
        double2 *x2 = reinterpret_cast<double2 *>(A.x + row * A.ldx);
        for (int j = tid; j < A.H; j += T)
            x2[j] = conj2(dft_h_out(s, A, j));
    }
}

// Output of the quarter-length transform: the pair q of half rho of a row
// is the conjugate of DFT value q (w_q conj of the second FFT's output q).
struct OutRowQ
{
    double2 *x2;
    const double2 *w;
    int rho;
    __device__ __forceinline__ void operator()(int q, double2 v) const
    {
        x2[2 * q + rho] = conj2(cmul(__ldg(&w[q]), conj2(v)));
    }
};

// Synthesis of rows of length 4H with spectra below H: CTA 2 row + rho
// computes half rho of the row (SrcQuarter), Bluestein with the plan fixed
// at compile time.
template <int V, int NR, int MC>
__global__ void RFFT_BOUNDS(NR) k_rfft_inv4(RfftArgs A)
{
    extern __shared__ __align__(16) double2 s[];
    const int tid = threadIdx.x;
    const long long row = blockIdx.x >> 1;
    const int rho = (int)(blockIdx.x & 1);
    SrcQuarter src{A.X + row * A.ldX, A.w, A.w4, A.H, A.kmax, rho};
    fft_ct<V, MC, 0, true>(s, A.tw, tid, src, A.bh);
    fft_ct<V, MC, 0, false, ct_npass(MC) - 1>(s, A.tw, tid, SrcSmem{s},
                                              nullptr);
    fft_ct_last_out<V, MC>(
        s, A.tw, tid, A.H,
        OutRowQ{reinterpret_cast<double2 *>(A.x + row * A.ldx), A.w, rho});
}

// Synthesis of rows of odd length L = H: Bluestein over the whole row
// (run-time plan), the row being the real part of the inverse DFT.
template <int V, int NR>
__global__ void RFFT_BOUNDS(NR) k_rfft_inv_odd(RfftArgs A)
{
    extern __shared__ __align__(16) double2 s[];
    const int tid = threadIdx.x, T = blockDim.x;
    const long long row = blockIdx.x;
    SrcSpectrumOdd src{A.X + row * A.ldX, A.w, A.H, A.kmax};
    dft_h<V, 0>(s, A, tid, T, src);
    double *x = A.x + row * A.ldx;
    for (int j = tid; j < A.H; j += T)
        x[j] = dft_h_out(s, A, j).x;
}

// Analysis direction of a cluster plan (A.C CTAs per row, double rows).
template <int V, int NR, int MC = 0>
__global__ void RFFT_BOUNDS(NR) k_rfftc_fwd(RfftArgs A)
{
    namespace cg = cooperative_groups;
    extern __shared__ __align__(16) double2 s[];
    cg::cluster_group cl = cg::this_cluster();
    const int tid = threadIdx.x, T = blockDim.x;
    const int C = A.C, q = (int)cl.block_rank(), H = A.H;
    const int Mc = A.M / C;
    const long long row = blockIdx.x / C;
    SrcRow src{reinterpret_cast<const double2 *>(A.x + row * A.ldx), A.w, H};
    SrcClusterDif<SrcRow> dif{src, A.twM, q, C, Mc, A.M, H};
    if constexpr (MC > 0)
    {
        // plan fixed at compile time (Mc == MC)
        fft_ct<V, MC, 0, false>(s, A.tw, tid, dif, A.bh + (size_t)q * Mc);
        fft_ct<V, MC, 0, false>(s, A.tw, tid, SrcSmem{s}, nullptr);
    }
    else
    {
        fft_m<V>(s, A.tw, Mc, A.npass, tid, T, dif, A.bh + (size_t)q * Mc);
        fft_m<V>(s, A.tw, Mc, A.npass, tid, T, SrcSmem{s}, nullptr);
    }
    cl.sync();
    // this CTA's share of the half spectrum X_0..X_kmax
    const int nk = A.kmax + 1;
    const int k0 = (int)((long long)nk * q / C);
    const int k1 = (int)((long long)nk * (q + 1) / C);
    double2 *X = A.X + row * A.ldX;
    for (int k = k0 + tid; k < k1; k += T)
    {
        const int ka = (k == H) ? 0 : k;
        const int kb = (k == 0) ? 0 : H - k;
        const double2 va = cluster_v(cl, s, A.twM, C, Mc, A.M, ka);
        const double2 vb = cluster_v(cl, s, A.twM, C, Mc, A.M, kb);
        const double2 zk = cmul(__ldg(&A.w[ka]), conj2(va));
        const double2 zh = conj2(cmul(__ldg(&A.w[kb]), conj2(vb)));
        const double2 e = cmul(__ldg(&A.ht[k]), sub2(zk, zh));
        const double2 sm = add2(zk, zh);
        X[k] = make_double2(0.5 * (sm.x + e.y), 0.5 * (sm.y - e.x));
    }
    // no CTA leaves while another still reads its shared memory
    cl.sync();
}

// Synthesis direction of a cluster plan: rows of even length (ODD false,
// pairs x_2t + i x_2t+1 for t < H) or of odd length H (the real part).
template <int V, int NR, bool ODD, int MC = 0>
__global__ void RFFT_BOUNDS(NR) k_rfftc_inv(RfftArgs A)
{
    namespace cg = cooperative_groups;
    extern __shared__ __align__(16) double2 s[];
    cg::cluster_group cl = cg::this_cluster();
    const int tid = threadIdx.x, T = blockDim.x;
    const int C = A.C, q = (int)cl.block_rank(), H = A.H;
    const int Mc = A.M / C;
    const long long row = blockIdx.x / C;
    if constexpr (ODD)
    {
        SrcSpectrumOdd src{A.X + row * A.ldX, A.w, H, A.kmax};
        SrcClusterDif<SrcSpectrumOdd> dif{src, A.twM, q, C, Mc, A.M, H};
        fft_m<V>(s, A.tw, Mc, A.npass, tid, T, dif, A.bh + (size_t)q * Mc);
    }
    else
    {
        SrcSpectrum src{A.X + row * A.ldX, A.w, A.ht, H, A.kmax};
        SrcClusterDif<SrcSpectrum> dif{src, A.twM, q, C, Mc, A.M, H};
        if constexpr (MC > 0)
            fft_ct<V, MC, 0, false>(s, A.tw, tid, dif,
                                    A.bh + (size_t)q * Mc);
        else
            fft_m<V>(s, A.tw, Mc, A.npass, tid, T, dif,
                     A.bh + (size_t)q * Mc);
    }
    if constexpr (MC > 0)
        fft_ct<V, MC, 0, false>(s, A.tw, tid, SrcSmem{s}, nullptr);
    else
        fft_m<V>(s, A.tw, Mc, A.npass, tid, T, SrcSmem{s}, nullptr);
    cl.sync();
    const int t0 = (int)((long long)H * q / C);
    const int t1 = (int)((long long)H * (q + 1) / C);
    for (int t = t0 + tid; t < t1; t += T)
    {
        const double2 v = cluster_v(cl, s, A.twM, C, Mc, A.M, t);
        const double2 z = cmul(__ldg(&A.w[t]), conj2(v));
        if constexpr (ODD)
            A.x[row * A.ldx + t] = z.x;
        else
            reinterpret_cast<double2 *>(A.x + row * A.ldx)[t] = conj2(z);
    }
    cl.sync();
}

// Residue-ordered FFT_M of the Bluestein kernel, times 1/M: CTA q
// (blockIdx.x, no cluster needed) writes bh[q Mc + l] = FFT_M(b)[C l + q] / M.
template <int V, int NR>
__global__ void RFFT_BOUNDS(NR) k_rfftc_kspec(RfftArgs A, double2 *bh)
{
    extern __shared__ __align__(16) double2 s[];
    const int tid = threadIdx.x, T = blockDim.x;
    const int C = A.C, q = (int)blockIdx.x;
    const int Mc = A.M / C;
    SrcClusterDif<SrcKernel> dif{SrcKernel{A.w, A.H, A.M}, A.twM, q, C, Mc,
                                 A.M, A.M};
    fft_m<V>(s, A.tw, Mc, A.npass, tid, T, dif, nullptr);
    const double inv = 1.0 / (double)A.M;
    for (int l = tid; l < Mc; l += T)
    {
        const double2 v = s[pidx(l)];
        bh[(size_t)q * Mc + l] = make_double2(v.x * inv, v.y * inv);
    }
}

// tw[k] = exp(-2 pi i k / n), k < n
__global__ void k_rfft_twiddles(int n, double2 *tw)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
    {
        double sn, cs;
        sincospi(2.0 * (double)i / (double)n, &sn, &cs);
        tw[i] = make_double2(cs, -sn);
    }
}

// w4[k] = exp(2 pi i k / 4H), k < H
__global__ void k_rfft_w4(int H, double2 *w4)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < H)
    {
        double sn, cs;
        sincospi((double)k / (2.0 * (double)H), &sn, &cs);
        w4[k] = make_double2(cs, sn);
    }
}

// Tables of one transform length: twiddles exp(-2 pi i k / M), chirp
// w_n = exp(-i pi n^2 / H) (n^2 reduced mod 2H in integers), and
// ht_k = exp(-i pi k / H), k <= H.
__global__ void k_rfft_tables(int H, int M, double2 *tw, double2 *w,
                              double2 *ht)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double sn, cs;
    if (i < M)
    {
        sincospi(2.0 * (double)i / (double)M, &sn, &cs);
        tw[i] = make_double2(cs, -sn);
    }
    if (w && i < H)
    {
        long long q = ((long long)i * i) % (2LL * H);
        sincospi((double)q / (double)H, &sn, &cs);
        w[i] = make_double2(cs, -sn);
    }
    if (i <= H)
    {
        sincospi((double)i / (double)H, &sn, &cs);
        ht[i] = make_double2(cs, -sn);
    }
}

// FFT_M of the Bluestein kernel, times 1/M.
template <int V, int NR>
__global__ void RFFT_BOUNDS(NR) k_rfft_kernel_spectrum(RfftArgs A, double2 *bh)
{
    extern __shared__ __align__(16) double2 s[];
    const int tid = threadIdx.x, T = blockDim.x;
    fft_m<V>(s, A.tw, A.M, A.npass, tid, T, SrcKernel{A.w, A.H, A.M},
             nullptr);
    const double inv = 1.0 / (double)A.M;
    for (int k = tid; k < A.M; k += T)
    {
        double2 v = s[pidx(k)];
        bh[k] = make_double2(v.x * inv, v.y * inv);
    }
}

size_t rfft_smem_bytes(int M)
{
    return (size_t)(M + M / 8) * sizeof(double2);
}

cudaError_t launch_rfft_tables(RfftArgs &A, double2 *tw, double2 *w,
                               double2 *ht, double2 *bh, cudaStream_t st)
{
    const int n = (A.M > A.H + 1 ? A.M : A.H + 1);
    k_rfft_tables<<<(n + 255) / 256, 256, 0, st>>>(A.H, A.M, tw, w, ht);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || A.direct)
        return e;
    A.tw = tw;
    A.w = w;
    A.ht = ht;
    const size_t smem = rfft_smem_bytes(A.M);
    k_rfft_kernel_spectrum<16, 96><<<1, A.M / 16, smem, st>>>(A, bh);
    return cudaGetLastError();
}

cudaError_t launch_rfft_w4(int H, double2 *w4, cudaStream_t st)
{
    k_rfft_w4<<<(H + 255) / 256, 256, 0, st>>>(H, w4);
    return cudaGetLastError();
}

cudaError_t rfft_set_smem(size_t smem)
{
    const void *fns[] = {
        (const void *)k_rfft_fwd<16, 96, false, 0>,
        (const void *)k_rfft_inv<16, 96, false, 0>,
        (const void *)k_rfft_fwd<16, 96, true, 0>,
        (const void *)k_rfft_inv<16, 96, true, 0>,
        (const void *)k_rfft_fwd<16, 96, false, 4608>,
        (const void *)k_rfft_inv<16, 96, false, 4608>,
        (const void *)k_rfft_fwd<16, 96, true, 4608>,
        (const void *)k_rfft_inv<16, 96, true, 4608>,
        (const void *)k_rfft_fwd<16, 96, false, 9216>,
        (const void *)k_rfft_inv<16, 96, false, 9216>,
        (const void *)k_rfft_fwd<16, 96, true, 9216>,
        (const void *)k_rfft_inv<16, 96, true, 9216>,
        (const void *)k_rfft_fwd<16, 96, false, 4096>,
        (const void *)k_rfft_inv<16, 96, false, 4096>,
        (const void *)k_rfft_fwd<16, 96, true, 4096>,
        (const void *)k_rfft_inv<16, 96, true, 4096>,
        (const void *)k_rfft_fwd<16, 96, false, 2048>,
        (const void *)k_rfft_inv<16, 96, false, 2048>,
        (const void *)k_rfft_fwd<16, 96, true, 2048>,
        (const void *)k_rfft_inv<16, 96, true, 2048>,
        (const void *)k_rfft_fwd<16, 96, false, 3072>,
        (const void *)k_rfft_inv<16, 96, false, 3072>,
        (const void *)k_rfft_fwd<16, 96, true, 3072>,
        (const void *)k_rfft_inv<16, 96, true, 3072>,
        (const void *)k_rfft_fwd<16, 96, false, 3456>,
        (const void *)k_rfft_inv<16, 96, false, 3456>,
        (const void *)k_rfft_fwd<16, 96, true, 3456>,
        (const void *)k_rfft_inv<16, 96, true, 3456>,
        (const void *)k_rfft_fwd<16, 96, false, 768>,
        (const void *)k_rfft_inv<16, 96, false, 768>,
        (const void *)k_rfft_fwd<16, 96, true, 768>,
        (const void *)k_rfft_inv<16, 96, true, 768>,
        (const void *)k_rfft_fwd<16, 96, false, 1152>,
        (const void *)k_rfft_inv<16, 96, false, 1152>,
        (const void *)k_rfft_fwd<16, 96, true, 1152>,
        (const void *)k_rfft_inv<16, 96, true, 1152>,
        (const void *)k_rfft_inv4<16, 96, 4608>,
        (const void *)k_rfft_kernel_spectrum<16, 96>,
        (const void *)k_rfft_inv_odd<16, 96>,
        (const void *)k_rfftc_fwd<16, 96>,
        (const void *)k_rfftc_inv<16, 96, false>,
        (const void *)k_rfftc_inv<16, 96, true>,
        (const void *)k_rfftc_fwd<16, 96, 6144>,
        (const void *)k_rfftc_inv<16, 96, false, 6144>,
        (const void *)k_rfftc_kspec<16, 96>};
    for (const void *f : fns)
    {
        cudaError_t e = cudaFuncSetAttribute(
            f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess)
            return e;
    }
    // clusters of 16 CTAs (rows beyond 8 x 9216) are a non-portable size
    const void *cfns[] = {(const void *)k_rfftc_fwd<16, 96>,
                          (const void *)k_rfftc_inv<16, 96, false>,
                          (const void *)k_rfftc_inv<16, 96, true>,
                          (const void *)k_rfftc_fwd<16, 96, 6144>,
                          (const void *)k_rfftc_inv<16, 96, false, 6144>};
    for (const void *f : cfns)
    {
        // where refused, plans with 16 CTAs fail their occupancy check
        // (rfftc_max_clusters) instead
        if (cudaFuncSetAttribute(
                f, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
            cudaSuccess)
            cudaGetLastError();
    }
    return cudaSuccess;
}

int rfftc_max_clusters(int C, int Mc)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)C, 1, 1);
    cfg.blockDim = dim3((unsigned)(Mc / 16), 1, 1);
    cfg.dynamicSmemBytes = rfft_smem_bytes(Mc);
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k_rfftc_fwd<16, 96>, &cfg) !=
        cudaSuccess)
    {
        cudaGetLastError();
        return 0;
    }
    int n2 = 0;
    if (cudaOccupancyMaxActiveClusters(&n2, k_rfftc_inv<16, 96, false>,
                                       &cfg) != cudaSuccess)
    {
        cudaGetLastError();
        return 0;
    }
    return n < n2 ? n : n2;
}

cudaError_t launch_rfftc_tables(RfftArgs &A, double2 *tw, double2 *twM,
                                double2 *w, double2 *ht, double2 *bh,
                                cudaStream_t st)
{
    const int Mc = A.M / A.C;
    k_rfft_twiddles<<<(Mc + 255) / 256, 256, 0, st>>>(Mc, tw);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return e;
    const int n = (A.M > A.H + 1 ? A.M : A.H + 1);
    k_rfft_tables<<<(n + 255) / 256, 256, 0, st>>>(A.H, A.M, twM, w, ht);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return e;
    A.tw = tw;
    A.twM = twM;
    A.w = w;
    A.ht = ht;
    k_rfftc_kspec<16, 96><<<A.C, Mc / 16, rfft_smem_bytes(Mc), st>>>(A, bh);
    return cudaGetLastError();
}

cudaError_t launch_rfft(const RfftArgs &A, bool inverse, cudaStream_t st)
{
    const unsigned grid = (unsigned)A.nrows;
    if (grid == 0)
        return cudaSuccess;
    if (A.C > 1)
    {
        // one cluster of A.C CTAs per row
        if (A.f32_rows || A.quarter || A.direct || (!inverse && A.odd))
            return cudaErrorInvalidValue;
        const int Mc = A.M / A.C;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(grid * (unsigned)A.C, 1, 1);
        cfg.blockDim = dim3((unsigned)(Mc / 16), 1, 1);
        cfg.dynamicSmemBytes = rfft_smem_bytes(Mc);
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = (unsigned)A.C;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        // Mc = 6144 (the nmax 10800 rows): the plan fixed at compile time
        const bool ct = Mc == 6144;
        if (!inverse)
            return ct ? cudaLaunchKernelEx(&cfg, k_rfftc_fwd<16, 96, 6144>, A)
                      : cudaLaunchKernelEx(&cfg, k_rfftc_fwd<16, 96>, A);
        if (A.odd)
            return cudaLaunchKernelEx(&cfg, k_rfftc_inv<16, 96, true>, A);
        return ct ? cudaLaunchKernelEx(&cfg, k_rfftc_inv<16, 96, false, 6144>,
                                       A)
                  : cudaLaunchKernelEx(&cfg, k_rfftc_inv<16, 96, false>, A);
    }
    const size_t smem = rfft_smem_bytes(A.M);
    const int T = A.M / 16;
    if (A.odd)
    {
        // rows of odd length: synthesis only, Bluestein, run-time plan
        if (!inverse || A.f32_rows || A.direct)
            return cudaErrorInvalidValue;
        k_rfft_inv_odd<16, 96><<<grid, T, smem, st>>>(A);
        return cudaGetLastError();
    }
    if (A.quarter)
    {
        // two CTAs per row (rfft plans set quarter only with M = 4608,
        // double rows, synthesis)
        if (!inverse || A.M != 4608 || A.f32_rows || A.direct)
            return cudaErrorInvalidValue;
        k_rfft_inv4<16, 96, 4608><<<2 * grid, T, smem, st>>>(A);
        return cudaGetLastError();
    }
    // the grids' common Bluestein lengths with the plan fixed at compile
    // time
    auto go = [&](auto mc) {
        constexpr int MC = decltype(mc)::value;
        constexpr int NR = 96;
        if (A.f32_rows)
        {
            if (inverse)
                k_rfft_inv<16, NR, true, MC><<<grid, T, smem, st>>>(A);
            else
                k_rfft_fwd<16, NR, true, MC><<<grid, T, smem, st>>>(A);
        }
        else if (inverse)
            k_rfft_inv<16, NR, false, MC><<<grid, T, smem, st>>>(A);
        else
            k_rfft_fwd<16, NR, false, MC><<<grid, T, smem, st>>>(A);
    };
    if (A.direct)
        go(std::integral_constant<int, 0>{});
    else if (A.M == 4608)
        go(std::integral_constant<int, 4608>{});
    else if (A.M == 9216)
        go(std::integral_constant<int, 9216>{});
    else if (A.M == 4096)
        go(std::integral_constant<int, 4096>{});
    else if (A.M == 2048)
        go(std::integral_constant<int, 2048>{});
    else if (A.M == 1152)
        go(std::integral_constant<int, 1152>{});
    else if (A.M == 768)
        go(std::integral_constant<int, 768>{});
    else if (A.M == 3072)
        go(std::integral_constant<int, 3072>{});
    else if (A.M == 3456)
        go(std::integral_constant<int, 3456>{});
    else
        go(std::integral_constant<int, 0>{});
    return cudaGetLastError();
}

} // namespace cb
