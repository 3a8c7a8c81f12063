/* FFT shim with FFTW 3's interface (declared in fftw3.h), used only to build
 * CHarm's own sources as the oracle's reference CPU implementation
 * (oracle/build_ref.py).  Compiled once per precision:
 *
 *     -DSHIM_PREC=1   double      fftw_*
 *     -DSHIM_PREC=2   float       fftwf_*
 *     -DSHIM_PREC=3   __float128  fftwq_*  (libquadmath)
 *
 * Algorithms (all standard, written here from their textbook statements):
 *
 *   - complex DFT of length n by the Stockham autosort form of the
 *     decimation-in-frequency Cooley-Tukey FFT, one pass per radix
 *     (4, 2, 3, 5 with explicit butterflies; other primes up to 31 by an
 *     O(r^2) butterfly), data held as separate real / imaginary arrays so
 *     that the inner loops vectorise;
 *   - lengths with a prime factor above 31 by Bluestein's chirp-z identity
 *     2jk = j^2 + k^2 - (k - j)^2, i.e. a circular convolution of length
 *     M >= 2n - 1 (M = 2^a 3^b 5^c) done with the FFT above; the chirp
 *     exp(-i pi k^2 / n) uses k^2 mod 2n in exact integer arithmetic;
 *   - real transforms of even length n through one complex DFT of length
 *     n/2 (even samples as real parts, odd samples as imaginary parts) and
 *     the usual split of its spectrum; odd n through a complex DFT of
 *     length n;
 *   - the inverse DFT as conj(DFT(conj(x))).
 *
 * Twiddles are computed in a wider type (long double for double, double for
 * float) or in binary128 with libquadmath's cosq / sinq.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#include "fftw3.h"

#if SHIM_PREC == 1
typedef double R;
typedef long double TW;
#define X(name) fftw_##name
#define COSW(a) cosl(a)
#define SINW(a) sinl(a)
#define PIW 3.141592653589793238462643383279502884L
#define VERSION_STR "fftw-3-oracle-shim-double"
#elif SHIM_PREC == 2
typedef float R;
typedef double TW;
#define X(name) fftwf_##name
#define COSW(a) cos(a)
#define SINW(a) sin(a)
#define PIW 3.141592653589793238462643383279502884
#define VERSION_STR "fftw-3-oracle-shim-float"
#elif SHIM_PREC == 3
#include <quadmath.h>
typedef __float128 R;
typedef __float128 TW;
#define X(name) fftwq_##name
#define COSW(a) cosq(a)
#define SINW(a) sinq(a)
#define PIW M_PIq
#define VERSION_STR "fftw-3-oracle-shim-quad"
#else
#error "define SHIM_PREC as 1 (double), 2 (float) or 3 (quad)"
#endif

typedef R C2[2];

#define MAXST 64
#define MAXGEN 31

/* ------------------------------------------------------------------------ */
/* Complex plan                                                              */
/* ------------------------------------------------------------------------ */
typedef struct cplan {
    int n;
    int nst;                 /* Stockham passes (0 when n == 1 or Bluestein) */
    int radix[MAXST];
    size_t twoff[MAXST];     /* offset of each pass's twiddles in tw_* */
    R *tw_re, *tw_im;        /* pass twiddles w_len^(p k), p < len/r, k < r */
    R *gen_re, *gen_im;      /* generic butterflies: w_r^(j k) per radix, r^2 */
    size_t genoff[MAXGEN + 1];
    /* Bluestein */
    int blue;
    int M;
    struct cplan *inner;
    R *ch_re, *ch_im;        /* c_k = exp(-i pi k^2 / n), k < n */
    R *bf_re, *bf_im;        /* DFT_M of the filter conj(c_|l|), scaled 1/M */
} cplan;

static void *xalloc(size_t bytes)
{
    void *p = NULL;
    if (bytes == 0)
        bytes = 64;
    if (posix_memalign(&p, 64, (bytes + 63) & ~(size_t)63) != 0)
        return NULL;
    return p;
}

static int smallest_factor(int n)
{
    if (n % 4 == 0)
        return 4;
    for (int f = 2; (long)f * f <= n; f++)
        if (n % f == 0)
            return f;
    return n;
}

static int is_smooth31(int n)
{
    for (int f = 2; f <= MAXGEN && n > 1; f++)
        while (n % f == 0)
            n /= f;
    return n == 1;
}

static int bluestein_length(int n)
{
    long need = 2L * n - 1, best = -1;
    for (long a = 1; a < 4 * need; a *= 2)
        for (long b = a; b < 4 * need; b *= 3)
            for (long c = b; c < 4 * need; c *= 5)
                if (c >= need && (best < 0 || c < best))
                    best = c;
    return (int)best;
}

static void cplan_free(cplan *p);
static void cfft(const cplan *p, R *re, R *im, R *wre, R *wim);

static cplan *cplan_make(int n)
{
    cplan *p = (cplan *)calloc(1, sizeof(cplan));
    if (p == NULL)
        return NULL;
    p->n = n;
    if (n <= 1)
        return p;
    if (!is_smooth31(n)) {
        /* Bluestein */
        int M = bluestein_length(n);
        p->blue = 1;
        p->M = M;
        p->inner = cplan_make(M);
        p->ch_re = (R *)xalloc(sizeof(R) * n);
        p->ch_im = (R *)xalloc(sizeof(R) * n);
        p->bf_re = (R *)xalloc(sizeof(R) * M);
        p->bf_im = (R *)xalloc(sizeof(R) * M);
        R *wre = (R *)xalloc(sizeof(R) * M);
        R *wim = (R *)xalloc(sizeof(R) * M);
        if (!p->inner || !p->ch_re || !p->ch_im || !p->bf_re || !p->bf_im ||
            !wre || !wim) {
            free(wre);
            free(wim);
            cplan_free(p);
            return NULL;
        }
        uint64_t twon = 2u * (uint64_t)n;
        for (int k = 0; k < n; k++) {
            uint64_t q = ((uint64_t)k * (uint64_t)k) % twon;
            TW a = PIW * (TW)q / (TW)n;
            p->ch_re[k] = (R)COSW(a);
            p->ch_im[k] = (R)(-SINW(a));
        }
        for (int l = 0; l < M; l++) {
            p->bf_re[l] = 0;
            p->bf_im[l] = 0;
        }
        for (int l = 0; l < n; l++) {
            p->bf_re[l] = p->ch_re[l];
            p->bf_im[l] = -p->ch_im[l];
            if (l > 0) {
                p->bf_re[M - l] = p->ch_re[l];
                p->bf_im[M - l] = -p->ch_im[l];
            }
        }
        cfft(p->inner, p->bf_re, p->bf_im, wre, wim);
        for (int l = 0; l < M; l++) {
            p->bf_re[l] /= (R)M;
            p->bf_im[l] /= (R)M;
        }
        free(wre);
        free(wim);
        return p;
    }
    /* Stockham passes */
    int len = n, nst = 0;
    size_t tot = 0;
    while (len > 1) {
        int r = smallest_factor(len);
        p->radix[nst] = r;
        p->twoff[nst] = tot;
        tot += (size_t)len;
        len /= r;
        nst++;
    }
    p->nst = nst;
    p->tw_re = (R *)xalloc(sizeof(R) * tot);
    p->tw_im = (R *)xalloc(sizeof(R) * tot);
    size_t gtot = 0;
    for (int r = 0; r <= MAXGEN; r++)
        p->genoff[r] = 0;
    for (int st = 0; st < nst; st++) {
        int r = p->radix[st];
        if (r > 5 && r <= MAXGEN && p->genoff[r] == 0) {
            p->genoff[r] = gtot + 1;   /* 1-based: 0 means absent */
            gtot += (size_t)r * r;
        }
    }
    p->gen_re = (R *)xalloc(sizeof(R) * (gtot + 1));
    p->gen_im = (R *)xalloc(sizeof(R) * (gtot + 1));
    if (!p->tw_re || !p->tw_im || !p->gen_re || !p->gen_im) {
        cplan_free(p);
        return NULL;
    }
    len = n;
    for (int st = 0; st < nst; st++) {
        int r = p->radix[st], m = len / r;
        R *tr = p->tw_re + p->twoff[st], *ti = p->tw_im + p->twoff[st];
        for (int q = 0; q < m; q++)
            for (int k = 0; k < r; k++) {
                long e = ((long)q * k) % len;
                TW a = 2 * PIW * (TW)e / (TW)len;
                tr[q * r + k] = (R)COSW(a);
                ti[q * r + k] = (R)(-SINW(a));
            }
        len = m;
    }
    for (int r = 6; r <= MAXGEN; r++) {
        if (p->genoff[r] == 0)
            continue;
        R *gr = p->gen_re + p->genoff[r] - 1, *gi = p->gen_im + p->genoff[r] - 1;
        for (int j = 0; j < r; j++)
            for (int k = 0; k < r; k++) {
                long e = ((long)j * k) % r;
                TW a = 2 * PIW * (TW)e / (TW)r;
                gr[j * r + k] = (R)COSW(a);
                gi[j * r + k] = (R)(-SINW(a));
            }
    }
    return p;
}

static void cplan_free(cplan *p)
{
    if (p == NULL)
        return;
    free(p->tw_re);
    free(p->tw_im);
    free(p->gen_re);
    free(p->gen_im);
    free(p->ch_re);
    free(p->ch_im);
    free(p->bf_re);
    free(p->bf_im);
    cplan_free(p->inner);
    free(p);
}

/* One Stockham pass of radix r: x (length len = r m, stride s) -> y.
 * Output y[t + s (r q + k)] = w_len^(q k) sum_j x[t + s q + j s m] w_r^(j k)
 * for q < m, t < s.  The loop over t is innermost when s is large enough to
 * vectorise, otherwise the loop over q is. */
#define RADIX_LOOPS(...)                                                      \
    if (s >= 4) {                                                             \
        for (int q = 0; q < m; q++) {                                         \
            _Pragma("omp simd")                                               \
            for (int t = 0; t < s; t++) {                                     \
                __VA_ARGS__                                                   \
            }                                                                 \
        }                                                                     \
    } else {                                                                  \
        for (int t = 0; t < s; t++)                                           \
            _Pragma("omp simd")                                               \
            for (int q = 0; q < m; q++) {                                     \
                __VA_ARGS__                                                   \
            }                                                                 \
    }

#define LD(j) const size_t i##j = (size_t)s * q + t + (size_t)(j) * sm;      \
    const R x##j##r = xr[i##j], x##j##i = xi[i##j];
#define ST(k, br, bi)                                                         \
    {                                                                         \
        const size_t o = (size_t)s * ((size_t)RAD * q + (k)) + t;             \
        const R wr_ = tr[(size_t)RAD * q + (k)];                              \
        const R wi_ = ti[(size_t)RAD * q + (k)];                              \
        yr[o] = (br) * wr_ - (bi) * wi_;                                      \
        yi[o] = (br) * wi_ + (bi) * wr_;                                      \
    }

static void pass(int r, int m, int s, const R *restrict tr,
                 const R *restrict ti, const R *gr, const R *gi,
                 const R *restrict xr, const R *restrict xi,
                 R *restrict yr, R *restrict yi)
{
    const size_t sm = (size_t)s * m;
    if (r == 2) {
        enum { RAD = 2 };
        RADIX_LOOPS(
            LD(0) LD(1)
            const size_t o = (size_t)s * 2 * q + t;
            yr[o] = x0r + x1r;
            yi[o] = x0i + x1i;
            ST(1, x0r - x1r, x0i - x1i))
    } else if (r == 4) {
        enum { RAD = 4 };
        RADIX_LOOPS(
            LD(0) LD(1) LD(2) LD(3)
            const R s02r = x0r + x2r, s02i = x0i + x2i;
            const R d02r = x0r - x2r, d02i = x0i - x2i;
            const R s13r = x1r + x3r, s13i = x1i + x3i;
            const R d13r = x1r - x3r, d13i = x1i - x3i;
            /* forward: X1 = d02 - i d13, X3 = d02 + i d13 */
            const size_t o = (size_t)s * 4 * q + t;
            yr[o] = s02r + s13r;
            yi[o] = s02i + s13i;
            ST(1, d02r + d13i, d02i - d13r)
            ST(2, s02r - s13r, s02i - s13i)
            ST(3, d02r - d13i, d02i + d13r))
    } else if (r == 3) {
        /* w_3 = c1 + i s1 */
        const R c1 = (R)(-0.5), s1 = (R)(-SINW(2 * PIW / 3));
        enum { RAD = 3 };
        RADIX_LOOPS(
            LD(0) LD(1) LD(2)
            const R pr = x1r + x2r, pi = x1i + x2i;
            const R mr = x1r - x2r, mi = x1i - x2i;
            const R hr = x0r + c1 * pr, hi = x0i + c1 * pi;
            const size_t o = (size_t)s * 3 * q + t;
            yr[o] = x0r + pr;
            yi[o] = x0i + pi;
            /* X1 = h + i s1 m, X2 = h - i s1 m */
            ST(1, hr - s1 * mi, hi + s1 * mr)
            ST(2, hr + s1 * mi, hi - s1 * mr))
    } else if (r == 5) {
        const R c1 = (R)COSW(2 * PIW / 5), c2 = (R)COSW(4 * PIW / 5);
        const R s1 = (R)(-SINW(2 * PIW / 5)), s2 = (R)(-SINW(4 * PIW / 5));
        enum { RAD = 5 };
        RADIX_LOOPS(
            LD(0) LD(1) LD(2) LD(3) LD(4)
            const R p1r = x1r + x4r, p1i = x1i + x4i;
            const R m1r = x1r - x4r, m1i = x1i - x4i;
            const R p2r = x2r + x3r, p2i = x2i + x3i;
            const R m2r = x2r - x3r, m2i = x2i - x3i;
            const R t1r = x0r + c1 * p1r + c2 * p2r;
            const R t1i = x0i + c1 * p1i + c2 * p2i;
            const R t2r = x0r + c2 * p1r + c1 * p2r;
            const R t2i = x0i + c2 * p1i + c1 * p2i;
            /* i (s1 m1 + s2 m2) and i (s2 m1 - s1 m2) */
            const R u1r = -(s1 * m1i + s2 * m2i), u1i = s1 * m1r + s2 * m2r;
            const R u2r = -(s2 * m1i - s1 * m2i), u2i = s2 * m1r - s1 * m2r;
            const size_t o = (size_t)s * 5 * q + t;
            yr[o] = x0r + p1r + p2r;
            yi[o] = x0i + p1i + p2i;
            ST(1, t1r + u1r, t1i + u1i)
            ST(2, t2r + u2r, t2i + u2i)
            ST(3, t2r - u2r, t2i - u2i)
            ST(4, t1r - u1r, t1i - u1i))
    } else {
        /* generic radix r (odd prime <= MAXGEN): O(r^2) butterfly */
        const int RAD = r;
        for (int q = 0; q < m; q++)
            for (int k = 0; k < r; k++)
                for (int t = 0; t < s; t++) {
                    R accr = 0, acci = 0;
                    for (int j = 0; j < r; j++) {
                        const size_t ii = (size_t)s * q + t + (size_t)j * sm;
                        const R cr = gr[(size_t)j * r + k];
                        const R ci = gi[(size_t)j * r + k];
                        accr += xr[ii] * cr - xi[ii] * ci;
                        acci += xr[ii] * ci + xi[ii] * cr;
                    }
                    ST(k, accr, acci)
                }
    }
}
#undef LD
#undef ST
#undef RADIX_LOOPS

/* Forward complex DFT in place on (re, im); (wre, wim) is scratch of the
 * plan's length, or 2 M + M for a Bluestein plan. */
static void cfft(const cplan *p, R *re, R *im, R *wre, R *wim)
{
    const int n = p->n;
    if (n <= 1)
        return;
    if (p->blue) {
        const int M = p->M;
        R *ar = wre, *ai = wim;                 /* M */
        R *sr = wre + M, *si = wim + M;          /* inner scratch, M */
        for (int j = 0; j < n; j++) {
            R xr = re[j], xi = im[j];
            ar[j] = xr * p->ch_re[j] - xi * p->ch_im[j];
            ai[j] = xr * p->ch_im[j] + xi * p->ch_re[j];
        }
        for (int j = n; j < M; j++) {
            ar[j] = 0;
            ai[j] = 0;
        }
        cfft(p->inner, ar, ai, sr, si);
        /* pointwise product, then the inverse DFT as conj(DFT(conj(.))) */
        for (int j = 0; j < M; j++) {
            R xr = ar[j], xi = ai[j];
            R br = p->bf_re[j], bi = p->bf_im[j];
            ar[j] = xr * br - xi * bi;
            ai[j] = -(xr * bi + xi * br);
        }
        cfft(p->inner, ar, ai, sr, si);
        for (int k = 0; k < n; k++) {
            R yr = ar[k], yi = -ai[k];
            re[k] = yr * p->ch_re[k] - yi * p->ch_im[k];
            im[k] = yr * p->ch_im[k] + yi * p->ch_re[k];
        }
        return;
    }
    R *xr = re, *xi = im, *yr = wre, *yi = wim;
    int len = n, s = 1;
    for (int st = 0; st < p->nst; st++) {
        int r = p->radix[st], m = len / r;
        const R *gr = NULL, *gi = NULL;
        if (r > 5)
            gr = p->gen_re + p->genoff[r] - 1, gi = p->gen_im + p->genoff[r] - 1;
        pass(r, m, s, p->tw_re + p->twoff[st], p->tw_im + p->twoff[st], gr, gi,
             xr, xi, yr, yi);
        R *t;
        t = xr; xr = yr; yr = t;
        t = xi; xi = yi; yi = t;
        len = m;
        s *= r;
    }
    if (xr != re) {
        memcpy(re, xr, sizeof(R) * n);
        memcpy(im, xi, sizeof(R) * n);
    }
}

/* ------------------------------------------------------------------------ */
/* Real plans (FFTW interface)                                               */
/* ------------------------------------------------------------------------ */
struct X(plan_s) {
    int n;
    int dir;          /* -1: r2c, +1: c2r */
    int h;            /* complex length: n / 2 (even n) or n (odd n) */
    cplan *cp;
    R *wk_re, *wk_im; /* exp(-2 pi i k / n), k <= n / 2 (even n) */
    size_t scratch;   /* reals per array needed by one execution */
};

static __thread R *tls_buf = NULL;
static __thread size_t tls_cap = 0;

/* Distance between the four scratch arrays: the length rounded up to 64
 * bytes plus an odd number of 64-byte lines, so that the arrays do not
 * start at the same cache set when the length is a large power of two. */
static size_t scratch_ld(size_t nreal)
{
    const size_t line = 64 / sizeof(R) ? 64 / sizeof(R) : 1;
    return (nreal + line - 1) / line * line + 3 * line;
}

static R *scratch_get(size_t nreal)
{
    if (nreal > tls_cap) {
        free(tls_buf);
        tls_buf = (R *)xalloc(sizeof(R) * nreal);
        tls_cap = tls_buf ? nreal : 0;
    }
    return tls_buf;
}

static X(plan) plan_make(int n, int dir)
{
    if (n < 1)
        return NULL;
    X(plan) p = (X(plan))calloc(1, sizeof(*p));
    if (p == NULL)
        return NULL;
    p->n = n;
    p->dir = dir;
    p->h = (n % 2 == 0) ? n / 2 : n;
    p->cp = cplan_make(p->h);
    if (p->cp == NULL) {
        free(p);
        return NULL;
    }
    if (n % 2 == 0) {
        int h = n / 2;
        p->wk_re = (R *)xalloc(sizeof(R) * (h + 1));
        p->wk_im = (R *)xalloc(sizeof(R) * (h + 1));
        if (!p->wk_re || !p->wk_im) {
            X(destroy_plan)(p);
            return NULL;
        }
        for (int k = 0; k <= h; k++) {
            TW a = 2 * PIW * (TW)k / (TW)n;
            p->wk_re[k] = (R)COSW(a);
            p->wk_im[k] = (R)(-SINW(a));
        }
    }
    size_t inner = p->cp->blue ? (size_t)p->cp->M * 2 : (size_t)p->h;
    p->scratch = (size_t)p->h + inner;
    return p;
}

X(plan) X(plan_dft_r2c_1d)(int n, R *in, X(complex) *out, unsigned flags)
{
    (void)in;
    (void)out;
    (void)flags;
    return plan_make(n, -1);
}

X(plan) X(plan_dft_c2r_1d)(int n, X(complex) *in, R *out, unsigned flags)
{
    (void)in;
    (void)out;
    (void)flags;
    return plan_make(n, +1);
}

void X(execute_dft_r2c)(const X(plan) p, R *in, X(complex) *out)
{
    const int n = p->n, h = p->h;
    const size_t ld = scratch_ld(p->scratch);
    R *buf = scratch_get(4 * ld);
    if (buf == NULL)
        return;
    R *zr = buf, *zi = buf + ld;
    R *wr = buf + 2 * ld, *wi = buf + 3 * ld;
    if (n % 2 != 0) {
        for (int j = 0; j < n; j++) {
            zr[j] = in[j];
            zi[j] = 0;
        }
        cfft(p->cp, zr, zi, wr, wi);
        for (int k = 0; k <= n / 2; k++) {
            out[k][0] = zr[k];
            out[k][1] = zi[k];
        }
        return;
    }
    for (int j = 0; j < h; j++) {
        zr[j] = in[2 * j];
        zi[j] = in[2 * j + 1];
    }
    cfft(p->cp, zr, zi, wr, wi);
    const R half = (R)0.5;
    for (int k = 0; k <= h; k++) {
        int k1 = (k == h) ? 0 : k;
        int k2 = (k == 0) ? 0 : h - k;
        R ar = zr[k1], ai = zi[k1];
        R br = zr[k2], bi = -zi[k2];          /* conj(Z_{h-k}) */
        R er = half * (ar + br), ei = half * (ai + bi);
        /* O = -i (A - B) / 2 */
        R or_ = half * (ai - bi), oi = -half * (ar - br);
        R wre = p->wk_re[k], wim = p->wk_im[k];
        out[k][0] = er + (or_ * wre - oi * wim);
        out[k][1] = ei + (or_ * wim + oi * wre);
    }
}

void X(execute_dft_c2r)(const X(plan) p, X(complex) *in, R *out)
{
    const int n = p->n, h = p->h;
    const size_t ld = scratch_ld(p->scratch);
    R *buf = scratch_get(4 * ld);
    if (buf == NULL)
        return;
    R *zr = buf, *zi = buf + ld;
    R *wr = buf + 2 * ld, *wi = buf + 3 * ld;
    if (n % 2 != 0) {
        /* Hermitian extension, inverse DFT as conj(DFT(conj(.))) */
        zr[0] = in[0][0];
        zi[0] = 0;
        for (int k = 1; k <= n / 2; k++) {
            zr[k] = in[k][0];
            zi[k] = -in[k][1];
            zr[n - k] = in[k][0];
            zi[n - k] = in[k][1];
        }
        cfft(p->cp, zr, zi, wr, wi);
        for (int j = 0; j < n; j++)
            out[j] = zr[j];
        return;
    }
    for (int k = 0; k < h; k++) {
        R ar = in[k][0], ai = (k == 0) ? (R)0 : in[k][1];
        int k2 = h - k;
        R br = in[k2][0], bi = (k2 == h) ? (R)0 : -in[k2][1];  /* conj X_{h-k} */
        R er = ar + br, ei = ai + bi;                   /* 2 E_k */
        R dr = ar - br, di = ai - bi;
        /* 2 O_k = (A - B) exp(+2 pi i k / n) */
        R wre = p->wk_re[k], wim = -p->wk_im[k];
        R or_ = dr * wre - di * wim, oi = dr * wim + di * wre;
        /* Z_k = 2E + i 2O, conjugated for the inverse */
        zr[k] = er - oi;
        zi[k] = -(ei + or_);
    }
    cfft(p->cp, zr, zi, wr, wi);
    for (int j = 0; j < h; j++) {
        out[2 * j] = zr[j];
        out[2 * j + 1] = -zi[j];
    }
}

void X(destroy_plan)(X(plan) p)
{
    if (p == NULL)
        return;
    cplan_free(p->cp);
    free(p->wk_re);
    free(p->wk_im);
    free(p);
}

void *X(malloc)(size_t n)
{
    return xalloc(n);
}

void X(free)(void *p)
{
    free(p);
}

void X(cleanup)(void)
{
}

int X(init_threads)(void)
{
    return 1;
}

void X(plan_with_nthreads)(int nthreads)
{
    (void)nthreads;
}

void X(cleanup_threads)(void)
{
}

const char X(version)[] = VERSION_STR;
