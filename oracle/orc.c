/* ORACLE -- TEST INFRASTRUCTURE ONLY.
 *
 * A CPU restatement, in plain C, of CHarm 0.4.9's point spherical-harmonic
 * synthesis and analysis (the Legendre sums with X-number arithmetic, the
 * lumped-coefficient post-processing, and the Gauss--Legendre and
 * Driscoll--Healy grid generators).  It is the checker that the CUDA path is
 * compared against: only the test-suite, the smoke check and the CPU-baseline
 * leg of bench.py load it.  The product library never links or calls it.
 *
 * The file compiles twice: as double precision (symbols "orc_d_*") and, with
 * -DORC_QUAD, as IEEE binary128 via libquadmath (symbols "orc_q_*").  The
 * quad build stands in for CHarm's own quadruple-precision build, which cannot
 * be compiled here (it needs FFTW and configure-generated headers).
 *
 * Citations are to files of the CHarm source tree.  Every arithmetic step
 * restates the reference in the same order of operations, so in double the
 * results agree with CHarm to the rounding of its SIMD/OpenMP summation order.
 * The longitude sums (FFT in CHarm) are done by the Python side of the oracle
 * (oracle/orc.py); this file produces and consumes the lumped coefficients.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef ORC_QUAD
#include <quadmath.h>
typedef __float128 real;
#define RSQRT sqrtq
#define RSIN sinq
#define RCOS cosq
#define RASIN asinq
#define RFABS fabsq
#define RLDEXP ldexpq
#define ORC(x) orc_q_##x
#define XRADIX 16000
#define REPS FLT128_EPSILON
#define RPI M_PIq
#define RPI_2 M_PI_2q
#define RROOT3 1.732050807568877293527446341505872367Q
#else
typedef double real;
#define RSQRT sqrt
#define RSIN sin
#define RCOS cos
#define RASIN asin
#define RFABS fabs
#define RLDEXP ldexp
#define ORC(x) orc_d_##x
#define XRADIX 960
#define REPS DBL_EPSILON
#define RPI 3.14159265358979323846
#define RPI_2 1.57079632679489661923
#define RROOT3 1.73205080756887729353
#endif

/* X-number radix constants, src/prec.h:293-320 (double), :210-237 (quad). */
static real BIG, BIGI, BIGS, BIGSI;
static int consts_ready = 0;

static void init_consts(void)
{
    if (consts_ready)
        return;
    BIG = RLDEXP((real)1, XRADIX);
    BIGI = RLDEXP((real)1, -XRADIX);
    BIGS = RLDEXP((real)1, XRADIX / 2);
    BIGSI = RLDEXP((real)1, -XRADIX / 2);
    consts_ready = 1;
}

/* glob_threshold = 100 eps, src/glob/glob.c:16 */
#define THRESHOLD ((real)100 * REPS)

/* src/misc/misc_is_nearly_equal.c:20-31 */
static int nearly_equal(real a, real b, real eps)
{
    real aa = RFABS(a), ba = RFABS(b), d = RFABS(a - b), s = aa + ba;
    if (a == b)
        return 1;
    if (a == (real)0 || b == (real)0)
        return d <= eps;
    if (s == aa || s == ba)
        return d <= eps;
    return d / (aa > ba ? aa : ba) <= eps;
}

/* ------------------------------------------------------------------------ */
/* Recurrence coefficient tables                                            */
/* ------------------------------------------------------------------------ */

/* sqrt(k) and 1/sqrt(k) for k <= 2 nmax + 3, src/leg/leg_func_r_ri.c:15-30 */
static void leg_r_ri(unsigned long nmax, real *r, real *ri)
{
    r[0] = ri[0] = 0;
    for (unsigned long k = 1; k <= 2 * nmax + 3; k++)
    {
        real w = RSQRT((real)k);
        r[k] = w;
        ri[k] = (real)1 / w;
    }
}

/* Sectorial factors, src/leg/leg_func_dm.c:14-22 */
static void leg_dm(unsigned long nmax, const real *r, const real *ri, real *dm)
{
    dm[0] = 0;
    for (unsigned long n = 1; n <= nmax; n++)
        dm[n] = r[2 * n + 3] * ri[2 * n + 2];
}

/* a_nm, b_nm, src/leg/leg_func_anm_bnm.c:14-65 */
static void leg_anm_bnm(unsigned long nmax, unsigned long m, const real *r,
                        const real *ri, real *anm, real *bnm)
{
    anm[m] = bnm[m] = 0;
    if (m == nmax)
        return;
    anm[m + 1] = r[2 * m + 3];
    bnm[m + 1] = 0;
    for (unsigned long n = m + 2; n <= nmax; n++)
    {
        real w = r[2 * n + 1] * ri[n - m] * ri[n + m];
        anm[n] = r[2 * n - 1] * w;
        bnm[n] = r[n - m - 1] * r[n + m - 1] * ri[2 * n - 3] * w;
    }
}

/* e_nm, src/leg/leg_func_enm.c:14-55 */
static void leg_enm(unsigned long nmax, unsigned long m, const real *r,
                    const real *ri, real *enm)
{
    enm[m] = 0;
    for (unsigned long n = m + 1; n <= nmax; n++)
        enm[n] = r[2 * n + 1] * r[n - m] * r[n + m] * ri[2 * n - 1];
}

/* ------------------------------------------------------------------------ */
/* X-number primitives (scalar), src/leg/leg_func_xnum.h:299-443           */
/* ------------------------------------------------------------------------ */
static inline real x2f(real x, int64_t ix)
{
    if (ix == 0)
        return x;
    else if (ix < -1)
        return 0;
    else if (ix < 0)
        return x * BIGI;
    return x * BIG;
}

static inline void xnorm(real *x, int64_t *ix)
{
    real w = RFABS(*x);
    if (w >= BIGS)
    {
        *x *= BIGI;
        *ix += 1;
    }
    else if (w < BIGSI)
    {
        *x *= BIG;
        *ix -= 1;
    }
}

/* Sectorial seeds for one latitude, src/leg/leg_func_prepare.c:18-69.
 * ps[k], ips[k] hold P_{k+1,k+1}. */
static void leg_prepare(real u, const real *dm, unsigned long nmax, real *ps,
                        int64_t *ips)
{
    if (nmax == 0)
        return;
    real x = RROOT3 * u;
    int64_t ix = 0;
    ps[0] = x;
    ips[0] = ix;
    for (unsigned long n = 1; n < nmax; n++)
    {
        x = (dm[n] * u) * x;
        real y = RFABS(x);
        if (y >= BIGS)
        {
            x *= BIGI;
            ix += 1;
        }
        else if (y < BIGSI)
        {
            x *= BIG;
            ix -= 1;
        }
        ps[n] = x;
        ips[n] = ix;
    }
}

/* ------------------------------------------------------------------------ */
/* Synthesis kernel, src/shs/shs_point_kernel.c:745-2010                    */
/* ------------------------------------------------------------------------ */
/* Lumped coefficients of one order "m" at one latitude (and its mirror if
 * "symm").  Index layout of "lc": [quantity][north/south][a/b] with quantity
 * 0 = potential-like ("a"), 1 = "r", 2 = "p", 3 = "rr", 4 = "rp", 5 = "pp"
 * (src/shs/shs_lc_struct.h:17-72). */
typedef struct
{
    real v[6][2][2];
} lc_t;

enum { Q0 = 0, QR, QP, QRR, QRP, QPP };

typedef struct
{
    int kgrad;     /* 0 single quantity, 1 full grad1, 2 full grad2 */
    int dr, dlat, dlon;
    unsigned dorder;
} kmode_t;

/* Add the contribution of degree "n" with Legendre values p (dp, ddp).
 * "even" is the parity of n+m; rp, rp2 are (R/r)^(n+1+dorder) at the latitude
 * and at its mirror.  Restates LFCS/LCAB, shs_point_kernel.c:355-540. */
static inline void add_term(const kmode_t *k, lc_t *lc, unsigned long n,
                            real p, real dp, real ddp, real cnm, real snm,
                            real rp, real rp2, int symm, int even)
{
    real cs[2] = {cnm, snm};
    for (int j = 0; j < 2; j++)
    {
        real leg[6] = {0, 0, 0, 0, 0, 0};
        int qs[6];
        int nq = 0;
        int sgn[6]; /* +1 add to mirror when even, -1 subtract when even */
        if (k->kgrad == 0)
        {
            real base = (k->dlat == 0) ? p : ((k->dlat == 1) ? dp : ddp);
            real l = base * cs[j];
            if (k->dr == 1)
                l = (real)(n + 1) * l;
            else if (k->dr == 2)
                l = (real)((n + 1) * (n + 2)) * l;
            leg[0] = l;
            qs[0] = Q0;
            /* SIGN1/SIGN2, shs_point_kernel.c:224-240: dlat == 1 flips */
            sgn[0] = (k->dlat == 1) ? -1 : 1;
            nq = 1;
        }
        else
        {
            real l = p * cs[j];
            real lr = (real)(n + 1) * l;
            real lp = dp * cs[j];
            leg[0] = l;
            qs[0] = Q0;
            sgn[0] = 1;
            leg[1] = lr;
            qs[1] = QR;
            sgn[1] = 1;
            leg[2] = lp;
            qs[2] = QP;
            sgn[2] = -1;
            nq = 3;
            if (k->kgrad == 2)
            {
                leg[3] = (real)(n + 2) * lr;
                qs[3] = QRR;
                sgn[3] = 1;
                leg[4] = (real)(n + 1) * lp;
                qs[4] = QRP;
                sgn[4] = -1;
                leg[5] = ddp * cs[j];
                qs[5] = QPP;
                sgn[5] = 1;
                nq = 6;
            }
        }
        for (int q = 0; q < nq; q++)
        {
            lc->v[qs[q]][0][j] = lc->v[qs[q]][0][j] + rp * leg[q];
            if (symm)
            {
                real t2 = rp2 * leg[q];
                int add = even ? (sgn[q] > 0) : (sgn[q] < 0);
                if (add)
                    lc->v[qs[q]][1][j] = lc->v[qs[q]][1][j] + t2;
                else
                    lc->v[qs[q]][1][j] = lc->v[qs[q]][1][j] - t2;
            }
        }
    }
}

static inline void neg2(lc_t *lc, int q, int symm)
{
    for (int h = 0; h < (symm ? 2 : 1); h++)
        for (int j = 0; j < 2; j++)
            lc->v[q][h][j] = -lc->v[q][h][j];
}

/* dlon1: (a, b) <- (m b, -m a), shs_point_kernel.c:680-700 */
static inline void dlon1(real *a, real *b, unsigned long m)
{
    real ta = *a;
    *a = (real)m * (*b);
    *b = (real)m * (-ta);
}

static void shs_kernel(const kmode_t *k, unsigned long nmax, unsigned long m,
                       const real *cm, const real *sm, const real *anm,
                       const real *bnm, const real *enm, real t, real u,
                       const real *ps, const int64_t *ips,
                       const real *rpows, const real *rpows2, int symm,
                       lc_t *lc)
{
    memset(lc, 0, sizeof(*lc));
    unsigned dorder = k->dorder;
    int need_dp = (k->kgrad > 0) || (k->dlat > 0);
    int need_ddp = (k->kgrad > 1) || (k->dlat > 1);
    real u_rec = (real)1 / u;
    real tu = t * u_rec;
    real u2_rec = u_rec * u_rec;
    real m2s = (real)(m * m);
#define RP(n) rpows[(n) + 1 + dorder]
#define RP2(n) (symm ? rpows2[(n) + 1 + dorder] : (real)0)
    if (m == 0)
    {
        /* Zonal harmonics, shs_point_kernel.c:1014-1248 */
        real p0 = 1, dp0 = 0, ddp0 = 0;
        add_term(k, lc, 0, p0, dp0, ddp0, cm[0], 0, RP(0), RP2(0), symm, 1);
        if (nmax >= 1)
        {
            real p1 = RROOT3 * t;
            real dp1 = RROOT3 * u;
            real ddp1 = -p1;
            add_term(k, lc, 1, p1, dp1, ddp1, cm[1], 0, RP(1), RP2(1), symm,
                     0);
            int even = 1;
            for (unsigned long n = 2; n <= nmax; n++, even = !even)
            {
                real p2 = (anm[n] * t) * p1 - bnm[n] * p0;
                real dp2 = 0, ddp2 = 0;
                if (need_dp)
                    dp2 = (enm[n] * u_rec) * p1 - ((real)n * tu) * p2;
                if (need_ddp)
                    ddp2 = tu * dp2 +
                           (m2s * u2_rec - (real)(n * (n + 1))) * p2;
                add_term(k, lc, n, p2, dp2, ddp2, cm[n], 0, RP(n), RP2(n),
                         symm, even);
                p0 = p1;
                p1 = p2;
            }
        }
    }
    else
    {
        /* Sectorial, shs_point_kernel.c:1255-1370 */
        real x = ps[m - 1];
        int64_t ix = ips[m - 1];
        real pnm0 = x2f(x, ix);
        real ns = (real)m;
        real dpnm0 = 0, ddpnm0 = 0;
        if (need_dp)
            dpnm0 = -(((ns * t) * u_rec) * pnm0);
        if (need_ddp)
            ddpnm0 = tu * dpnm0 +
                     (m2s * u2_rec - (real)(m * (m + 1))) * pnm0;
        add_term(k, lc, m, pnm0, dpnm0, ddpnm0, cm[0], sm[0], RP(m), RP2(m),
                 symm, 1);
        if (m < nmax)
        {
            /* Semi-sectorial, shs_point_kernel.c:1375-1460 */
            unsigned long n = m + 1;
            real y = x;
            int64_t iy = ix;
            x = (anm[n] * t) * y;
            ix = iy;
            xnorm(&x, &ix);
            real pnm1 = x2f(x, ix);
            real dpnm1 = 0, ddpnm1 = 0;
            if (need_dp)
                dpnm1 = (enm[n] * u_rec) * pnm0 - ((real)n * tu) * pnm1;
            if (need_ddp)
                ddpnm1 = tu * dpnm1 +
                         (m2s * u2_rec - (real)(n * (n + 1))) * pnm1;
            add_term(k, lc, n, pnm1, dpnm1, ddpnm1, cm[1], sm[1], RP(n),
                     RP2(n), symm, 0);

            /* Tesseral: X-numbers until dynamical switching, then
             * F-numbers, shs_point_kernel.c:1464-1623 */
            int ds = 0;
            int even = 1;
            real prev = pnm1; /* F-number P_{n-1} for the derivative */
            for (n = m + 2; n <= nmax; n++, even = !even)
            {
                real pnm2;
                if (ds)
                {
                    pnm2 = (anm[n] * t) * x - bnm[n] * y;
                    y = x;
                    x = pnm2;
                }
                else
                {
                    int64_t ixy = ix - iy, iz;
                    real z;
                    if (ixy == 0)
                    {
                        z = (anm[n] * t) * x - bnm[n] * y;
                        iz = ix;
                    }
                    else if (ixy == 1)
                    {
                        z = (anm[n] * t) * x - bnm[n] * (y * BIGI);
                        iz = ix;
                    }
                    else if (ixy == -1)
                    {
                        z = (anm[n] * t) * (x * BIGI) - bnm[n] * y;
                        iz = iy;
                    }
                    else if (ixy > 1)
                    {
                        z = (anm[n] * t) * x;
                        iz = ix;
                    }
                    else
                    {
                        z = -bnm[n] * y;
                        iz = iy;
                    }
                    xnorm(&z, &iz);
                    y = x;
                    iy = ix;
                    x = z;
                    ix = iz;
                    pnm2 = x2f(z, iz);
                    if (ix == 0 && iy == 0)
                        ds = 1;
                }
                real dp2 = 0, ddp2 = 0;
                if (need_dp)
                    dp2 = (enm[n] * u_rec) * prev - ((real)n * tu) * pnm2;
                if (need_ddp)
                    ddp2 = tu * dp2 +
                           (m2s * u2_rec - (real)(n * (n + 1))) * pnm2;
                add_term(k, lc, n, pnm2, dp2, ddp2, cm[n - m], sm[n - m],
                         RP(n), RP2(n), symm, even);
                prev = pnm2;
            }
        }
    }
#undef RP
#undef RP2

    /* Post-processing, shs_point_kernel.c:1643-1946 */
    if (k->kgrad == 0 && k->dr == 1)
        neg2(lc, Q0, symm);
    if (k->kgrad > 0)
        neg2(lc, QR, symm);
    if (k->kgrad > 1)
        neg2(lc, QRP, symm);

    int nh = symm ? 2 : 1;
    if (k->kgrad == 0)
    {
        for (int h = 0; h < nh; h++)
        {
            real *a = &lc->v[Q0][h][0], *b = &lc->v[Q0][h][1];
            if (k->dlon == 1)
            {
                *a = u_rec * *a;
                *b = u_rec * *b;
                dlon1(a, b, m);
            }
            else if (k->dlon == 2)
            {
                *a = u2_rec * *a;
                *b = u2_rec * *b;
                real mm = (real)(m * m);
                *a = mm * (-*a);
                *b = mm * (-*b);
            }
        }
    }
    else if (k->kgrad == 1)
    {
        for (int h = 0; h < nh; h++)
        {
            real *a = &lc->v[Q0][h][0], *b = &lc->v[Q0][h][1];
            dlon1(a, b, m);
            *a = -*a;
            *b = -*b;
            *a = u_rec * *a;
            *b = u_rec * *b;
        }
    }
    else
    {
        for (int h = 0; h < nh; h++)
        {
            /* The mirror latitude has tu -> -tu (the reference's PM
             * arguments in YY and XY). */
            real tuh = (h == 0) ? tu : -tu;
            for (int j = 0; j < 2; j++)
            {
                /* xx */
                lc->v[QPP][h][j] = lc->v[QR][h][j] + lc->v[QPP][h][j];
            }
            real a_ = lc->v[Q0][h][0], b_ = lc->v[Q0][h][1];
            /* yy: dlon2 then YY */
            real mm = (real)(m * m);
            real a = mm * (-lc->v[Q0][h][0]);
            real b = mm * (-lc->v[Q0][h][1]);
            lc->v[Q0][h][0] = (u2_rec * a - tuh * lc->v[QP][h][0]) +
                              lc->v[QR][h][0];
            lc->v[Q0][h][1] = (u2_rec * b - tuh * lc->v[QP][h][1]) +
                              lc->v[QR][h][1];
            /* xz */
            for (int j = 0; j < 2; j++)
                lc->v[QRP][h][j] = lc->v[QRP][h][j] - lc->v[QP][h][j];
            /* xy */
            dlon1(&lc->v[QP][h][0], &lc->v[QP][h][1], m);
            dlon1(&a_, &b_, m);
            lc->v[QP][h][0] = -(u_rec * lc->v[QP][h][0]) -
                              (tuh * u_rec) * a_;
            lc->v[QP][h][1] = -(u_rec * lc->v[QP][h][1]) -
                              (tuh * u_rec) * b_;
            /* yz */
            dlon1(&lc->v[QR][h][0], &lc->v[QR][h][1], m);
            lc->v[QR][h][0] = u_rec * (a_ - lc->v[QR][h][0]);
            lc->v[QR][h][1] = u_rec * (b_ - lc->v[QR][h][1]);
        }
    }
}

/* Order of the lumped quantities as written to the output: for grad1 "l",
 * "r", "p"; for grad2 "ll", "lr", "lp", "rr", "rp", "pp"
 * (src/shs/shs_grd_fft_lc.c:120-150). */
static int npar_of(const kmode_t *k)
{
    return k->kgrad == 1 ? 3 : (k->kgrad == 2 ? 6 : 1);
}

/* Public: lumped coefficients of synthesis.
 *
 * nmax       maximum degree of the synthesis
 * shc_nmax   maximum degree of the coefficient triangle in c, s
 * c, s       coefficient triangles, order-major c[m][n-m] with row lengths
 *            shc_nmax+1-m (src/shc/shc_init_chunk.c:126-145)
 * nrow       number of evaluated latitudes
 * lat        latitudes of the evaluated rows
 * rr, rr2    R/r at the row and at its mirror
 * symm       1 if the row has a mirror at -lat
 * mode       kgrad, dr, dlat, dlon
 * a, b       out [npar][nrow][nmax+1] for the rows
 * a2, b2     out [npar][nrow][nmax+1] for the mirrors (zero when !symm)
 */
void ORC(shs_lumped)(unsigned long nmax, unsigned long shc_nmax,
                     const real *c, const real *s, size_t nrow,
                     const real *lat, const real *rr, const real *rr2,
                     const int *symm, int kgrad, int dr, int dlat, int dlon,
                     real *a, real *b, real *a2, real *b2)
{
    init_consts();
    kmode_t k = {kgrad, dr, dlat, dlon, 0};
    if (kgrad == 1)
        k.dorder = 1;
    else if (kgrad == 2)
        k.dorder = 2;
    else
        k.dorder = (unsigned)(dr + dlat + dlon);
    int npar = npar_of(&k);
    size_t L = nmax + 1;
    real *r = calloc(2 * nmax + 4, sizeof(real));
    real *ri = calloc(2 * nmax + 4, sizeof(real));
    real *dm = calloc(nmax + 1, sizeof(real));
    leg_r_ri(nmax, r, ri);
    leg_dm(nmax, r, ri, dm);
    /* column starts of the coefficient triangle */
    size_t *col = malloc((shc_nmax + 1) * sizeof(size_t));
    size_t idx = 0;
    for (unsigned long m = 0; m <= shc_nmax; m++)
    {
        col[m] = idx;
        idx += shc_nmax + 1 - m;
    }
    memset(a, 0, (size_t)npar * nrow * L * sizeof(real));
    memset(b, 0, (size_t)npar * nrow * L * sizeof(real));
    memset(a2, 0, (size_t)npar * nrow * L * sizeof(real));
    memset(b2, 0, (size_t)npar * nrow * L * sizeof(real));

#pragma omp parallel
    {
        real *anm = calloc(nmax + 2, sizeof(real));
        real *bnm = calloc(nmax + 2, sizeof(real));
        real *enm = calloc(nmax + 2, sizeof(real));
        real *ps = calloc(nmax + 1, sizeof(real));
        int64_t *ips = calloc(nmax + 1, sizeof(int64_t));
        real *rp = malloc((nmax + 4) * sizeof(real));
        real *rp2 = malloc((nmax + 4) * sizeof(real));
#pragma omp for schedule(dynamic)
        for (size_t i = 0; i < nrow; i++)
        {
            real t = RSIN(lat[i]);
            real u = RCOS(lat[i]);
            /* r-powers, src/shs/shs_rpows.c:16-37 */
            rp[0] = rp2[0] = 1;
            for (size_t q = 1; q < nmax + 4; q++)
            {
                rp[q] = rp[q - 1] * rr[i];
                rp2[q] = rp2[q - 1] * rr2[i];
            }
            leg_prepare(u, dm, nmax, ps, ips);
            for (unsigned long m = 0; m <= nmax; m++)
            {
                leg_anm_bnm(nmax, m, r, ri, anm, bnm);
                if (k.dorder > 0)
                    leg_enm(nmax, m, r, ri, enm);
                lc_t lc;
                shs_kernel(&k, nmax, m, c + col[m], s + col[m], anm, bnm, enm,
                           t, u, ps, ips, rp, rp2, symm[i], &lc);
                static const int order1[3] = {Q0, QR, QP};
                static const int order2[6] = {Q0, QR, QP, QRR, QRP, QPP};
                for (int p = 0; p < npar; p++)
                {
                    int q = (k.kgrad == 2) ? order2[p]
                                           : ((k.kgrad == 1) ? order1[p] : Q0);
                    size_t o = ((size_t)p * nrow + i) * L + m;
                    a[o] = lc.v[q][0][0];
                    b[o] = lc.v[q][0][1];
                    if (symm[i])
                    {
                        a2[o] = lc.v[q][1][0];
                        b2[o] = lc.v[q][1][1];
                    }
                }
            }
        }
        free(anm);
        free(bnm);
        free(enm);
        free(ps);
        free(ips);
        free(rp);
        free(rp2);
    }
    free(r);
    free(ri);
    free(dm);
    free(col);
}

/* ------------------------------------------------------------------------ */
/* Analysis contraction, src/sha/sha_point.c:713-980                        */
/* ------------------------------------------------------------------------ */
/* Given, for each evaluated latitude, the quadrature-weighted Fourier
 * coefficients amp, amm, bmp, bmm [nrow][nmax+1] (sha_point.c:728-748),
 * accumulate C_nm, S_nm into the order-major triangles c, s of degree nmax
 * (which must be zeroed by the caller). */
void ORC(sha_contract)(unsigned long nmax, size_t nrow, const real *lat,
                       const real *amp, const real *amm, const real *bmp,
                       const real *bmm, real *c, real *s)
{
    init_consts();
    size_t L = nmax + 1;
    real *r = calloc(2 * nmax + 4, sizeof(real));
    real *ri = calloc(2 * nmax + 4, sizeof(real));
    real *dm = calloc(nmax + 1, sizeof(real));
    leg_r_ri(nmax, r, ri);
    leg_dm(nmax, r, ri, dm);
    size_t *col = malloc((nmax + 1) * sizeof(size_t));
    size_t idx = 0;
    for (unsigned long m = 0; m <= nmax; m++)
    {
        col[m] = idx;
        idx += nmax + 1 - m;
    }
    real *ps = calloc(nrow * (nmax + 1), sizeof(real));
    int64_t *ips = calloc(nrow * (nmax + 1), sizeof(int64_t));
    real *t = malloc(nrow * sizeof(real));
    for (size_t i = 0; i < nrow; i++)
    {
        t[i] = RSIN(lat[i]);
        leg_prepare(RCOS(lat[i]), dm, nmax, ps + i * (nmax + 1),
                    ips + i * (nmax + 1));
    }
#pragma omp parallel
    {
        real *anm = calloc(nmax + 2, sizeof(real));
        real *bnm = calloc(nmax + 2, sizeof(real));
#pragma omp for schedule(dynamic)
        for (unsigned long m = 0; m <= nmax; m++)
        {
            leg_anm_bnm(nmax, m, r, ri, anm, bnm);
            real *cm = c + col[m], *sm = s + col[m];
            for (size_t i = 0; i < nrow; i++)
            {
                const real *ap = amp + i * L, *am = amm + i * L;
                const real *bp = bmp + i * L, *bm = bmm + i * L;
                real ti = t[i];
                if (m == 0)
                {
                    real p0 = 1;
                    cm[0] += p0 * ap[0];
                    if (nmax >= 1)
                    {
                        real p1 = RROOT3 * ti;
                        cm[1] += p1 * am[0];
                        int even = 1;
                        for (unsigned long n = 2; n <= nmax; n++, even = !even)
                        {
                            real p2 = (anm[n] * ti) * p1 - bnm[n] * p0;
                            p0 = p1;
                            p1 = p2;
                            cm[n] += p2 * (even ? ap[0] : am[0]);
                        }
                    }
                    continue;
                }
                real x = ps[i * (nmax + 1) + m - 1];
                int64_t ix = ips[i * (nmax + 1) + m - 1];
                real pnm0 = x2f(x, ix);
                cm[0] += pnm0 * ap[m];
                sm[0] += pnm0 * bp[m];
                if (m == nmax)
                    continue;
                unsigned long n = m + 1;
                real y = x;
                int64_t iy = ix;
                x = (anm[n] * ti) * y;
                ix = iy;
                xnorm(&x, &ix);
                real pnm1 = x2f(x, ix);
                cm[1] += pnm1 * am[m];
                sm[1] += pnm1 * bm[m];
                int ds = 0, even = 1;
                for (n = m + 2; n <= nmax; n++, even = !even)
                {
                    real pnm2;
                    if (ds)
                    {
                        pnm2 = (anm[n] * ti) * x - bnm[n] * y;
                        y = x;
                        x = pnm2;
                    }
                    else
                    {
                        int64_t ixy = ix - iy, iz;
                        real z;
                        if (ixy == 0)
                        {
                            z = (anm[n] * ti) * x - bnm[n] * y;
                            iz = ix;
                        }
                        else if (ixy == 1)
                        {
                            z = (anm[n] * ti) * x - bnm[n] * (y * BIGI);
                            iz = ix;
                        }
                        else if (ixy == -1)
                        {
                            z = (anm[n] * ti) * (x * BIGI) - bnm[n] * y;
                            iz = iy;
                        }
                        else if (ixy > 1)
                        {
                            z = (anm[n] * ti) * x;
                            iz = ix;
                        }
                        else
                        {
                            z = -bnm[n] * y;
                            iz = iy;
                        }
                        xnorm(&z, &iz);
                        y = x;
                        iy = ix;
                        x = z;
                        ix = iz;
                        pnm2 = x2f(z, iz);
                        if (ix == 0 && iy == 0)
                            ds = 1;
                    }
                    cm[n - m] += pnm2 * (even ? ap[m] : am[m]);
                    sm[n - m] += pnm2 * (even ? bp[m] : bm[m]);
                }
            }
        }
        free(anm);
        free(bnm);
    }
    free(r);
    free(ri);
    free(dm);
    free(col);
    free(ps);
    free(ips);
    free(t);
}

/* ------------------------------------------------------------------------ */
/* Block-mean values in cells: latitude integrals of the Legendre functions  */
/* ------------------------------------------------------------------------ */
/* Un-normalised Legendre recurrence P_n = e_n t P_n-1 - f_n P_n-2,
 * src/leg/leg_pol_en_fn.c:14-38 (arrays of nmax + 1 entries). */
static void leg_en_fn(unsigned long nmax, real *en, real *fn)
{
    en[0] = fn[0] = 0;
    if (nmax == 0)
        return;
    en[1] = fn[1] = 0;
    for (unsigned long n = 2; n <= nmax; n++)
    {
        en[n] = (real)(2 * n - 1) / (real)n;
        fn[n] = (real)(n - 1) / (real)n;
    }
}

/* Coefficients of the integral recurrences, src/leg/leg_func_gm_hm.c:14-45:
 * I_mm = g_m I_m-2,m-2 + (t2 P_mm(t2) - t1 P_mm(t1)) / (m + 1) and
 * I_nm = h_n b_nm I_n-2,m - a_nm / (n + 1) (u2^2 P_n-1,m(t2) - ...). */
static void leg_gm_hm(unsigned long nmax, const real *r, const real *ri,
                      real *gm, real *hm)
{
    for (unsigned long n = 0; n <= nmax && n < 3; n++)
        gm[n] = 0;
    for (unsigned long n = 3; n <= nmax; n++)
        gm[n] = (real)1 / (real)(2 * n + 2) * r[n] * r[2 * n + 1] *
                r[2 * n - 1] * ri[n - 1];
    for (unsigned long n = 0; n <= nmax; n++)
        hm[n] = (real)((long)n - 2) / (real)(n + 1);
}

/* X-number state of one latitude's recurrence over the degrees and its
 * tesseral step (PNM_TESSERAL_XNUM, src/leg/leg_func_xnum.h), the same
 * arithmetic as the loop of shs_kernel above.  Returns P_n,m as an
 * F-number (zero below the X-number range). */
typedef struct
{
    real x, y;
    int64_t ix, iy;
    int ds;
} xrec_t;

static inline real xrec_sectorial(xrec_t *s, const real *ps,
                                  const int64_t *ips, unsigned long m)
{
    s->x = ps[m - 1];
    s->ix = ips[m - 1];
    s->y = 0;
    s->iy = 0;
    s->ds = 0;
    return x2f(s->x, s->ix);
}

static inline real xrec_semisectorial(xrec_t *s, real t, real anm)
{
    s->y = s->x;
    s->iy = s->ix;
    s->x = (anm * t) * s->y;
    s->ix = s->iy;
    xnorm(&s->x, &s->ix);
    return x2f(s->x, s->ix);
}

static inline real xrec_tesseral(xrec_t *s, real t, real anm, real bnm)
{
    real pnm2;
    if (s->ds)
    {
        pnm2 = (anm * t) * s->x - bnm * s->y;
        s->y = s->x;
        s->x = pnm2;
        return pnm2;
    }
    int64_t ixy = s->ix - s->iy, iz;
    real z;
    if (ixy == 0)
    {
        z = (anm * t) * s->x - bnm * s->y;
        iz = s->ix;
    }
    else if (ixy == 1)
    {
        z = (anm * t) * s->x - bnm * (s->y * BIGI);
        iz = s->ix;
    }
    else if (ixy == -1)
    {
        z = (anm * t) * (s->x * BIGI) - bnm * s->y;
        iz = s->iy;
    }
    else if (ixy > 1)
    {
        z = (anm * t) * s->x;
        iz = s->ix;
    }
    else
    {
        z = -bnm * s->y;
        iz = s->iy;
    }
    xnorm(&z, &iz);
    s->y = s->x;
    s->iy = s->ix;
    s->x = z;
    s->ix = iz;
    pnm2 = x2f(z, iz);
    if (s->ix == 0 && s->iy == 0)
        s->ds = 1;
    return pnm2;
}

/* I_mm of one cell row for m = 0..nmax (imm[0] unused), the sectorial
 * integrals of src/sha/sha_cell.c:586-660 (and the imm0..imm2 state that
 * src/shs/shs_cell_kernel.c:229-268 carries over the orders). */
static void cell_imm(unsigned long nmax, real latmin, real latmax, real t1,
                     real u1, real t2, real u2, const real *ps1,
                     const int64_t *ips1, const real *ps2,
                     const int64_t *ips2, const real *gm, real *imm)
{
    imm[0] = 0;
    for (unsigned long m = 1; m <= nmax; m++)
    {
        real p1 = x2f(ps1[m - 1], ips1[m - 1]);
        real p2 = x2f(ps2[m - 1], ips2[m - 1]);
        if (m == 1)
            imm[m] = (RROOT3 / (real)2) *
                     ((t2 * u2 - (RPI_2 - latmax)) -
                      (t1 * u1 - (RPI_2 - latmin)));
        else if (m == 2)
            imm[m] = (RSQRT((real)15) / (real)6) *
                     (t2 * ((real)3 - t2 * t2) - t1 * ((real)3 - t1 * t1));
        else
            imm[m] = gm[m] * imm[m - 2] +
                     ((real)1 / (real)(m + 1)) * (t2 * p2 - t1 * p1);
    }
}

/* Public: lumped coefficients of the cell synthesis, the latitude integrals
 * of src/shs/shs_cell_kernel.c:68-470 for every row and order:
 *   a_m = sum_n (R/r)^(n+1) I_nm C_nm,  b_m likewise with S_nm,
 * a2, b2 for the mirror row [-latmax, -latmin] ((-1)^(n+m) I_nm) when
 * symm[i].  Outputs [nrow][nmax+1]; orders skipped by the polar
 * optimisation (thr >= 0: m - nmax cos(latmin) > thr) are zero. */
void ORC(cell_lumped)(unsigned long nmax, unsigned long shc_nmax,
                      const real *c, const real *s, size_t nrow,
                      const real *latmin, const real *latmax, const real *rr,
                      const real *rr2, const int *symm, double polar_thr,
                      real *a, real *b, real *a2, real *b2)
{
    init_consts();
    size_t L = nmax + 1;
    real *r = calloc(2 * nmax + 6, sizeof(real));
    real *ri = calloc(2 * nmax + 6, sizeof(real));
    real *dm = calloc(nmax + 2, sizeof(real));
    real *en = calloc(nmax + 3, sizeof(real));
    real *fn = calloc(nmax + 3, sizeof(real));
    real *gm = calloc(nmax + 2, sizeof(real));
    real *hm = calloc(nmax + 2, sizeof(real));
    leg_r_ri(nmax, r, ri);
    leg_dm(nmax, r, ri, dm);
    leg_en_fn(nmax + 1, en, fn);
    leg_gm_hm(nmax, r, ri, gm, hm);
    size_t *col = malloc((shc_nmax + 1) * sizeof(size_t));
    size_t idx = 0;
    for (unsigned long m = 0; m <= shc_nmax; m++)
    {
        col[m] = idx;
        idx += shc_nmax + 1 - m;
    }
    memset(a, 0, nrow * L * sizeof(real));
    memset(b, 0, nrow * L * sizeof(real));
    memset(a2, 0, nrow * L * sizeof(real));
    memset(b2, 0, nrow * L * sizeof(real));

#pragma omp parallel
    {
        real *anm = calloc(nmax + 2, sizeof(real));
        real *bnm = calloc(nmax + 2, sizeof(real));
        real *ps1 = calloc(nmax + 1, sizeof(real));
        real *ps2 = calloc(nmax + 1, sizeof(real));
        int64_t *ips1 = calloc(nmax + 1, sizeof(int64_t));
        int64_t *ips2 = calloc(nmax + 1, sizeof(int64_t));
        real *imm = calloc(nmax + 1, sizeof(real));
#pragma omp for schedule(dynamic)
        for (size_t i = 0; i < nrow; i++)
        {
            real t1 = RSIN(latmin[i]), u1 = RCOS(latmin[i]);
            real t2 = RSIN(latmax[i]), u2 = RCOS(latmax[i]);
            leg_prepare(u1, dm, nmax, ps1, ips1);
            leg_prepare(u2, dm, nmax, ps2, ips2);
            cell_imm(nmax, latmin[i], latmax[i], t1, u1, t2, u2, ps1, ips1,
                     ps2, ips2, gm, imm);
            const int sy = symm[i];
            const real ratio = rr[i], ratio2 = sy ? rr2[i] : (real)0;
            real ratiom = ratio, ratio2m = ratio2;
            real *ar = a + i * L, *br = b + i * L;
            real *a2r = a2 + i * L, *b2r = b2 + i * L;
            for (unsigned long m = 0; m <= nmax;
                 m++, ratiom *= ratio, ratio2m *= ratio2)
            {
                if (polar_thr >= 0.0 &&
                    (real)polar_thr < (real)m - (real)nmax * u1)
                    continue;
                leg_anm_bnm(nmax, m, r, ri, anm, bnm);
                const real *cm = c + col[m], *sm = s + col[m];
                real ration = ratiom, ratio2n = ratio2m;
                real A = 0, B = 0, A2 = 0, B2 = 0;
                if (m == 0)
                {
                    /* zonal: un-normalised P_n and
                     * I_n0 = (P_n+1 - P_n-1) / sqrt(2n+1),
                     * shs_cell_kernel.c:97-175 */
                    real p0a = 1, p0b = 1, p1a = t1, p1b = t2;
                    real in0 = t2 - t1;
                    real v = in0 * cm[0];
                    A = ration * v;
                    ration *= ratio;
                    if (sy)
                    {
                        A2 = ratio2n * v;
                        ratio2n *= ratio2;
                    }
                    int even = 0;
                    for (unsigned long n = 1; n <= nmax; n++, even = !even)
                    {
                        real p2a = en[n + 1] * (t1 * p1a) - fn[n + 1] * p0a;
                        real p2b = en[n + 1] * (t2 * p1b) - fn[n + 1] * p0b;
                        in0 = ri[2 * n + 1] * ((p2b - p0b) - (p2a - p0a));
                        v = in0 * cm[n];
                        A = A + ration * v;
                        ration *= ratio;
                        if (sy)
                        {
                            A2 = even ? A2 + ratio2n * v : A2 - ratio2n * v;
                            ratio2n *= ratio2;
                        }
                        p0a = p1a;
                        p1a = p2a;
                        p0b = p1b;
                        p1b = p2b;
                    }
                }
                else
                {
                    xrec_t s1, s2;
                    real q1 = xrec_sectorial(&s1, ps1, ips1, m);
                    real q2 = xrec_sectorial(&s2, ps2, ips2, m);
                    real inm0 = imm[m];
                    real vc = inm0 * cm[0], vs = inm0 * sm[0];
                    A = ration * vc;
                    B = ration * vs;
                    ration *= ratio;
                    if (sy)
                    {
                        A2 = ratio2n * vc;
                        B2 = ratio2n * vs;
                        ratio2n *= ratio2;
                    }
                    if (m < nmax)
                    {
                        real pm1 = q1, pm2 = q2; /* P_mm */
                        q1 = xrec_semisectorial(&s1, t1, anm[m + 1]);
                        q2 = xrec_semisectorial(&s2, t2, anm[m + 1]);
                        real inm1 = -((anm[m + 1] / (real)(m + 2)) *
                                      ((u2 * u2) * pm2 - (u1 * u1) * pm1));
                        vc = inm1 * cm[1];
                        vs = inm1 * sm[1];
                        A = A + ration * vc;
                        B = B + ration * vs;
                        ration *= ratio;
                        if (sy)
                        {
                            A2 = A2 - ratio2n * vc;
                            B2 = B2 - ratio2n * vs;
                            ratio2n *= ratio2;
                        }
                        int even = 1;
                        for (unsigned long n = m + 2; n <= nmax;
                             n++, even = !even)
                        {
                            real pa = q1, pb = q2; /* P_n-1,m */
                            q1 = xrec_tesseral(&s1, t1, anm[n], bnm[n]);
                            q2 = xrec_tesseral(&s2, t2, anm[n], bnm[n]);
                            real inm2 = (hm[n] * bnm[n]) * inm0 -
                                        (anm[n] / (real)(n + 1)) *
                                        ((u2 * u2) * pb - (u1 * u1) * pa);
                            inm0 = inm1;
                            inm1 = inm2;
                            vc = inm2 * cm[n - m];
                            vs = inm2 * sm[n - m];
                            A = A + ration * vc;
                            B = B + ration * vs;
                            ration *= ratio;
                            if (sy)
                            {
                                if (even)
                                {
                                    A2 = A2 + ratio2n * vc;
                                    B2 = B2 + ratio2n * vs;
                                }
                                else
                                {
                                    A2 = A2 - ratio2n * vc;
                                    B2 = B2 - ratio2n * vs;
                                }
                                ratio2n *= ratio2;
                            }
                        }
                    }
                }
                ar[m] = A;
                br[m] = B;
                a2r[m] = A2;
                b2r[m] = B2;
            }
        }
        free(anm);
        free(bnm);
        free(ps1);
        free(ps2);
        free(ips1);
        free(ips2);
        free(imm);
    }
    free(r);
    free(ri);
    free(dm);
    free(en);
    free(fn);
    free(gm);
    free(hm);
    free(col);
}

/* Public: the Legendre contraction of the cell analysis,
 * src/sha/sha_cell.c:560-1110.  amp, amm, bmp, bmm [nrow][nmax+1] are the
 * longitude-integrated Fourier sums of each row (and its mirror) as formed
 * at sha_cell.c:790-840; C_nm, S_nm accumulate into the order-major
 * triangles c, s of degree nmax (zeroed by the caller), before the
 * 1 / (4 pi) r / mu factor. */
void ORC(cell_contract)(unsigned long nmax, size_t nrow, const real *latmin,
                        const real *latmax, const real *amp, const real *amm,
                        const real *bmp, const real *bmm, double polar_thr,
                        real *c, real *s)
{
    init_consts();
    size_t L = nmax + 1;
    real *r = calloc(2 * nmax + 6, sizeof(real));
    real *ri = calloc(2 * nmax + 6, sizeof(real));
    real *dm = calloc(nmax + 2, sizeof(real));
    real *en = calloc(nmax + 3, sizeof(real));
    real *fn = calloc(nmax + 3, sizeof(real));
    real *gm = calloc(nmax + 2, sizeof(real));
    real *hm = calloc(nmax + 2, sizeof(real));
    leg_r_ri(nmax, r, ri);
    leg_dm(nmax, r, ri, dm);
    leg_en_fn(nmax + 1, en, fn);
    leg_gm_hm(nmax, r, ri, gm, hm);
    size_t *col = malloc((nmax + 1) * sizeof(size_t));
    size_t idx = 0;
    for (unsigned long m = 0; m <= nmax; m++)
    {
        col[m] = idx;
        idx += nmax + 1 - m;
    }
    real *geo = malloc(nrow * 4 * sizeof(real));
    real *ps1 = calloc(nrow * L, sizeof(real));
    real *ps2 = calloc(nrow * L, sizeof(real));
    int64_t *ips1 = calloc(nrow * L, sizeof(int64_t));
    int64_t *ips2 = calloc(nrow * L, sizeof(int64_t));
    real *imm = calloc(nrow * L, sizeof(real));
    for (size_t i = 0; i < nrow; i++)
    {
        real *g = geo + 4 * i;
        g[0] = RSIN(latmin[i]);
        g[1] = RCOS(latmin[i]);
        g[2] = RSIN(latmax[i]);
        g[3] = RCOS(latmax[i]);
        leg_prepare(g[1], dm, nmax, ps1 + i * L, ips1 + i * L);
        leg_prepare(g[3], dm, nmax, ps2 + i * L, ips2 + i * L);
        cell_imm(nmax, latmin[i], latmax[i], g[0], g[1], g[2], g[3],
                 ps1 + i * L, ips1 + i * L, ps2 + i * L, ips2 + i * L, gm,
                 imm + i * L);
    }
#pragma omp parallel
    {
        real *anm = calloc(nmax + 2, sizeof(real));
        real *bnm = calloc(nmax + 2, sizeof(real));
#pragma omp for schedule(dynamic)
        for (unsigned long m = 0; m <= nmax; m++)
        {
            leg_anm_bnm(nmax, m, r, ri, anm, bnm);
            real *cm = c + col[m], *sm = s + col[m];
            for (size_t i = 0; i < nrow; i++)
            {
                const real *g = geo + 4 * i;
                const real t1 = g[0], u1 = g[1], t2 = g[2], u2 = g[3];
                if (polar_thr >= 0.0 &&
                    (real)polar_thr < (real)m - (real)nmax * u1)
                    continue;
                const real ap = amp[i * L + m], am = amm[i * L + m];
                const real bp = bmp[i * L + m], bm = bmm[i * L + m];
                if (m == 0)
                {
                    real p0a = 1, p0b = 1, p1a = t1, p1b = t2;
                    cm[0] += (t2 - t1) * ap;
                    int even = 0;
                    for (unsigned long n = 1; n <= nmax; n++, even = !even)
                    {
                        real p2a = en[n + 1] * (t1 * p1a) - fn[n + 1] * p0a;
                        real p2b = en[n + 1] * (t2 * p1b) - fn[n + 1] * p0b;
                        real in0 = ri[2 * n + 1] * ((p2b - p0b) - (p2a - p0a));
                        cm[n] += in0 * (even ? ap : am);
                        p0a = p1a;
                        p1a = p2a;
                        p0b = p1b;
                        p1b = p2b;
                    }
                    continue;
                }
                xrec_t s1, s2;
                real q1 = xrec_sectorial(&s1, ps1 + i * L, ips1 + i * L, m);
                real q2 = xrec_sectorial(&s2, ps2 + i * L, ips2 + i * L, m);
                real inm0 = imm[i * L + m];
                cm[0] += inm0 * ap;
                sm[0] += inm0 * bp;
                if (m == nmax)
                    continue;
                real pm1 = q1, pm2 = q2;
                q1 = xrec_semisectorial(&s1, t1, anm[m + 1]);
                q2 = xrec_semisectorial(&s2, t2, anm[m + 1]);
                real inm1 = -((anm[m + 1] / (real)(m + 2)) *
                              ((u2 * u2) * pm2 - (u1 * u1) * pm1));
                cm[1] += inm1 * am;
                sm[1] += inm1 * bm;
                int even = 1;
                for (unsigned long n = m + 2; n <= nmax; n++, even = !even)
                {
                    real pa = q1, pb = q2;
                    q1 = xrec_tesseral(&s1, t1, anm[n], bnm[n]);
                    q2 = xrec_tesseral(&s2, t2, anm[n], bnm[n]);
                    real inm2 = (hm[n] * bnm[n]) * inm0 -
                                (anm[n] / (real)(n + 1)) *
                                ((u2 * u2) * pb - (u1 * u1) * pa);
                    inm0 = inm1;
                    inm1 = inm2;
                    cm[n - m] += inm2 * (even ? ap : am);
                    sm[n - m] += inm2 * (even ? bp : bm);
                }
            }
        }
        free(anm);
        free(bnm);
    }
    free(r);
    free(ri);
    free(dm);
    free(en);
    free(fn);
    free(gm);
    free(hm);
    free(col);
    free(geo);
    free(ps1);
    free(ps2);
    free(ips1);
    free(ips2);
    free(imm);
}

/* ------------------------------------------------------------------------ */
/* Quadrature grids                                                          */
/* ------------------------------------------------------------------------ */
/* Gauss--Legendre latitudes and weights, src/crd/crd_point_gl_chunk.c:122-173.
 * nlat = nmax + 1, north to south.  Returns 0 on success. */
int ORC(gl)(unsigned long nmax, real *lat, real *w)
{
    unsigned long L = nmax + 1;
    real Lf = (real)L;
    real c1 = Lf + (real)0.5;
    size_t nlat = L;
    size_t nnorth = (nlat + 1) / 2;
    int error = 0;
#pragma omp parallel for reduction(| : error)
    for (size_t i = 0; i < nnorth; i++)
    {
        real z = RCOS(RPI * ((real)(i + 1) - (real)0.25) / c1), z1, p1, p2, p3,
             pp;
        unsigned long it = 0;
        do
        {
            p1 = 1;
            p2 = 0;
            for (unsigned long j = 1; j <= L; j++)
            {
                p3 = p2;
                p2 = p1;
                p1 = ((real)(2 * j - 1) * z * p2 - (real)(j - 1) * p3) /
                     (real)j;
            }
            pp = Lf * (z * p1 - p2) / (z * z - (real)1);
            z1 = z;
            z -= p1 / pp;
            it++;
        } while ((RFABS(z - z1) > REPS) && (it < 1000));
        if (it >= 1000)
            error |= 1;
        size_t north = i, south = nlat - 1 - i;
        lat[south] = -RASIN(z);
        w[south] = (real)2 / (((real)1 - z * z) * pp * pp);
        if (nearly_equal(lat[south], 0, THRESHOLD))
            continue;
        lat[north] = -lat[south];
        w[north] = w[south];
    }
    return error;
}

/* Driscoll--Healy latitudes and weights, src/crd/crd_point_dh_lat_w_chunk.c
 * :49-92.  nlat = 2 (nmax + 1) for both DH1 and DH2. */
void ORC(dh)(unsigned long nmax, real *lat, real *w)
{
    unsigned long L = nmax + 1;
    real Lf = (real)L;
    real c = (real)2 / Lf;
    real M_PI_2L = RPI / ((real)2 * Lf);
    size_t nlat = 2 * L;
    size_t nnorth = nlat / 2 + 1;
#pragma omp parallel for
    for (size_t i = 0; i < nnorth; i++)
    {
        real clti = M_PI_2L * (real)i;
        size_t north = i, south = nlat - 1 - i + 1;
        lat[north] = RPI_2 - clti;
        real sclti = RSIN(clti);
        if (nmax == 0)
            w[north] = c * sclti;
        else
        {
            real s0 = 0, s1 = sclti, cc2 = (real)2 * RCOS(clti), s2;
            real wt = s1;
            for (unsigned long k = 1; k < L; k++)
            {
                s2 = cc2 * s1 - s0;
                s0 = s1;
                s1 = s2;
                s2 = cc2 * s1 - s0;
                wt += s2 / (real)(2 * k + 1);
                s0 = s1;
                s1 = s2;
            }
            w[north] = c * sclti * wt;
        }
        if (i == 0)
            continue;
        if (nearly_equal(lat[north], 0, THRESHOLD))
            continue;
        w[south] = w[north];
        lat[south] = -lat[north];
    }
}

#ifdef ORC_QUAD
/* Conversion helpers for the Python side: binary128 <-> (hi, lo) double
 * pairs and decimal strings. */
void orc_q_from_dd(const double *hi, const double *lo, real *out, size_t n)
{
    for (size_t i = 0; i < n; i++)
        out[i] = (real)hi[i] + (real)lo[i];
}

void orc_q_to_dd(const real *in, double *hi, double *lo, size_t n)
{
    for (size_t i = 0; i < n; i++)
    {
        double h = (double)in[i];
        hi[i] = h;
        lo[i] = (double)(in[i] - (real)h);
    }
}

int orc_q_from_str(const char *str, real *out)
{
    char *end = NULL;
    *out = strtoflt128(str, &end);
    return (end == str) ? 1 : 0;
}

/* Elementwise helpers so the Python driver can keep quad arithmetic in
 * quad: out = sum_k x[k] * y[k] over rows (used for longitude sums). */
void orc_q_lonsum(size_t nrow, size_t L, const real *a, const real *b,
                  size_t nlon, const real *lon, const real *scalep, real *f)
{
    real scale = *scalep;
#pragma omp parallel for
    for (size_t i = 0; i < nrow; i++)
        for (size_t j = 0; j < nlon; j++)
        {
            real acc = 0;
            for (size_t m = 0; m < L; m++)
            {
                real ml = (real)m * lon[j];
                acc += a[i * L + m] * RCOS(ml) + b[i * L + m] * RSIN(ml);
            }
            f[i * nlon + j] = scale * acc;
        }
}

void orc_q_sin(const real *x, real *y, size_t n)
{
    for (size_t i = 0; i < n; i++)
        y[i] = RSIN(x[i]);
}

void orc_q_cos(const real *x, real *y, size_t n)
{
    for (size_t i = 0; i < n; i++)
        y[i] = RCOS(x[i]);
}
#endif

#ifdef ORC_QUAD
/* Scalar/vector arithmetic in binary128 for the Python driver:
 * op 0 add, 1 sub, 2 mul, 3 div; b is a scalar when scalar_b != 0. */
void orc_q_arith(int op, const real *a, const real *b, real *out, size_t n,
                 int scalar_b)
{
    for (size_t i = 0; i < n; i++)
    {
        real bb = scalar_b ? b[0] : b[i];
        switch (op)
        {
        case 0: out[i] = a[i] + bb; break;
        case 1: out[i] = a[i] - bb; break;
        case 2: out[i] = a[i] * bb; break;
        default: out[i] = a[i] / bb; break;
        }
    }
}

void orc_q_from_double(const double *x, real *out, size_t n)
{
    for (size_t i = 0; i < n; i++)
        out[i] = (real)x[i];
}
#endif
