/* FFTW-API header of the oracle's FFT shim.
 *
 * Test infrastructure only: it lets CHarm's own sources (the reference CPU
 * implementation, compiled by oracle/build_ref.py into oracle/_ref/) build
 * and run without FFTW 3, which is an external library that is neither
 * vendored with CHarm nor installed here (CHarm's configure.ac:141,217,252
 * require it).  Nothing in the charm_b200 package uses it.
 *
 * Only the part of FFTW 3's documented interface that CHarm 0.4.9 calls is
 * declared (src/prec.h's FFTW()/FFTWC() macros; src/shs/shs_point_grd.c:417,
 * src/sha/sha_point.c:359,520,540, src/misc/misc_buildopt_version_fftw.c:21):
 * 1-D real-to-complex and complex-to-real plans with the new-array execute
 * functions, aligned allocation and the thread / clean-up calls, in double
 * (fftw_), single (fftwf_) and IEEE binary128 (fftwq_) precision.
 *
 * Semantics follow FFTW's manual: transforms are unnormalised; r2c computes
 * X_k = sum_j x_j exp(-2 pi i j k / n) for k = 0..n/2; c2r computes
 * x_j = sum_k X_k exp(+2 pi i j k / n) over the Hermitian extension of its
 * n/2 + 1 inputs, ignoring the imaginary parts of X_0 and (n even) X_n/2.
 * Execution with a plan is thread-safe; the implementation is in
 * fftw_shim.c (mixed-radix Stockham FFT, Bluestein for lengths with a prime
 * factor above 31).
 */
#ifndef ORACLE_FFTW_SHIM_FFTW3_H
#define ORACLE_FFTW_SHIM_FFTW3_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_ESTIMATE (1U << 6)

#define ORACLE_FFTW_DECLARE(X, R)                                             \
    typedef R X##_complex[2];                                                 \
    typedef struct X##_plan_s *X##_plan;                                      \
    void *X##_malloc(size_t n);                                               \
    void X##_free(void *p);                                                   \
    X##_plan X##_plan_dft_r2c_1d(int n, R *in, X##_complex *out,              \
                                 unsigned flags);                             \
    X##_plan X##_plan_dft_c2r_1d(int n, X##_complex *in, R *out,              \
                                 unsigned flags);                             \
    void X##_execute_dft_r2c(const X##_plan p, R *in, X##_complex *out);      \
    void X##_execute_dft_c2r(const X##_plan p, X##_complex *in, R *out);      \
    void X##_destroy_plan(X##_plan p);                                        \
    void X##_cleanup(void);                                                   \
    int X##_init_threads(void);                                               \
    void X##_plan_with_nthreads(int nthreads);                                \
    void X##_cleanup_threads(void);                                           \
    extern const char X##_version[];

ORACLE_FFTW_DECLARE(fftw, double)
ORACLE_FFTW_DECLARE(fftwf, float)
ORACLE_FFTW_DECLARE(fftwq, __float128)

#undef ORACLE_FFTW_DECLARE

#ifdef __cplusplus
}
#endif

#endif
