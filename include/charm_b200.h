/* charm_b200.h -- C interface of the B200 (sm_100a) implementation of CHarm's
 * point spherical-harmonic synthesis and analysis.
 *
 * This header mirrors, symbol for symbol, the part of CHarm 0.4.9's public C
 * API that the point-synthesis/analysis path needs, with the same struct
 * layouts (non-MPI build), enum values, argument meaning and error
 * behaviour, so that C code and PyHarm's ctypes bindings written against
 * CHarm link against libcharm.so from this project unchanged.  Each
 * declaration cites the CHarm header line it replaces.  All arrays are host
 * memory owned by the caller; the library stages them to the GPU internally.
 *
 * Threading: calls are serialised on one CUDA stream per process and device;
 * concurrent calls from several host threads must use distinct charm_err
 * objects and are executed one after another.
 */
#ifndef CHARM_B200_H
#define CHARM_B200_H

#include <stddef.h>
#include <limits.h>

#ifdef __cplusplus
/* C's _Bool and C++'s bool share size and representation on the supported
 * platforms, so the struct layouts are identical in both languages. */
#   ifndef _Bool
#       define _Bool bool
#   endif
extern "C"
{
#endif

#ifndef CHARM_EXTERN
#   define CHARM_EXTERN __attribute__((visibility("default")))
#endif
#ifndef CHARM_CDECL
#   define CHARM_CDECL
#endif

/* ------------------------------------------------------------------------- */
/* Errors: src/err/err.h.in:80-130 (enum), :159-222 (struct)                  */
/* ------------------------------------------------------------------------- */
enum
{
    CHARM_FAILURE = -1,
    CHARM_SUCCESS,
    CHARM_EMEM,
    CHARM_EFUNCARG,
    CHARM_EFILEIO,
    CHARM_EFFTWINIT,
    CHARM_EMPIPROCESS
};

#define CHARM_ERR_MAX_FILE 4096U    /* err.h.in:58 */
#define CHARM_ERR_MAX_FUNC 256U     /* err.h.in:65 */
#define CHARM_ERR_MAX_MSG 4096U     /* err.h.in:71 */
#define CHARM_ERR_MAX_LEVEL 10U     /* err.h.in:77 */
#define CHARM_ERR_MALLOC_FAILURE "Memory allocation failure."  /* :137 */

typedef struct
{
    size_t level;
    char **file;
    size_t *line;
    char **func;
    int code;
    char *msg;
    _Bool saturated;
    _Bool distributed;
} charm_err;

/* err.h.in:236-294 */
CHARM_EXTERN charm_err * CHARM_CDECL charm_err_init(void);
CHARM_EXTERN void CHARM_CDECL charm_err_free(charm_err *err);
CHARM_EXTERN void CHARM_CDECL charm_err_reset(charm_err *err);
CHARM_EXTERN void CHARM_CDECL charm_err_handler(charm_err *err,
                                                 _Bool terminate);
CHARM_EXTERN _Bool CHARM_CDECL charm_err_isempty(const charm_err *err);

/* ------------------------------------------------------------------------- */
/* Points: src/crd/crd.h.in:70-90 (enum), :125-332 (struct)                   */
/* ------------------------------------------------------------------------- */
enum
{
    CHARM_CRD_CELL_GRID = -2,
    CHARM_CRD_CELL_SCATTERED,
    CHARM_CRD_POINT_SCATTERED = 1,
    CHARM_CRD_POINT_GRID,
    CHARM_CRD_POINT_GRID_GL,
    CHARM_CRD_POINT_GRID_DH1,
    CHARM_CRD_POINT_GRID_DH2
};

typedef struct
{
    int type;
    size_t nlat;
    size_t nlon;
    size_t npoint;
    double *lat;
    double *lon;
    double *r;
    double *w;
    _Bool owner;
    _Bool distributed;
} charm_point;

/* crd.h.in:477-564 */
CHARM_EXTERN charm_point * CHARM_CDECL charm_crd_point_malloc(int type,
                                                              size_t nlat,
                                                              size_t nlon);
CHARM_EXTERN charm_point * CHARM_CDECL charm_crd_point_calloc(int type,
                                                              size_t nlat,
                                                              size_t nlon);
CHARM_EXTERN charm_point * CHARM_CDECL charm_crd_point_init(int type,
                                                            size_t nlat,
                                                            size_t nlon,
                                                            double *lat,
                                                            double *lon,
                                                            double *r);
CHARM_EXTERN void CHARM_CDECL charm_crd_point_free(charm_point *pnt);
/* crd.h.in:615-686: quadrature grids (nodes and weights computed on the
 * GPU) */
CHARM_EXTERN charm_point * CHARM_CDECL charm_crd_point_gl(unsigned long nmax,
                                                          double r);
CHARM_EXTERN charm_point * CHARM_CDECL charm_crd_point_dh1(unsigned long nmax,
                                                           double r);
CHARM_EXTERN charm_point * CHARM_CDECL charm_crd_point_dh2(unsigned long nmax,
                                                           double r);
/* crd.h.in:700-760: shapes of the quadrature grids */
CHARM_EXTERN void CHARM_CDECL charm_crd_point_gl_shape(unsigned long nmax,
                                                       size_t *nlat,
                                                       size_t *nlon);
CHARM_EXTERN void CHARM_CDECL charm_crd_point_dh1_shape(unsigned long nmax,
                                                        size_t *nlat,
                                                        size_t *nlon);
CHARM_EXTERN void CHARM_CDECL charm_crd_point_dh2_shape(unsigned long nmax,
                                                        size_t *nlat,
                                                        size_t *nlon);

/* Cells: src/crd/crd.h.in:339-409 (struct), :702-846 (functions).
 * Block-mean values over latitude-longitude cells: a grid (latmin, latmax
 * and r per cell row, lonmin and lonmax per cell column, f[i * nlon + j])
 * or scattered cells (nlat == nlon == ncell, all five arrays per cell). */
typedef struct
{
    int type;
    size_t nlat;
    size_t nlon;
    size_t ncell;
    double *latmin;
    double *latmax;
    double *lonmin;
    double *lonmax;
    double *r;
    _Bool owner;
} charm_cell;

/* crd.h.in:761-846 (src/crd/crd_cell_alloc.c, crd_cell_init.c,
 * crd_cell_free.c): NULL for an unsupported type, for scattered cells with
 * nlat != nlon, or when memory runs out */
CHARM_EXTERN charm_cell * CHARM_CDECL charm_crd_cell_malloc(int type,
                                                            size_t nlat,
                                                            size_t nlon);
CHARM_EXTERN charm_cell * CHARM_CDECL charm_crd_cell_calloc(int type,
                                                            size_t nlat,
                                                            size_t nlon);
CHARM_EXTERN charm_cell * CHARM_CDECL charm_crd_cell_init(int type,
                                                          size_t nlat,
                                                          size_t nlon,
                                                          double *latmin,
                                                          double *latmax,
                                                          double *lonmin,
                                                          double *lonmax,
                                                          double *r);
CHARM_EXTERN void CHARM_CDECL charm_crd_cell_free(charm_cell *cell);

/* ------------------------------------------------------------------------- */
/* Spherical harmonic coefficients: src/shc/shc.h.in:139-381 (struct)         */
/* ------------------------------------------------------------------------- */
typedef struct
{
    unsigned long nmax;
    double mu;
    double r;
    size_t nc;
    size_t ns;
    double **c;
    double **s;
    _Bool owner;
    _Bool distributed;
} charm_shc;

/* shc.h.in:423-602 */
CHARM_EXTERN charm_shc * CHARM_CDECL charm_shc_malloc(unsigned long nmax,
                                                      double mu, double r);
CHARM_EXTERN charm_shc * CHARM_CDECL charm_shc_calloc(unsigned long nmax,
                                                      double mu, double r);
CHARM_EXTERN charm_shc * CHARM_CDECL charm_shc_init(unsigned long nmax,
                                                    double mu, double r,
                                                    double *c, double *s);
CHARM_EXTERN void CHARM_CDECL charm_shc_free(charm_shc *shcs);

/* Coefficient files in CHarm's binary format: src/shc/shc.h.in:98-108
 * (constants), :628-722 (charm_shc_read_bin), the writer's counterpart
 * (src/shc/shc_write_bin.c).  The file holds nmax (unsigned long), mu, r
 * (double) and the order-major columns of C, then of S, column m with
 * nmax + 1 - m values.  nmax = CHARM_SHC_NMAX_MODEL with shcs = NULL only
 * reads the file's maximum degree, which every successful call returns;
 * CHARM_SHC_NMAX_ERROR on error. */
#define CHARM_SHC_NMAX_MODEL (ULONG_MAX - 1UL)
#define CHARM_SHC_NMAX_ERROR (ULONG_MAX)
CHARM_EXTERN unsigned long CHARM_CDECL charm_shc_read_bin(const char *pathname,
                                                          unsigned long nmax,
                                                          charm_shc *shcs,
                                                          charm_err *err);
CHARM_EXTERN void CHARM_CDECL charm_shc_write_bin(const charm_shc *shcs,
                                                  unsigned long nmax,
                                                  const char *pathname,
                                                  charm_err *err);

/* ------------------------------------------------------------------------- */
/* Synthesis: src/shs/shs.h.in:168-173, :239-244, :344-349, :428-435          */
/* ------------------------------------------------------------------------- */
CHARM_EXTERN void CHARM_CDECL charm_shs_point(const charm_point *pnt,
                                              const charm_shc *shcs,
                                              unsigned long nmax,
                                              double *f,
                                              charm_err *err);
CHARM_EXTERN void CHARM_CDECL charm_shs_point_grad1(const charm_point *pnt,
                                                    const charm_shc *shcs,
                                                    unsigned long nmax,
                                                    double **f,
                                                    charm_err *err);
CHARM_EXTERN void CHARM_CDECL charm_shs_point_grad2(const charm_point *pnt,
                                                    const charm_shc *shcs,
                                                    unsigned long nmax,
                                                    double **f,
                                                    charm_err *err);
CHARM_EXTERN void CHARM_CDECL charm_shs_point_guru(const charm_point *pnt,
                                                   const charm_shc *shcs,
                                                   unsigned long nmax,
                                                   unsigned dr,
                                                   unsigned dlat,
                                                   unsigned dlon,
                                                   double *f,
                                                   charm_err *err);

/* Block means in cells: src/shs/shs.h.in:603-609 (src/shs/shs_cell.c).  A
 * grid of cells takes the FFT along its rows when its cells cover the
 * parallels from 0 to 2 pi with (nlon - 1) / 2 >= nmax, else sums at the
 * cell centres; scattered cells need nlat == nlon. */
CHARM_EXTERN void CHARM_CDECL charm_shs_cell(const charm_cell *cell,
                                             const charm_shc *shcs,
                                             unsigned long nmax,
                                             double *f,
                                             charm_err *err);

/* ------------------------------------------------------------------------- */
/* Analysis: src/sha/sha.h.in:164-169                                         */
/* ------------------------------------------------------------------------- */
CHARM_EXTERN void CHARM_CDECL charm_sha_point(const charm_point *pnt,
                                              const double *f,
                                              unsigned long nmax,
                                              charm_shc *shcs,
                                              charm_err *err);

/* Analysis of block means on a cell grid covering the sphere:
 * src/sha/sha.h.in:50-59 (method), :315-320 (src/sha/sha_cell.c).  The
 * only method is the approximate quadrature CHARM_SHA_CELL_AQ. */
enum
{
    CHARM_SHA_CELL_AQ
};
CHARM_EXTERN void CHARM_CDECL charm_sha_cell(const charm_cell *cell,
                                             const double *f,
                                             unsigned long nmax,
                                             int method,
                                             charm_shc *shcs,
                                             charm_err *err);

/* ------------------------------------------------------------------------- */
/* Global spectral gravity forward modelling: src/gfm/gfm.h.in:223-320        */
/* (src/gfm/gfm_sgfm.c).  Masses between the sphere of radius                */
/* shape_radius_ref and the surface given by shape_shcs, with a density      */
/* polynomial in the radius whose coefficients density_shcs[0..order] vary   */
/* laterally (3d), one lateral density (lateral) or a constant (const); the  */
/* shape-density functions of topography powers shape_power_min..max are    */
/* synthesised, multiplied and analysed on Gauss--Legendre grids on the GPU. */
/* The optional exports of partial coefficients take the "bin" format.      */
/* ------------------------------------------------------------------------- */
CHARM_EXTERN void CHARM_CDECL charm_gfm_global_density_3d(
    const charm_shc *shape_shcs, unsigned long shape_nmax,
    double shape_radius_ref, charm_shc **density_shcs,
    unsigned long *density_nmax, unsigned density_order, double grav_const,
    double mass, unsigned shape_power_min, unsigned shape_power_max,
    unsigned long potential_shcs_nmax, const char *shape_density_shcs_path,
    const char *potential_shcs_path, const char *shcs_file_format,
    charm_shc *potential_shcs, charm_err *err);
CHARM_EXTERN void CHARM_CDECL charm_gfm_global_density_lateral(
    const charm_shc *shape_shcs, unsigned long shape_nmax,
    double shape_radius_ref, charm_shc *density_shcs,
    unsigned long density_nmax, double grav_const, double mass,
    unsigned shape_power_min, unsigned shape_power_max,
    unsigned long potential_shcs_nmax, const char *shape_density_shcs_path,
    const char *potential_shcs_path, const char *shcs_file_format,
    charm_shc *potential_shcs, charm_err *err);
CHARM_EXTERN void CHARM_CDECL charm_gfm_global_density_const(
    const charm_shc *shape_shcs, unsigned long shape_nmax,
    double shape_radius_ref, double density, double grav_const, double mass,
    unsigned shape_power_min, unsigned shape_power_max,
    unsigned long potential_shcs_nmax, const char *shape_shcs_path,
    const char *potential_shcs_path, const char *shcs_file_format,
    charm_shc *potential_shcs, charm_err *err);

/* ------------------------------------------------------------------------- */
/* Runtime globals: src/glob/glob.h.in:66-241 (values glob.c:16-23)            */
/* ------------------------------------------------------------------------- */
CHARM_EXTERN extern double charm_glob_threshold;
CHARM_EXTERN extern double charm_glob_threshold2;
CHARM_EXTERN extern unsigned long charm_glob_polar_optimization_a1;
CHARM_EXTERN extern double charm_glob_polar_optimization_a2;

/* ------------------------------------------------------------------------- */
/* Extensions of this library (no counterpart in CHarm's API).               */
/* ------------------------------------------------------------------------- */
/* Synthesis with the coefficient triangles and the output in device memory:
 * d_c, d_s hold order-major triangles of degree shc_nmax (CHarm's layout of
 * charm_shc.c[0]), d_f receives [npar][npoint] values (npar = 1, 3 or 6 as
 * for charm_shs_point, charm_shs_point_grad1/2; grad outputs in CHarm's
 * computation order l, r, p and ll, lr, lp, rr, rp, pp).  kgrad 0 with
 * (dr, dlat, dlon) selects a single quantity as charm_shs_point_guru.  pnt
 * stays in host memory.  Errors as charm_shs_point. */
CHARM_EXTERN void CHARM_CDECL charm_b200_shs_point_dev(
    const charm_point *pnt, unsigned long shc_nmax, double mu, double r,
    const double *d_c, const double *d_s, unsigned long nmax, int kgrad,
    unsigned dr, unsigned dlat, unsigned dlon, double *d_f, charm_err *err);

/* Cell synthesis and analysis with the coefficient triangles, the block
 * means and the output in device memory (layouts as for
 * charm_b200_shs_point_dev and charm_b200_sha_point_dev); cell stays in
 * host memory.  Checks and errors as charm_shs_cell / charm_sha_cell. */
CHARM_EXTERN void CHARM_CDECL charm_b200_shs_cell_dev(
    const charm_cell *cell, unsigned long shc_nmax, double mu, double r,
    const double *d_c, const double *d_s, unsigned long nmax, double *d_f,
    charm_err *err);
CHARM_EXTERN void CHARM_CDECL charm_b200_sha_cell_dev(
    const charm_cell *cell, const double *d_f, unsigned long nmax, double mu,
    double r, unsigned long shc_nmax, double *d_c, double *d_s,
    charm_err *err);

/* A binary coefficient file (charm_shc_read_bin's format) streamed into
 * device triangles d_c, d_s of degree shc_nmax (CHarm's order-major layout,
 * zero above nmax): the columns are read in chunks into two page-locked
 * buffers, each chunk copied to the device while the next one is read.
 * *mu and *r receive the file's values.  Returns the file's maximum degree,
 * or CHARM_SHC_NMAX_ERROR with err set (file I/O: CHARM_EFILEIO; nmax above
 * the file's or above shc_nmax: CHARM_EFUNCARG). */
CHARM_EXTERN unsigned long CHARM_CDECL charm_b200_shc_read_bin_dev(
    const char *pathname, unsigned long nmax, unsigned long shc_nmax,
    double *d_c, double *d_s, double *mu, double *r, charm_err *err);

/* Analysis with the grid values (d_f, nlat x nlon) and the output triangles
 * (degree shc_nmax, zero above nmax) in device memory; the coefficients
 * refer to (mu, r) as charm_sha_point's shcs would. */
CHARM_EXTERN void CHARM_CDECL charm_b200_sha_point_dev(
    const charm_point *pnt, const double *d_f, unsigned long nmax, double mu,
    double r, unsigned long shc_nmax, double *d_c, double *d_s,
    charm_err *err);

/* Batched synthesis of nsets coefficient sets on one grid (no counterpart
 * in CHarm, which synthesises one set per charm_shs_point call): set j has
 * device triangles d_c[j], d_s[j] of degree shc_nmax[j] (order-major),
 * maximum degree nmax[j] and scaling mu[j]; all share the reference radius
 * r.  kgrad 0: the potential; 1: grad1 (x, y, z); 2: grad2 (xx, xy, xz, yy,
 * yz, zz); 3: all ten quantities in that order.  d_f[j] (device) receives
 * ncomp x nlat x nlon doubles, components in that order (CHarm's order after
 * its pointer reordering, src/shs/shs_point_gradn.c:133-165).  The grid
 * needs FFT longitudes (0, 2 pi / nlon, ..., nlon > 2 max nmax); every work
 * item (set, order, latitude tile) of a derivative kind runs in one launch. */
CHARM_EXTERN void CHARM_CDECL charm_b200_shs_point_batch_dev(
    const charm_point *pnt, size_t nsets, const unsigned long *nmax,
    const unsigned long *shc_nmax, const double *mu, double r,
    const double *const *d_c, const double *const *d_s, int kgrad,
    double *const *d_f, charm_err *err);

/* A batched synthesis captured into a CUDA graph (no counterpart in CHarm):
 * split_precision 0 captures charm_b200_shs_point_batch_dev, 1 captures
 * charm_b200_shs_point_batch_i8_dev, with these arguments.  The
 * call runs once plainly (checks, tables, buffers, tuned choices), then once
 * under stream capture; returns the graph's handle, or NULL with err set.
 * charm_b200_graph_launch replays the whole call (every launch, copy and
 * row transform of it) on the same device buffers, whose contents the
 * caller may change between launches, and reports the kernels' status;
 * charm_b200_graph_free releases the graph.  The graph also reads the
 * library's own cached buffers and tables by address: a launch after a
 * call that reallocated or rewrote them (larger sizes, another maximum
 * degree) is refused with CHARM_EFUNCARG, and the graph must be captured
 * again. */
CHARM_EXTERN void *CHARM_CDECL charm_b200_shs_point_batch_graph(
    const charm_point *pnt, size_t nsets, const unsigned long *nmax,
    const unsigned long *shc_nmax, const double *mu, double r,
    const double *const *d_c, const double *const *d_s, int kgrad,
    double *const *d_f, int split_precision, charm_err *err);
CHARM_EXTERN void CHARM_CDECL charm_b200_graph_launch(void *graph,
                                                      charm_err *err);
CHARM_EXTERN void CHARM_CDECL charm_b200_graph_free(void *graph);

/* The synthesis kernel's autotuner (no counterpart in CHarm): on the first
 * call of a problem shape (derivative kind, nmax >= 256, latitude pairs, on
 * or off the reference sphere) the latitude pairs per lane of the grid
 * synthesis are chosen by timing every candidate once; the results do not
 * depend on the choice.  CHARM_B200_AUTOTUNE=0 keeps the built-in choice.
 * Copies up to n - 1 characters of a report of the choices so far (one line
 * per shape: chosen K, measured ms of each candidate) into buf and returns
 * the report's full length. */
CHARM_EXTERN size_t CHARM_CDECL charm_b200_autotune_report(char *buf,
                                                            size_t n);

/* charm_b200_shs_point_batch_dev with the degree sums of every (order,
 * 128-latitude tile) on the tensor cores for up to 16 sets at once (no
 * counterpart in CHarm): the Legendre values and the coefficients become
 * 54-bit fixed-point integers, cut into seven 8-bit digits whose products
 * are summed exactly in INT32 (tcgen05 kind::i8) and recombined in FP64.
 * Agrees with the FP64 path to a relative RMS of about 1e-15 per set.
 * kgrad as charm_b200_shs_point_batch_dev: 0 the potential; 1, 2 and 3
 * (grad1, grad2, all ten quantities) contract the same Legendre values
 * against five coefficient families per set (C_n, n C_n, n (n + 1) C_n,
 * e_n+1 C_n+1, n e_n+1 C_n+1 and the same of S), from which the derivative
 * terms follow by the per-degree relations of CHarm's kernels
 * (src/shs/shs_point_kernel.c:1639-1946), 3 sets per launch.  The polar
 * optimisation must be off. */
CHARM_EXTERN void CHARM_CDECL charm_b200_shs_point_batch_i8_dev(
    const charm_point *pnt, size_t nsets, const unsigned long *nmax,
    const unsigned long *shc_nmax, const double *mu, double r,
    const double *const *d_c, const double *const *d_s, int kgrad,
    double *const *d_f, charm_err *err);

/* Single-precision mode of the device-resident potential synthesis and
 * analysis: the Legendre recurrence and sums in FP32 (as CHarm's float
 * build, charmf_shs_point / charmf_sha_point, does them), the longitude
 * transforms in FP64; float coefficient triangles (degree shc_nmax,
 * order-major) and a float grid [nlat][nlon] in device memory.  Grids whose
 * longitudes are 0, 2 pi / nlon, ... with even nlon (the quadrature grids
 * and such user grids), every row at the coefficients' radius r;
 * anything else is rejected with CHARM_EFUNCARG. */
CHARM_EXTERN void CHARM_CDECL charm_b200_shs_point_dev_f32(
    const charm_point *pnt, unsigned long shc_nmax, double mu, double r,
    const float *d_c, const float *d_s, unsigned long nmax, float *d_f,
    charm_err *err);
CHARM_EXTERN void CHARM_CDECL charm_b200_sha_point_dev_f32(
    const charm_point *pnt, const float *d_f, unsigned long nmax, double mu,
    double r, unsigned long shc_nmax, float *d_c, float *d_s,
    charm_err *err);

/* Adjoint of charm_shs_point on scattered points with respect to the
 * coefficients (no counterpart in CHarm, which has no transpose routine;
 * the forward it transposes is src/shs/shs_point_sctr.c:86-728): for the
 * model (shcs->mu, shcs->r) and weights g[npoint] it overwrites shcs->c and
 * shcs->s with
 *     C_nm = (mu / r) sum_i g_i (r / r_i)^(n+1) P_nm(sin lat_i) cos(m lon_i)
 * (sin for S_nm), degrees above nmax zero, i.e. the gradient of
 * sum_i g_i f_i with f = charm_shs_point(pnt, shcs, nmax).  pnt must hold
 * scattered points (CHARM_CRD_POINT_SCATTERED). */
CHARM_EXTERN void CHARM_CDECL charm_b200_shs_point_sctr_adjoint(
    const charm_point *pnt, const double *g, unsigned long nmax,
    charm_shc *shcs, charm_err *err);

/* Same with the weights d_g[npoint] and the output triangles d_c, d_s
 * (degree shc_nmax, order-major) in device memory; mu, r describe the
 * model as shcs->mu, shcs->r would. */
CHARM_EXTERN void CHARM_CDECL charm_b200_shs_point_sctr_adjoint_dev(
    const charm_point *pnt, const double *d_g, unsigned long nmax, double mu,
    double r, unsigned long shc_nmax, double *d_c, double *d_s,
    charm_err *err);

/* Largest degree and size of the fixed device scratch of
 * charm_b200_sha_point_dev_static. */
#define CHARM_B200_STATIC_NMAX 511
#define CHARM_B200_STATIC_SCRATCH_BYTES 33554432

/* charm_b200_sha_point_dev that allocates nothing: no cudaMalloc, cudaFree,
 * pinned or heap memory and no allocating library routine.
 * No counterpart in CHarm; it serves callers that cannot allocate during
 * the call -- device memory owned by another allocator (a framework's
 * caching pool), or a loop that must not synchronise the device as
 * cudaMalloc / cudaFree do.  Every temporary lives in one file-scope static
 * device array of CHARM_B200_STATIC_SCRATCH_BYTES (32 MiB) whose address is
 * taken once per device with cudaGetSymbolAddress.  Limits: GL / DH grids,
 * nmax <= CHARM_B200_STATIC_NMAX, at most 8192 latitudes, an even number
 * of longitudes whose shared-memory transform exists (half length >= 8,
 * transform length <= 9216), d_f on a 16-byte boundary, and the scratch
 * large enough for the grid and nmax; anything else is rejected with
 * CHARM_EFUNCARG and a message naming the limit.  The library serialises
 * these calls on its stream and returns after the stream is idle; kernels
 * of calls that overlap on the GPU (another process's context aside) would
 * race on the scratch.  The host-side staging of the call (latitude
 * geometry and table sources, fixed arrays in engine.cpp) is one
 * process-wide object as well: call it from one host thread at a time.
 * Like the rest of the library it serves one device per process.  The
 * first call on a device performs the set-up
 * (symbol address, kernel attributes, recurrence and transform tables) and
 * should precede any stream capture.  Only the scratch's status and
 * work-counter words must start at zero; each call clears them. */
CHARM_EXTERN void CHARM_CDECL charm_b200_sha_point_dev_static(
    const charm_point *pnt, const double *d_f, unsigned long nmax, double mu,
    double r, unsigned long shc_nmax, double *d_c, double *d_s,
    charm_err *err);

/* ------------------------------------------------------------------------
 * Single-precision ABI: the entry points of CHarm's float build
 * (src/prec.h:84-86 with @P@ = f, RDT = float): the same structures with
 * float arrays, the same functions with the prefix charmf_.  The transforms
 * run on the single-precision kernels where they serve the call (the
 * potential on grids with FFT longitudes, nmax <= 2200, every row at the
 * coefficients' radius); every other call (gradients, scattered points,
 * higher degrees) runs the FP64 path and rounds its results to float.  The
 * comparison thresholds of a charmf_ call are charmf_glob_threshold and
 * charmf_glob_threshold2 (src/glob/glob.c with EPS = FLT_EPSILON).
 * ------------------------------------------------------------------------ */
/* err.h.in: the error structure has no precision-dependent member */
typedef charm_err charmf_err;

/* crd.h.in:125-300 with RDT = float */
typedef struct
{
    int type;
    size_t nlat;
    size_t nlon;
    size_t npoint;
    float *lat;
    float *lon;
    float *r;
    float *w;
    _Bool owner;
    _Bool distributed;
} charmf_point;

/* shc.h.in:139-381 with RDT = float */
typedef struct
{
    unsigned long nmax;
    float mu;
    float r;
    size_t nc;
    size_t ns;
    float **c;
    float **s;
    _Bool owner;
    _Bool distributed;
} charmf_shc;

/* glob.h.in (float build) */
CHARM_EXTERN extern float charmf_glob_threshold;
CHARM_EXTERN extern float charmf_glob_threshold2;
CHARM_EXTERN extern unsigned long charmf_glob_polar_optimization_a1;
CHARM_EXTERN extern float charmf_glob_polar_optimization_a2;

/* err.h.in:236-294 */
CHARM_EXTERN charmf_err *CHARM_CDECL charmf_err_init(void);
CHARM_EXTERN void CHARM_CDECL charmf_err_free(charmf_err *err);
CHARM_EXTERN void CHARM_CDECL charmf_err_reset(charmf_err *err);
CHARM_EXTERN void CHARM_CDECL charmf_err_handler(charmf_err *err,
                                                  _Bool terminate);
CHARM_EXTERN _Bool CHARM_CDECL charmf_err_isempty(const charmf_err *err);

/* crd.h.in:477-760 */
CHARM_EXTERN charmf_point *CHARM_CDECL charmf_crd_point_malloc(int type,
                                                               size_t nlat,
                                                               size_t nlon);
CHARM_EXTERN charmf_point *CHARM_CDECL charmf_crd_point_calloc(int type,
                                                               size_t nlat,
                                                               size_t nlon);
CHARM_EXTERN charmf_point *CHARM_CDECL charmf_crd_point_init(
    int type, size_t nlat, size_t nlon, float *lat, float *lon, float *r);
CHARM_EXTERN void CHARM_CDECL charmf_crd_point_free(charmf_point *pnt);
CHARM_EXTERN charmf_point *CHARM_CDECL charmf_crd_point_gl(unsigned long nmax,
                                                           float r);
CHARM_EXTERN charmf_point *CHARM_CDECL charmf_crd_point_dh1(unsigned long nmax,
                                                            float r);
CHARM_EXTERN charmf_point *CHARM_CDECL charmf_crd_point_dh2(unsigned long nmax,
                                                            float r);
CHARM_EXTERN void CHARM_CDECL charmf_crd_point_gl_shape(unsigned long nmax,
                                                        size_t *nlat,
                                                        size_t *nlon);
CHARM_EXTERN void CHARM_CDECL charmf_crd_point_dh1_shape(unsigned long nmax,
                                                         size_t *nlat,
                                                         size_t *nlon);
CHARM_EXTERN void CHARM_CDECL charmf_crd_point_dh2_shape(unsigned long nmax,
                                                         size_t *nlat,
                                                         size_t *nlon);

/* shc.h.in:423-602 */
CHARM_EXTERN charmf_shc *CHARM_CDECL charmf_shc_malloc(unsigned long nmax,
                                                       float mu, float r);
CHARM_EXTERN charmf_shc *CHARM_CDECL charmf_shc_calloc(unsigned long nmax,
                                                       float mu, float r);
CHARM_EXTERN charmf_shc *CHARM_CDECL charmf_shc_init(unsigned long nmax,
                                                     float mu, float r,
                                                     float *c, float *s);
CHARM_EXTERN void CHARM_CDECL charmf_shc_free(charmf_shc *shcs);

/* shs.h.in:168-173, 239-244, 344-349, 428-435; sha.h.in:164-169 */
CHARM_EXTERN void CHARM_CDECL charmf_shs_point(const charmf_point *pnt,
                                               const charmf_shc *shcs,
                                               unsigned long nmax, float *f,
                                               charmf_err *err);
CHARM_EXTERN void CHARM_CDECL charmf_shs_point_grad1(const charmf_point *pnt,
                                                     const charmf_shc *shcs,
                                                     unsigned long nmax,
                                                     float **f,
                                                     charmf_err *err);
CHARM_EXTERN void CHARM_CDECL charmf_shs_point_grad2(const charmf_point *pnt,
                                                     const charmf_shc *shcs,
                                                     unsigned long nmax,
                                                     float **f,
                                                     charmf_err *err);
CHARM_EXTERN void CHARM_CDECL charmf_shs_point_guru(
    const charmf_point *pnt, const charmf_shc *shcs, unsigned long nmax,
    unsigned dr, unsigned dlat, unsigned dlon, float *f, charmf_err *err);
CHARM_EXTERN void CHARM_CDECL charmf_sha_point(const charmf_point *pnt,
                                               const float *f,
                                               unsigned long nmax,
                                               charmf_shc *shcs,
                                               charmf_err *err);

/* Latitude-band sharding of one transform over several GPUs (one process
 * per GPU; the reference's MPI build distributes latitude chunks, src/mpi,
 * and sums the coefficients, src/shc/shc_block_set_coeffs.c:80-86; no
 * single-call counterpart in CHarm).  charm_b200_grid_pairs lists the
 * latitude pairs of a grid as the transforms group them (row_n[p] and its
 * mirror row row_s[p], -1 when it has none; at most cap entries written)
 * and returns their number.  charm_b200_sha_point_dev_band is
 * charm_b200_sha_point_dev restricted to the pairs [pair0, pair1): the
 * contribution of those rows of d_f (the other rows are not read) to the
 * coefficients, so that the bands of a partition of the pairs sum to the
 * whole analysis. */
CHARM_EXTERN int CHARM_CDECL charm_b200_grid_pairs(const charm_point *pnt,
                                                   int *row_n, int *row_s,
                                                   int cap);
CHARM_EXTERN void CHARM_CDECL charm_b200_sha_point_dev_band(
    const charm_point *pnt, const double *d_f, unsigned long nmax, double mu,
    double r, unsigned long shc_nmax, int pair0, int pair1, double *d_c,
    double *d_s, charm_err *err);

/* The CUDA stream the library runs on (a cudaStream_t), or NULL when no
 * usable device is present. */
CHARM_EXTERN void *CHARM_CDECL charm_b200_stream(void);

/* Per-kernel event timing: enable (resets the counters) or disable. */
CHARM_EXTERN void CHARM_CDECL charm_b200_timing(int enable);

/* Reads the accumulated timers: ms[i], count[i] for i < n (0 grid synthesis
 * kernel, 1 grid analysis kernel, 2 scattered synthesis kernel, 3 row
 * transforms, 4 direct longitude sums, 5 preparation kernels, 6 tables) and
 * the number of this library's kernel launches and of library (non-charm)
 * kernel launches since enabled; the latter stays 0, since every transform
 * runs this library's own kernels.
 * Returns the number of timers available. */
CHARM_EXTERN int CHARM_CDECL charm_b200_timing_read(
    double *ms, unsigned long long *count, int n,
    unsigned long long *kernel_launches, unsigned long long *fft_execs);

/* Measured FP64 fused-multiply-add throughput of the current device,
 * TFLOP/s (an FMA counted as two flops); negative on error. */
CHARM_EXTERN double CHARM_CDECL charm_b200_fp64_peak_tflops(void);

#ifdef __cplusplus
}
#endif

#endif
