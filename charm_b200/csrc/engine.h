// Host runtime of charm_b200: device context, buffer and plan caches, and
// the call flows of grid synthesis, scattered synthesis and grid analysis.
// Used by capi.cpp; independent of any framework (plain CUDA runtime).
#pragma once

#include <string>

#include "../../include/charm_b200.h"

namespace cb
{

// Per-kernel timers (indices of charm_b200_timing_read).
enum
{
    TIMER_SHS = 0,   // grid synthesis Legendre kernel
    TIMER_SHA = 1,   // grid analysis Legendre kernel
    TIMER_SCTR = 2,  // scattered synthesis kernel
    TIMER_FFT = 3,   // row transforms along the parallels (rfft.cu)
    TIMER_LON = 4,   // direct longitude sums (non-FFT grids)
    TIMER_PREP = 5,  // seeds, interleave, reductions, nodes
    TIMER_TABLES = 6,
    TIMER_COUNT = 7
};

// Result of an engine call: CHARM_SUCCESS or a CHarm error code with a
// message.
struct Status
{
    int code = CHARM_SUCCESS;
    std::string msg;
    bool ok() const { return code == CHARM_SUCCESS; }
};

// Synthesis at grids or scattered points.  kgrad: 0 single quantity
// (dr, dlat, dlon), 1 full grad1, 2 full grad2.  f[q] receive the output
// components in CHarm's computation order (the caller reorders pointers).
Status shs_point(const charm_point *pnt, const charm_shc *shcs,
                 unsigned long nmax, int kgrad, int dr, int dlat, int dlon,
                 double **f);

// Same with the coefficient triangles (degree shc_nmax) and the output
// ([npar][npoint]) in device memory.
Status shs_point_dev(const charm_point *pnt, unsigned long shc_nmax,
                     double mu, double r, const double *d_c,
                     const double *d_s, unsigned long nmax, int kgrad, int dr,
                     int dlat, int dlon, double *d_f);

// Analysis on GL/DH grids; overwrites shcs->c, shcs->s.
Status sha_point(const charm_point *pnt, const double *f, unsigned long nmax,
                 charm_shc *shcs);

// Same with the grid values and the output triangles (degree shc_nmax) in
// device memory.
Status sha_point_dev(const charm_point *pnt, const double *d_f,
                     unsigned long nmax, double mu, double r,
                     unsigned long shc_nmax, double *d_c, double *d_s);

// One latitude band of a sharded analysis: the contribution of the
// latitude pairs [pair0, pair1) of the grid's pairing to the coefficients
// (linear in the grid, so the bands' outputs sum to sha_point_dev's).
// Block means in cells (cell.cu): host arrays (charm_shs_cell,
// charm_sha_cell) or device arrays.  Callers have done CHarm's checks that
// precede the dispatch (nmax against shcs->nmax, zero cells, cell type).
Status shs_cell(const charm_cell *cell, const charm_shc *shcs,
                unsigned long nmax, double *f);
Status shs_cell_dev(const charm_cell *cell, unsigned long shc_nmax,
                    double mu, double r, const double *d_c, const double *d_s,
                    unsigned long nmax, double *d_f);
Status sha_cell(const charm_cell *cell, const double *f, unsigned long nmax,
                charm_shc *shcs);
Status sha_cell_dev(const charm_cell *cell, const double *d_f,
                    unsigned long nmax, double mu, double r,
                    unsigned long shc_nmax, double *d_c, double *d_s);
// Global spectral gravity forward modelling (src/gfm/gfm_sgfm.c,
// SGFM_GLOBAL): density null for a constant density rho; the callers have
// made CHarm's checks.  Exports go to binary coefficient files.
struct GfmArgs
{
    const charm_shc *shape;
    unsigned long shape_nmax;
    double R;
    charm_shc *const *density;
    const unsigned long *density_nmax;
    unsigned density_order;
    double rho;
    double G, mass;
    unsigned pmin, pmax;
    unsigned long nmax_pot;
    const char *hro_path, *pot_path;
    charm_shc *pot;
};
Status gfm_global(const GfmArgs &g);
// A coefficient file in CHarm's binary format streamed into device
// triangles of degree shc_nmax (charm_b200_shc_read_bin_dev).
Status shc_read_bin_dev(const char *path, unsigned long nmax,
                        unsigned long shc_nmax, double *d_c, double *d_s,
                        double *mu, double *r, unsigned long *nmax_file);
Status sha_point_dev_band(const charm_point *pnt, const double *d_f,
                          unsigned long nmax, double mu, double r,
                          unsigned long shc_nmax, int pair0, int pair1,
                          double *d_c, double *d_s);
// The latitude pairs of a grid as the transforms group them: row_n[p] and
// the mirror row row_s[p] (-1: none); returns their number (fills at most
// cap entries).
int grid_pair_rows(const charm_point *pnt, int *row_n, int *row_s, int cap);

// Batched synthesis of nsets coefficient sets (degree shc_nmax[j], maximum
// degree nmax[j], scaling mu[j], common reference radius r; device
// triangles d_c[j], d_s[j]) on one grid with FFT longitudes; kgrad 0, 1, 2
// or 3 (potential, grad1 and grad2: ten quantities); d_f[j] receives
// ncomp x nlat x nlon doubles in CHarm's component order.
Status shs_point_batch_dev(const charm_point *pnt, size_t nsets,
                           const unsigned long *nmax,
                           const unsigned long *shc_nmax, const double *mu,
                           double r, const double *const *d_c,
                           const double *const *d_s, int kgrad,
                           double *const *d_f);
// A batched synthesis call (FP64 batch or, split != 0, the split-precision
// one) captured into a CUDA graph; launch replays it on the same device
// buffers and checks the kernels' status word.
Status batch_graph_create(const charm_point *pnt, size_t nsets,
                          const unsigned long *nmax,
                          const unsigned long *shc_nmax, const double *mu,
                          double r, const double *const *d_c,
                          const double *const *d_s, int kgrad,
                          double *const *d_f, int split, void **out);
Status batch_graph_launch(void *graph);
void batch_graph_free(void *graph);

// The autotuner's choices so far (one line per problem shape).
std::string autotune_report();

// The batch with the degree sums on the tensor cores (INT8 digit products,
// FP64 recombination): kgrad 0 the potential, 1 grad1, 2 grad2, 3 all ten
// quantities (as shs_point_batch_dev).
Status shs_point_batch_i8_dev(const charm_point *pnt, size_t nsets,
                              const unsigned long *nmax,
                              const unsigned long *shc_nmax, const double *mu,
                              double r, const double *const *d_c,
                              const double *const *d_s, int kgrad,
                              double *const *d_f);

// Single-precision potential synthesis / analysis on grids whose rows admit
// the shared-memory row transform, every row at r = R; float coefficient
// triangles (degree shc_nmax) and float grid [nlat][nlon] in device memory.
Status shs_point_dev_f32(const charm_point *pnt, unsigned long shc_nmax,
                         double mu, double r, const float *d_c,
                         const float *d_s, unsigned long nmax, float *d_f);
Status sha_point_dev_f32(const charm_point *pnt, const float *d_f,
                         unsigned long nmax, double mu, double r,
                         unsigned long shc_nmax, float *d_c, float *d_s);

// The same mode with float host arrays (the charmf_* ABI): whether the
// single-precision kernels serve a call (grid with FFT longitudes and an
// even row length, nmax <= 2200, every row at r = R), and the calls
// themselves (contiguous float triangles of degree shc_nmax, float grid).
bool f32_serves(const charm_point *pnt, unsigned long nmax, double R);
Status shs_point_f32_host(const charm_point *pnt, unsigned long shc_nmax,
                          double mu, double r, const float *c, const float *s,
                          unsigned long nmax, float *f);
Status sha_point_f32_host(const charm_point *pnt, const float *f,
                          unsigned long nmax, double mu, double r,
                          unsigned long shc_nmax, float *c, float *s);

// Adjoint of the scattered-point potential synthesis with respect to the
// coefficients: shcs->c, shcs->s (degree shcs->nmax, zero above nmax)
// receive sum_i g_i d f_i / d C_nm and d f_i / d S_nm for the model
// (shcs->mu, shcs->r).
Status shs_point_sctr_adjoint(const charm_point *pnt, const double *g,
                              unsigned long nmax, charm_shc *shcs);

// Same with the weights and the output triangles in device memory.
Status shs_point_sctr_adjoint_dev(const charm_point *pnt, const double *d_g,
                                  unsigned long nmax, double mu, double r,
                                  unsigned long shc_nmax, double *d_c,
                                  double *d_s);

// sha_point_dev without any allocation: every temporary lives in a fixed
// static device scratch (sha_static.cu); nmax <= 511, grids of at most 8192
// latitudes and rows the shared-memory transform handles.  Calls are
// serialised and synchronous; the first call on a device does the set-up
// (scratch address, tables).
Status sha_point_dev_static(const charm_point *pnt, const double *d_f,
                            unsigned long nmax, double mu, double r,
                            unsigned long shc_nmax, double *d_c, double *d_s);

// Quadrature grid nodes and weights on the GPU (north to south).
Status quad_nodes(int type, unsigned long nmax, double *lat, double *w);

// Measured FP64 FMA throughput of this device in TFLOP/s.
Status fp64_peak(double *tflops);

// The library's CUDA stream (cudaStream_t), or null without a device.
void *stream_handle();

// Per-kernel event timing and launch counting.
void set_timing(bool on);
void read_timing(double *ms, unsigned long long *n, unsigned long long *kern,
                 unsigned long long *ffts);

// Releases all device memory and plans.
void shutdown();

} // namespace cb
