// Kernel argument blocks and launchers of charm_b200 (host <-> device
// boundary inside the library; no torch types anywhere).
#pragma once

#include <cuda_runtime.h>

namespace cb
{

// Error bits written by kernels into the per-call device status word.
enum : unsigned
{
    DEV_ERR_WAIT_TIMEOUT = 1u,   // an mbarrier wait exceeded its limit
    DEV_ERR_BAD_ARGS = 2u,       // a kernel received inconsistent sizes
    DEV_ERR_TC_RANGE = 4u        // a value outside the fixed-point grid of
                                 // the tensor-core synthesis
};


// One coefficient set of a batched synthesis: its degree, its first work
// item, its scaled coefficients (in the layout of the shared tables' degree)
// and its lumped-coefficient output.
struct BatchSet
{
    long long nmax;
    long long item0;
    const double2 *cs;
    double2 *out;
    double mur;
    double polar_thr;
};

// Grid synthesis: lumped coefficients out[q][row][m] of every output
// component q, row and order m (shs_grid.cu).  tb, tmul, sg are the
// recurrence tables of leg.cuh / tables.cu.
struct ShsGridArgs
{
    long long nmax;
    int npairs;            // evaluated latitudes (north rows of the pairs)
    int ntiles;            // latitude tiles per order in this launch
    int tile0;             // first tile of this launch
    long long m0;          // first order of this launch (single set)
    long long nitems;      // (nmax + 1) * ntiles
    const double2 *tb;     // (beta_n, e_n / a_n) per (n, m), order-major
    const double *tmul;    // chunk entry multipliers [m][chunk]
    int ldmul;
    const double *sg;      // per m: (S_m 2^g_0, g_0)
    const double2 *cs;     // (ct C_nm, ct S_nm)
    const double *t;       // sin(lat) per pair
    const double *u;       // cos(lat) per pair
    const double *rho;     // R / r per pair (r != R only)
    const int *row_n;      // row index of the pair's latitude
    const int *row_s;      // row index of its mirror, or -1
    int nlat;              // rows of the output
    int ldf;               // leading dimension of the output rows (double2)
    double2 *out;          // [npar][nlat][ldf]
    double mur;            // GM / R^(dorder + 1)
    int fft_pack;          // 1: FFTW c2r packing (c a, -c b), c = 1/2 for m > 0
    int dlon;              // longitudinal derivative order (single quantity)
    double polar_thr;      // polar optimisation threshold, < 0 when off
    unsigned long long *counter;
    unsigned *status;
    // batched sets (nsets > 0): each item belongs to the set j with
    // sets[j].item0 <= item < sets[j + 1].item0, whose nmax (<= the tables'
    // nmax), cs, out, mur and polar_thr replace the fields above
    const BatchSet *sets;
    int nsets;
};

// Grid analysis: C_nm, S_nm partial sums per latitude group (sha_grid.cu).
struct ShaGridArgs
{
    long long nmax;
    int npairs;
    int ntiles;            // latitude tiles per order
    int ngroups;           // tile groups per order in this launch
    int group0;            // first group of this launch (partial sums)
    long long m0;          // first order of this launch (items: orders
                           // m0, m0 + 1, ... times ngroups)
    int tiles_per_group;
    long long nitems;      // (nmax + 1) * ngroups
    const double2 *tb;
    const double *tmul;
    int ldmul;
    const double *sg;
    const double *t;
    const double *u;
    const int *row_n;
    const int *row_s;
    const double *cw_n;    // quadrature weight times constant, north row
    const double *cw_s;    // same for the mirror row (0 when none)
    const double2 *F;      // r2c output [nlat][ldF]
    int ldF;
    double2 *part;         // [ngroups][T] (C, S) partial sums in R~ units
    double polar_thr;
    unsigned long long *counter;
    unsigned *status;
    // scattered points instead of grid pairs (adjoint of the scattered
    // synthesis): npairs counts points, and these replace t, u, F, cw_*
    const double *lat;
    const double *lon;
    const double *r;       // radius per point (read when r != R)
    const double *g;       // weight of each point's value
    double R;              // reference radius of the coefficients
};

// Block-mean values in cells (cell.cu).  Grid synthesis and analysis run
// over pairs of cell rows (a northern row and its mirror [-latmax,
// -latmin], or a row alone); scattered synthesis over single cells.
struct CellArgs
{
    long long nmax;
    int npairs;            // cell-row pairs (grids) or cells (scattered)
    int ntiles;            // tiles of 32 pairs
    long long nitems;      // work items of this launch
    const double2 *tb;     // (beta_n, e_n / a_n) per (n, m), order-major
    const double *tc;      // ct_n per (n, m)
    const double *tmul;    // chunk entry multipliers [m][chunk]
    int ldmul;
    const double *sg;      // per m: (S_m 2^g_0, g_0)
    const double *dm;      // sectorial factors d_m (leg_func_dm.c)
    const double *gm;      // g_m of the I_mm recurrence (leg_func_gm_hm.c)
    const double2 *cs;     // (ct C_nm, ct S_nm); synthesis only
    const double2 *hn;     // per n: (h_n, 1 / (n + 1))
    const double4 *zn;     // per n >= 1: (e_n+1, f_n+1, 1 / sqrt(2n + 1), 0)
                           // of the un-normalised zonal recurrence
    const double *geo;     // [8][npairs]: sin, cos of latmin; sin, cos of
                           // latmax; R / r; block-mean scale mu / (R dA);
                           // latmin; latmax
    double *imm;           // [nmax + 1][npairs] I_mm in real units
    const int *row_n;      // output row of the pair's northern cell row
    const int *row_s;      // row of its mirror, or -1
    double dlon;           // longitude step (= cell width) of a grid
    int fft;               // 1: FFTW c2r packing with (sm, cm); 0: (2/m)
                           // sin(m dlon / 2) for sums at cell centres
    int ldf;               // leading dimension of out (double2)
    double2 *out;          // lumped coefficients [nlat][ldf]
    double polar_thr;      // polar optimisation threshold, < 0 when off
    unsigned long long *counter;
    unsigned *status;
    // analysis: r2c rows and the group partial sums
    const double2 *F;
    int ldF;
    double2 *part;         // [ngroups][T] in J~ units
    int ngroups;
    int tiles_per_group;
    // scattered cells
    const double *lonsum;  // lonmin + lonmax per cell
    const double *dlonc;   // lonmax - lonmin per cell
    double *fout;          // block means per cell
    double mur;            // mu / R
};

// Scattered-point synthesis (sctr.cu).
struct SctrArgs
{
    long long nmax;
    long long npoint;
    long long ntiles;
    const double2 *tb;
    const double *tmul;
    int ldmul;
    const double *sg;
    const double *dm;      // sectorial factors d_m (leg_func_dm.c)
    const double2 *cs;
    const double *lat;
    const double *lon;
    const double *r;       // radius per point (read when r != R)
    double R;              // reference radius of the coefficients
    double *f;             // [npar][npoint]
    double mur;
    int dlon;
    double polar_thr;
    unsigned long long *counter;
    unsigned *status;
};

// Single-precision grid synthesis and analysis (f32.cu): potential only,
// r = R.  Same work split as the FP64 kernels.
struct ShsF32Args
{
    long long nmax;
    int npairs;
    int ntiles;
    long long nitems;
    const float4 *abcs;    // (a, a, -b, -b), (C, C, S, S) per (n, m)
    const double *smm;     // S_m = P_mm / u^m
    const double *t;
    const double *u;
    const int *row_n;
    const int *row_s;
    int nlat;
    int ldf;
    double2 *out;          // lumped coefficients [nlat][ldf], FFTW packing
    double mur;
    double polar_thr;
    unsigned long long *counter;
    unsigned *status;
};

struct ShaF32Args
{
    long long nmax;
    int npairs;
    int ntiles;
    int ngroups;
    int tiles_per_group;
    long long nitems;
    const float4 *ab;      // (a_nm, a_nm, -b_nm, -b_nm) per (n, m)
    const double *smm;
    const double *t;
    const double *u;
    const int *row_n;
    const int *row_s;
    const double *cw_n;
    const double *cw_s;
    const double2 *F;
    int ldF;
    float2 *part;          // [ngroups][T] partial sums
    double polar_thr;
    unsigned long long *counter;
    unsigned *status;
};

// Real <-> half-spectrum transforms of grid rows of even length L = 2H in
// shared memory (rfft.cu).
struct RfftArgs
{
    long long nrows;
    int H;                 // half length
    int M;                 // FFT length: H (direct) or >= 2H - 1 (Bluestein)
    int V;                 // values per thread (16); M / V threads
    int direct;            // 1: H = 2^a 3^b, no chirp convolution
    int4 npass;            // passes of FFT_M of radix 8, 4, 2, 3 (in order)
    const double2 *tw;     // exp(-2 pi i k / M), k < M
    const double2 *w;      // chirp exp(-i pi n^2 / H), n < H (Bluestein)
    const double2 *bh;     // FFT_M of the wrapped conjugate chirp, / M
    const double2 *ht;     // exp(-i pi k / H), k <= H
    double *x;             // real rows, leading dimension ldx (even)
    long long ldx;
    double2 *X;            // half spectra, leading dimension ldX
    long long ldX;
    int kmax;              // spectrum entries read (inverse) / written (forward)
    int f32_rows;          // 1: x points to float rows (converted on the fly)
    // synthesis of rows of length 4H whose spectra stop below H (kmax < H):
    // two complex DFTs of length H per row, each writing every other pair
    // of the row (rfft.cu, k_rfft_inv4); w4 = exp(+2 pi i k / 4H), k < H
    int quarter;
    const double2 *w4;
    // rows of odd length L (synthesis only): one complex DFT of length
    // H = L by Bluestein, the row being its real part
    int odd;
    // transforms longer than one CTA's shared memory: a cluster of C CTAs
    // per row, each holding M / C values (rfft.cu, k_rfftc_*); tw then has
    // M / C entries (exp(-2 pi i k C / M)), twM the M twiddles
    // exp(-2 pi i k / M), and bh is stored by residue: bh[q M/C + l] is
    // the FFT_M value C l + q
    int C;
    const double2 *twM;
};

// Size of the fixed device scratch of the allocation-free analysis
// (sha_static.cu) and the largest degree it serves.
constexpr size_t STATIC_SCRATCH_BYTES = 32u << 20;
constexpr long long STATIC_NMAX = 511;
// device address of that scratch on the current device
cudaError_t static_scratch_address(void **ptr);

cudaError_t launch_tables(long long nmax, const double *r, const double *ri,
                          const double *smm, double2 *tb, double *tc,
                          double *tmul, int ldmul, double *sg,
                          cudaStream_t st);
// k_scale_cs for the orders [m_lo, m_hi) only
cudaError_t launch_scale_cs_orders(long long nmax, long long shc_nmax,
                                   const double *c, const double *s,
                                   const double *tc, double2 *cs,
                                   long long m_lo, long long m_hi,
                                   cudaStream_t st);
cudaError_t launch_scale_cs(long long nmax, long long shc_nmax,
                            const double *c, const double *s,
                            const double *tc, double2 *cs, cudaStream_t st);
// same into the layout of degree ntab >= nmax (zero above nmax)
cudaError_t launch_scale_cs_set(long long ntab, long long nmax,
                                long long shc_nmax, const double *c,
                                const double *s, const double *tc,
                                double2 *cs, cudaStream_t st);
cudaError_t launch_shs_grid(const ShsGridArgs &A, int kgrad, int dr,
                            int dlat, bool rr, int K, int grid,
                            cudaStream_t st);
cudaError_t launch_lon_direct(int npar, int nlat, int nlon, long long nmax,
                              const double2 *lc, int ldf, const double *lon,
                              double *f, cudaStream_t st);
cudaError_t launch_sha_grid(const ShaGridArgs &A, int K, int grid,
                            cudaStream_t st);
// src: 0 grid pairs, 1 scattered points on the sphere r = R, 2 scattered
// points with their own radii
cudaError_t launch_sha_points(const ShaGridArgs &A, int src, int K, int grid,
                              cudaStream_t st);
// k_sha_reduce for the orders [m_lo, m_hi) only
cudaError_t launch_sha_reduce_orders(long long nmax, long long shc_nmax,
                                     int ngroups, long long T,
                                     const double2 *part, const double *tc,
                                     const double *rescale, double scale,
                                     double *c, double *s, long long m_lo,
                                     long long m_hi, cudaStream_t st);
cudaError_t launch_sha_reduce(long long nmax, long long shc_nmax, int ngroups,
                              long long T, const double2 *part,
                              const double *tc, const double *rescale,
                              double scale, double *c, double *s,
                              cudaStream_t st);
cudaError_t launch_gl_nodes(unsigned long nmax, double *lat, double *w,
                            unsigned *status, cudaStream_t st);
cudaError_t launch_dh_nodes(unsigned long nmax, double *lat, double *w,
                            cudaStream_t st);
cudaError_t launch_fp64_probe(long long iters, int blocks, int threads,
                              double *sink, cudaStream_t st);
cudaError_t launch_sctr(const SctrArgs &A, int kgrad, int dr, int dlat,
                        bool rr, int K, int grid, cudaStream_t st);
cudaError_t launch_cell_imm(const CellArgs &A, cudaStream_t st);
// shared: two adjacent pairs per lane (tiles of 64 pairs, A.ntiles set
// accordingly), rows aligned so that pair 2l's lower boundary is pair
// 2l + 1's upper one
cudaError_t launch_shs_cell(const CellArgs &A, bool rr, bool shared,
                            int grid, cudaStream_t st);
// K cell-row pairs per lane (1 or 2); A.ntiles counts tiles of 32 K pairs
// shared: pairs 2l and 2l + 1 are adjacent cell rows (the lower boundary
// of the first is the upper one of the second); K must be 2
cudaError_t launch_sha_cell(const CellArgs &A, int K, bool shared, int grid,
                            cudaStream_t st);
cudaError_t launch_shs_cell_sctr(const CellArgs &A, bool rr, int grid,
                                 cudaStream_t st);
// unnormalised forward DFT X[row][k], k <= kmax, of rows of any length
cudaError_t launch_dft_rows_fwd(long long nrows, long long L, int kmax,
                                const double *x, long long ldx, double2 *X,
                                int ldX, cudaStream_t st);
// global spectral gravity forward modelling (gfm.cu)
cudaError_t launch_gfm_power(size_t n, const double *shape, double R,
                             unsigned p, double Ri, double *rho, double *out,
                             cudaStream_t st);
cudaError_t launch_gfm_accum(long long na, long long np, const double *v,
                             double *ac, double *as, double *pc, double *ps,
                             bool scaled, cudaStream_t st);
cudaError_t launch_rfft_w4(int H, double2 *w4, cudaStream_t st);
cudaError_t launch_rfft_tables(RfftArgs &A, double2 *tw, double2 *w,
                               double2 *ht, double2 *bh, cudaStream_t st);
size_t rfft_smem_bytes(int M);
cudaError_t rfft_set_smem(size_t smem);
cudaError_t launch_rfft(const RfftArgs &A, bool inverse, cudaStream_t st);
// tables of a cluster plan (A.C > 1): tw (M / C), twM (M), w (H), ht
// (H + 1) and the residue-ordered kernel spectrum bh (M)
cudaError_t launch_rfftc_tables(RfftArgs &A, double2 *tw, double2 *twM,
                                double2 *w, double2 *ht, double2 *bh,
                                cudaStream_t st);
// clusters of C CTAs with the largest shared memory that can be resident
// at once (0: the cluster shape cannot be scheduled)
int rfftc_max_clusters(int C, int Mc);

// Batched grid synthesis with the degree sums on the tensor cores
// (shs_tc.cu): up to SHS_TC_SETS coefficient sets per launch.
constexpr int SHS_TC_SETS = 16;
// with the gradients (ten quantities per set): five coefficient families
// (C and S each) per set in the 32 accumulator columns
constexpr int SHS_TC_GRAD_SETS = 3;
constexpr int SHS_TC_FAMILIES = 5;

// Coefficient digit tiles of a batch: per order m and 64-degree chunk,
// [parity][digit][32 columns x 32 bytes] (columns 2 s, 2 s + 1 = C, S of
// set s), and the column exponents ecol[m][32].
struct ShsTcPrep
{
    long long nmax;                       // largest degree of the launch
    int nsets;
    long long set_nmax[SHS_TC_SETS];
    long long shc_nmax[SHS_TC_SETS];      // layout of each set's triangle
    const double *c[SHS_TC_SETS];
    const double *s[SHS_TC_SETS];
    const long long *chunk0;              // first chunk of each order
    int *ecol;
    unsigned char *bdig;
    unsigned *status;
    // 0: columns (C, S) per set; 1: the gradient families of shs_tc.cu,
    // column 10 set + 2 family + (0: C, 1: S)
    int grad;
};

struct ShsTcArgs
{
    long long nmax;                       // degree of the tables
    long long nmax_sets;                  // largest degree of the launch
    int npairs;
    int ntiles;                           // tiles of 128 latitude pairs
    long long nitems;                     // (nmax_sets + 1) * ntiles
    const double *tmul;                   // recurrence tables (leg.cuh)
    int ldmul;
    const double *sg;
    const double *btp;                    // beta_n rows of ldmul * 64
    const double *ctp;                    // ct_n rows of ldmul * 64
    const unsigned char *bdig;
    const long long *chunk0;
    const int *ecol;
    const double *t, *u, *rho;
    const int *row_n, *row_s;
    // per (order m, pair p) at m * npairs + p: the seed R~_mm in the
    // fixed-point scale (or its mantissa while scaled) and (E, eA)
    const double *seed_x;
    const int2 *seed_e;
    int nlat, ldf;
    int nsets;
    double2 *out[SHS_TC_SETS];            // lumped coefficients [nlat][ldf]
                                          // ([10][nlat][ldf] with grad)
    double mur[SHS_TC_SETS];              // GM / R per set
    unsigned long long *counter;
    unsigned *status;
    // 1: potential, grad1 and grad2 of SHS_TC_GRAD_SETS sets (ten lumped
    // arrays per set in the order V, grad1 l r p, grad2 ll lr lp rr rp pp;
    // GM / R^(k+1) = mur / Rref^k for the derivatives of order k)
    int grad;
    double Rref;
};

size_t shs_tc_smem_bytes();
size_t shs_tc_chunk_bytes();
cudaError_t launch_tc_ctab(long long nmax, int ld, const double2 *tb,
                           const double *tc, double *btp, double *ctp,
                           cudaStream_t st);
cudaError_t launch_tc_prep(const ShsTcPrep &P, cudaStream_t st);
cudaError_t launch_tc_seeds(const ShsTcArgs &A, bool rr, double *seed_x,
                            int2 *seed_e, cudaStream_t st);
cudaError_t launch_shs_tc(const ShsTcArgs &A, bool rr, int grid,
                          cudaStream_t st);
cudaError_t launch_tables_f32(long long nmax, const double *r,
                              const double *ri, float4 *ab, cudaStream_t st);
cudaError_t launch_pack_cs_f32(long long nmax, long long shc_nmax,
                               const float *c, const float *s,
                               const float4 *ab, float4 *abcs,
                               cudaStream_t st);
cudaError_t launch_shs_grid_f32(const ShsF32Args &A, int K, int grid,
                                cudaStream_t st);
cudaError_t launch_sha_grid_f32(const ShaF32Args &A, int K, int grid,
                                cudaStream_t st);
cudaError_t launch_sha_reduce_f32(long long nmax, long long shc_nmax,
                                  int ngroups, long long T,
                                  const float2 *part, const double *rescale,
                                  float *c, float *s, cudaStream_t st);

} // namespace cb
