// Host runtime of charm_b200 (see engine.h).
//
// One process-wide context per CUDA device: a stream, grow-only device
// buffers, cached recurrence tables per maximum degree, cached cuFFT plans
// and a pinned staging area for the small per-call arrays.  Calls are
// serialised by a mutex.  Every call ends with a synchronisation of the
// stream and a check of the device status word written by the kernels.
#include "engine.h"

#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "kernels.h"

namespace cb
{

namespace
{

const double PI = 3.14159265358979323846;

// src/misc/misc_is_nearly_equal.c:20-31
bool nearly_equal(double a, double b, double eps)
{
    double aa = std::fabs(a), ba = std::fabs(b), d = std::fabs(a - b);
    double s = aa + ba;
    if (a == b)
        return true;
    if (a == 0.0 || b == 0.0)
        return d <= eps;
    if (s == aa || s == ba)
        return d <= eps;
    return d / std::max(aa, ba) <= eps;
}

struct DevBuf
{
    void *p = nullptr;
    size_t bytes = 0;
};

struct Context
{
    bool ready = false;
    int device = -1;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    std::map<std::string, DevBuf> bufs;
    void *pinned = nullptr;
    size_t pinned_bytes = 0;
    // recurrence tables of the last maximum degree
    long long tab_nmax = -1;
    bool tab_has_en = false;
    std::map<std::tuple<int, int, long long>, cufftHandle> plans;
    std::mutex mtx;
};

Context g_ctx;

#define CB_CUDA(call, st)                                                     \
    do                                                                        \
    {                                                                         \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess)                                                \
        {                                                                     \
            (st).code = (e_ == cudaErrorMemoryAllocation) ? CHARM_EMEM        \
                                                          : CHARM_EFUNCARG;   \
            (st).msg = std::string("CUDA error in \"") + #call + "\": " +     \
                       cudaGetErrorString(e_);                                \
            return st;                                                        \
        }                                                                     \
    } while (0)

Status init(Context &c)
{
    Status st;
    if (c.ready)
    {
        int dev = -1;
        cudaGetDevice(&dev);
        if (dev == c.device)
            return st;
    }
    int dev = 0;
    CB_CUDA(cudaGetDevice(&dev), st);
    cudaDeviceProp prop;
    CB_CUDA(cudaGetDeviceProperties(&prop, dev), st);
    if (prop.major < 10)
    {
        st.code = CHARM_EFUNCARG;
        st.msg = "charm_b200 requires an sm_100 (Blackwell B200) device; "
                 "found compute capability " + std::to_string(prop.major) +
                 "." + std::to_string(prop.minor) + ".";
        return st;
    }
    c.device = dev;
    c.num_sms = prop.multiProcessorCount;
    if (!c.stream)
        CB_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking), st);
    c.ready = true;
    return st;
}

Status buf(Context &c, const std::string &name, size_t bytes, void **out)
{
    Status st;
    DevBuf &b = c.bufs[name];
    if (b.bytes < bytes)
    {
        if (b.p)
        {
            cudaStreamSynchronize(c.stream);
            cudaFree(b.p);
            b.p = nullptr;
            b.bytes = 0;
        }
        size_t want = std::max<size_t>(bytes, 256);
        cudaError_t e = cudaMalloc(&b.p, want);
        if (e != cudaSuccess)
        {
            cudaGetLastError();
            st.code = CHARM_EMEM;
            st.msg = std::string(CHARM_ERR_MALLOC_FAILURE) +
                     " (device buffer \"" + name + "\", " +
                     std::to_string(want) + " bytes)";
            return st;
        }
        b.bytes = want;
    }
    *out = b.p;
    return st;
}

template <typename T>
Status dbuf(Context &c, const std::string &name, size_t count, T **out)
{
    void *p = nullptr;
    Status st = buf(c, name, count * sizeof(T), &p);
    *out = static_cast<T *>(p);
    return st;
}

Status pinned(Context &c, size_t bytes, void **out)
{
    Status st;
    if (c.pinned_bytes < bytes)
    {
        if (c.pinned)
        {
            cudaStreamSynchronize(c.stream);
            cudaFreeHost(c.pinned);
            c.pinned = nullptr;
            c.pinned_bytes = 0;
        }
        size_t want = std::max<size_t>(bytes, 1 << 16);
        CB_CUDA(cudaMallocHost(&c.pinned, want), st);
        c.pinned_bytes = want;
    }
    *out = c.pinned;
    return st;
}

// sqrt(k), 1/sqrt(k) (src/leg/leg_func_r_ri.c) and the sectorial factors
// d_m (src/leg/leg_func_dm.c), computed on the host with IEEE operations.
void host_r_ri_dm(long long nmax, std::vector<double> &r,
                  std::vector<double> &ri, std::vector<double> &dm)
{
    r.assign(2 * nmax + 4, 0.0);
    ri.assign(2 * nmax + 4, 0.0);
    dm.assign(nmax + 1, 0.0);
    for (long long k = 1; k <= 2 * nmax + 3; k++)
    {
        double w = std::sqrt((double)k);
        r[k] = w;
        ri[k] = 1.0 / w;
    }
    for (long long n = 1; n <= nmax; n++)
        dm[n] = r[2 * n + 3] * ri[2 * n + 2];
}

Status tables(Context &c, long long nmax, bool need_en, double2 **ab,
              double2 **en, double **dm)
{
    Status st;
    long long T = (nmax + 1) * (nmax + 2) / 2;
    st = dbuf(c, "tab_ab", (size_t)T, ab);
    if (!st.ok())
        return st;
    if (need_en)
    {
        st = dbuf(c, "tab_en", (size_t)T, en);
        if (!st.ok())
            return st;
    }
    st = dbuf(c, "tab_dm", (size_t)(nmax + 1), dm);
    if (!st.ok())
        return st;
    bool fresh = (c.tab_nmax != nmax);
    if (!fresh && (!need_en || c.tab_has_en))
        return st;
    std::vector<double> r, ri, dmh;
    host_r_ri_dm(nmax, r, ri, dmh);
    double *dr = nullptr, *dri = nullptr;
    st = dbuf(c, "tab_r", r.size(), &dr);
    if (!st.ok())
        return st;
    st = dbuf(c, "tab_ri", ri.size(), &dri);
    if (!st.ok())
        return st;
    CB_CUDA(cudaMemcpyAsync(dr, r.data(), r.size() * 8, cudaMemcpyHostToDevice,
                            c.stream), st);
    CB_CUDA(cudaMemcpyAsync(dri, ri.data(), ri.size() * 8,
                            cudaMemcpyHostToDevice, c.stream), st);
    CB_CUDA(cudaMemcpyAsync(*dm, dmh.data(), dmh.size() * 8,
                            cudaMemcpyHostToDevice, c.stream), st);
    CB_CUDA(launch_tables(nmax, dr, dri, *ab, need_en ? *en : nullptr,
                          c.stream), st);
    // the host vectors must outlive the copies
    CB_CUDA(cudaStreamSynchronize(c.stream), st);
    if (fresh)
        c.tab_has_en = need_en;
    else
        c.tab_has_en = c.tab_has_en || need_en;
    c.tab_nmax = nmax;
    return st;
}

Status plan(Context &c, cufftType type, int n, long long batch,
            cufftHandle *out)
{
    Status st;
    auto key = std::make_tuple((int)type, n, batch);
    auto it = c.plans.find(key);
    if (it != c.plans.end())
    {
        *out = it->second;
        return st;
    }
    if (c.plans.size() >= 8)
    {
        cudaStreamSynchronize(c.stream);
        for (auto &kv : c.plans)
            cufftDestroy(kv.second);
        c.plans.clear();
    }
    cufftHandle h;
    int nn[1] = {n};
    int nfc = n / 2 + 1;
    cufftResult r;
    if (type == CUFFT_Z2D)
        r = cufftPlanMany(&h, 1, nn, nn, 1, nfc, nn, 1, n, CUFFT_Z2D,
                          (int)batch);
    else
        r = cufftPlanMany(&h, 1, nn, nn, 1, n, nn, 1, nfc, CUFFT_D2Z,
                          (int)batch);
    if (r != CUFFT_SUCCESS)
    {
        st.code = (r == CUFFT_ALLOC_FAILED) ? CHARM_EMEM : CHARM_EFUNCARG;
        st.msg = "cuFFT plan creation failed (code " + std::to_string((int)r) +
                 ")";
        return st;
    }
    cufftSetStream(h, c.stream);
    c.plans[key] = h;
    *out = h;
    return st;
}

// Triangle pointer of a charm_shc if c[m] are laid out contiguously as in
// src/shc/shc_init_chunk.c:126-145 (the case for every charm_shc built by
// CHarm's constructors), else null.
const double *contiguous_tri(double *const *cols, unsigned long nmax)
{
    if (!cols || !cols[0])
        return nullptr;
    const double *base = cols[0];
    size_t idx = 0;
    for (unsigned long m = 0; m <= nmax; m++)
    {
        if (cols[m] != base + idx)
            return nullptr;
        idx += nmax + 1 - m;
    }
    return base;
}

// Uploads a coefficient triangle of degree shc_nmax to the device.
Status upload_tri(Context &c, double *const *cols, unsigned long shc_nmax,
                  double *dst)
{
    Status st;
    const double *base = contiguous_tri(cols, shc_nmax);
    size_t T = (size_t)(shc_nmax + 1) * (shc_nmax + 2) / 2;
    if (base)
    {
        CB_CUDA(cudaMemcpyAsync(dst, base, T * 8, cudaMemcpyHostToDevice,
                                c.stream), st);
        return st;
    }
    size_t idx = 0;
    for (unsigned long m = 0; m <= shc_nmax; m++)
    {
        size_t len = shc_nmax + 1 - m;
        CB_CUDA(cudaMemcpyAsync(dst + idx, cols[m], len * 8,
                                cudaMemcpyHostToDevice, c.stream), st);
        idx += len;
    }
    return st;
}

Status download_tri(Context &c, const double *src, unsigned long shc_nmax,
                    double *const *cols)
{
    Status st;
    const double *base = contiguous_tri(cols, shc_nmax);
    size_t T = (size_t)(shc_nmax + 1) * (shc_nmax + 2) / 2;
    if (base)
    {
        CB_CUDA(cudaMemcpyAsync(const_cast<double *>(base), src, T * 8,
                                cudaMemcpyDeviceToHost, c.stream), st);
        return st;
    }
    size_t idx = 0;
    for (unsigned long m = 0; m <= shc_nmax; m++)
    {
        size_t len = shc_nmax + 1 - m;
        CB_CUDA(cudaMemcpyAsync(cols[m], src + idx, len * 8,
                                cudaMemcpyDeviceToHost, c.stream), st);
        idx += len;
    }
    return st;
}

bool is_quad(int t)
{
    return t == CHARM_CRD_POINT_GRID_GL || t == CHARM_CRD_POINT_GRID_DH1 ||
           t == CHARM_CRD_POINT_GRID_DH2;
}

bool is_dh(int t)
{
    return t == CHARM_CRD_POINT_GRID_DH1 || t == CHARM_CRD_POINT_GRID_DH2;
}

// src/misc/misc_arr_chck_symm.c
int arr_chck_symm(const double *a, size_t n, double eps)
{
    size_t middle = n / 2;
    for (size_t i = 0; i < middle; i++)
        if (!nearly_equal(a[i], -a[n - 1 - i], eps))
            return 1;
    if ((n % 2) && !nearly_equal(0.0, a[middle], eps))
        return 2;
    return 0;
}

// Latitude pairs of a grid: evaluated rows, mirror rows (-1 when none),
// following src/shs/shs_point_grd.c:113-197 and
// src/crd/crd_grd_check_symm.c:21-72.
struct Pairs
{
    std::vector<int> row_n, row_s;
};

void grid_pairs(const charm_point *pnt, double thr2, bool allow_symm,
                Pairs &P)
{
    size_t nlat = pnt->nlat;
    bool dh = is_dh(pnt->type);
    bool quad = is_quad(pnt->type);
    size_t pnt_nlat = dh ? nlat + 1 : nlat;
    bool even = (pnt_nlat % 2) == 0;
    bool symm;
    if (pnt_nlat == 1)
        symm = false;
    else if (quad)
        symm = true;
    else
        symm = arr_chck_symm(pnt->lat, nlat, thr2) == 0;
    if (!allow_symm)
        symm = false;
    size_t equator = (size_t)-1;
    if (quad)
    {
        unsigned long nmax_grd = pnt->type == CHARM_CRD_POINT_GRID_GL
                                     ? nlat - 1
                                     : (nlat - 2) / 2;
        if (!(pnt->type == CHARM_CRD_POINT_GRID_GL && (nmax_grd % 2)))
            equator = nlat / 2;
    }
    size_t nlatdo = symm ? (pnt_nlat + 1 - (even ? 1 : 0)) / 2 : pnt_nlat;
    if (!symm && dh)
        nlatdo = nlat; // no phantom south pole when every row is evaluated
    P.row_n.clear();
    P.row_s.clear();
    for (size_t ipv = 0; ipv < nlatdo; ipv++)
    {
        int s;
        if (!symm)
            s = 0;
        else if (quad)
        {
            if (dh && ipv == 0)
                s = 0;
            else if (ipv < equator)
                s = 1;
            else
                s = 0;
        }
        else
            s = (!even && ipv == nlatdo - 1) ? 0 : 1;
        P.row_n.push_back((int)ipv);
        P.row_s.push_back(s ? (int)(pnt_nlat - ipv - 1) : -1);
    }
}

int choose_k(int kgrad, int dlat, long long nunits)
{
    if (kgrad == 2)
        return 1;
    if (kgrad == 1 || dlat > 0)
        return nunits >= 64 ? 2 : 1;
    if (nunits >= 1024)
        return 4;
    return nunits >= 64 ? 2 : 1;
}

Status finish(Context &c, unsigned *d_status)
{
    Status st;
    unsigned h_status = 0;
    CB_CUDA(cudaMemcpyAsync(&h_status, d_status, sizeof(unsigned),
                            cudaMemcpyDeviceToHost, c.stream), st);
    CB_CUDA(cudaStreamSynchronize(c.stream), st);
    if (h_status)
    {
        st.code = CHARM_EFUNCARG;
        st.msg = "A GPU kernel reported an internal error (status " +
                 std::to_string(h_status) + ").";
    }
    return st;
}

Status status_words(Context &c, unsigned **d_status,
                    unsigned long long **d_counter)
{
    Status st;
    void *p = nullptr;
    st = buf(c, "status", 256, &p);
    if (!st.ok())
        return st;
    *d_status = static_cast<unsigned *>(p);
    *d_counter = reinterpret_cast<unsigned long long *>(
        static_cast<char *>(p) + 64);
    CB_CUDA(cudaMemsetAsync(p, 0, 256, c.stream), st);
    return st;
}

double polar_threshold(unsigned long nmax)
{
    // src/misc/misc_polar_optimization_threshold.c:16
    if (charm_glob_polar_optimization_a2 < 0.0)
        return -1.0;
    return std::max((double)charm_glob_polar_optimization_a1,
                    charm_glob_polar_optimization_a2 * (double)nmax);
}

// src/shs/shs_get_mur_dorder_npar.c:30-72
void mur_dorder(const charm_shc *shcs, int kgrad, int dr, int dlat, int dlon,
                double *mur, int *dorder, int *npar)
{
    if (kgrad == 1)
    {
        *dorder = 1;
        *npar = 3;
    }
    else if (kgrad == 2)
    {
        *dorder = 2;
        *npar = 6;
    }
    else
    {
        *dorder = dr + dlat + dlon;
        *npar = 1;
    }
    double rpow = shcs->r;
    for (int i = 1; i <= *dorder; i++)
        rpow *= shcs->r;
    *mur = shcs->mu / rpow;
}

// ---------------------------------------------------------------------------
// Grid synthesis
// ---------------------------------------------------------------------------
Status shs_grid(Context &c, const charm_point *pnt, const charm_shc *shcs,
                unsigned long nmax, int kgrad, int dr, int dlat, int dlon,
                double **f)
{
    Status st;
    const double thr = charm_glob_threshold, thr2 = charm_glob_threshold2;
    const size_t nlat = pnt->nlat, nlon = pnt->nlon;

    // longitudes: constant step (custom grids), FFT applicability
    if (pnt->type == CHARM_CRD_POINT_GRID && nlon > 1)
    {
        // src/misc/misc_arr_chck_lin_incr.c with first = 0, every_nth = 1
        double mn = pnt->lon[0];
        for (size_t j = 1; j < nlon; j++)
            mn = std::min(mn, pnt->lon[j]);
        bool bad = !nearly_equal(pnt->lon[0], mn, thr2);
        double step = pnt->lon[1] - pnt->lon[0];
        if (!bad && step <= 0.0)
            bad = true;
        for (size_t j = 1; !bad && j < nlon; j++)
            if (!nearly_equal(step, pnt->lon[j] - pnt->lon[j - 1], thr2))
                bad = true;
        if (bad)
        {
            st.code = CHARM_EFUNCARG;
            st.msg = "\"pnt->lon\" is not a linearly increasing array within "
                     "the \"threshold2\".";
            return st;
        }
    }
    double dlon_step = nlon > 1 ? pnt->lon[1] - pnt->lon[0] : 0.0;
    bool use_fft = (nlon >= 1) && ((nlon - 1) / 2 >= nmax) &&
                   nearly_equal(pnt->lon[0], 0.0, thr) &&
                   nearly_equal(pnt->lon[nlon - 1] + dlon_step, 2.0 * PI, thr);

    // radii: r == R everywhere selects the faster kernels
    bool r_eq = true;
    for (size_t i = 0; i < nlat; i++)
        if (!nearly_equal(pnt->r[i], shcs->r, thr))
        {
            r_eq = false;
            break;
        }
    Pairs P;
    grid_pairs(pnt, thr2, true, P);
    if (!r_eq)
    {
        // a mirror row with another radius cannot share the recurrence
        for (size_t p = 0; p < P.row_n.size(); p++)
            if (P.row_s[p] >= 0 && P.row_s[p] < (int)nlat &&
                pnt->r[P.row_s[p]] != pnt->r[P.row_n[p]])
            {
                grid_pairs(pnt, thr2, false, P);
                break;
            }
    }
    const int np = (int)P.row_n.size();

    double mur;
    int dorder, npar;
    mur_dorder(shcs, kgrad, dr, dlat, dlon, &mur, &dorder, &npar);

    // per-pair geometry staged through pinned memory (one upload)
    size_t geo_bytes = (size_t)np * (3 * 8 + 2 * 4);
    void *hp = nullptr;
    st = pinned(c, geo_bytes, &hp);
    if (!st.ok())
        return st;
    double *ht = static_cast<double *>(hp);
    double *hu = ht + np;
    double *hrho = hu + np;
    int *hrn = reinterpret_cast<int *>(hrho + np);
    int *hrs = hrn + np;
    for (int p = 0; p < np; p++)
    {
        double la = pnt->lat[P.row_n[p]];
        ht[p] = std::sin(la);
        hu[p] = std::cos(la);
        hrho[p] = r_eq ? 1.0 : shcs->r / pnt->r[P.row_n[p]];
        hrn[p] = P.row_n[p];
        hrs[p] = P.row_s[p];
    }
    void *dgeo = nullptr;
    st = buf(c, "geo", geo_bytes, &dgeo);
    if (!st.ok())
        return st;
    CB_CUDA(cudaMemcpyAsync(dgeo, hp, geo_bytes, cudaMemcpyHostToDevice,
                            c.stream), st);
    const double *dt = static_cast<const double *>(dgeo);
    const double *du = dt + np;
    const double *drho = du + np;
    const int *drn = reinterpret_cast<const int *>(drho + np);
    const int *drs = drn + np;

    bool need_en = (kgrad > 0) || (dlat > 0);
    double2 *ab = nullptr, *en = nullptr;
    double *dm = nullptr;
    st = tables(c, (long long)nmax, need_en, &ab, &en, &dm);
    if (!st.ok())
        return st;

    // coefficients
    const long long Ts = (long long)(shcs->nmax + 1) * (shcs->nmax + 2) / 2;
    const long long T = (long long)(nmax + 1) * (nmax + 2) / 2;
    double *dcs_raw = nullptr;
    double2 *dcs = nullptr;
    st = dbuf(c, "shc_in", (size_t)(2 * Ts), &dcs_raw);
    if (!st.ok())
        return st;
    st = dbuf(c, "cs", (size_t)T, &dcs);
    if (!st.ok())
        return st;
    st = upload_tri(c, shcs->c, shcs->nmax, dcs_raw);
    if (!st.ok())
        return st;
    st = upload_tri(c, shcs->s, shcs->nmax, dcs_raw + Ts);
    if (!st.ok())
        return st;
    CB_CUDA(launch_interleave((long long)nmax, (long long)shcs->nmax, dcs_raw,
                              dcs_raw + Ts, dcs, c.stream), st);

    // sectorial seeds
    double *psx = nullptr;
    int *pse = nullptr;
    st = dbuf(c, "psx", (size_t)(nmax + 1) * np, &psx);
    if (!st.ok())
        return st;
    st = dbuf(c, "pse", (size_t)(nmax + 1) * np, &pse);
    if (!st.ok())
        return st;
    CB_CUDA(launch_sectorial((long long)nmax, np, du, drho, r_eq ? 0 : 1,
                             dorder, dm, psx, pse, c.stream), st);

    // lumped coefficients
    const int ldf = use_fft ? (int)(nlon / 2 + 1) : (int)(nmax + 1);
    double2 *lc = nullptr;
    st = dbuf(c, "lumped", (size_t)npar * nlat * ldf, &lc);
    if (!st.ok())
        return st;
    if (use_fft)
        CB_CUDA(cudaMemsetAsync(lc, 0, (size_t)npar * nlat * ldf * 16,
                                c.stream), st);
    unsigned *d_status;
    unsigned long long *d_counter;
    st = status_words(c, &d_status, &d_counter);
    if (!st.ok())
        return st;

    const int K = choose_k(kgrad, dlat, np);
    const int ntiles = (np + 32 * K - 1) / (32 * K);
    ShsGridArgs A{};
    A.nmax = (long long)nmax;
    A.npairs = np;
    A.ntiles = ntiles;
    A.nitems = (long long)(nmax + 1) * ntiles;
    A.ab = ab;
    A.cs = dcs;
    A.en = en;
    A.psx = psx;
    A.pse = pse;
    A.t = dt;
    A.u = du;
    A.rho = drho;
    A.row_n = drn;
    A.row_s = drs;
    A.nlat = (int)nlat;
    A.ldf = ldf;
    A.out = lc;
    A.mur = mur;
    A.fft_pack = use_fft ? 1 : 0;
    A.dlon = dlon;
    A.polar_thr = polar_threshold(nmax);
    A.counter = d_counter;
    A.status = d_status;
    long long warps_needed = A.nitems;
    int grid = (int)std::min<long long>((warps_needed + 3) / 4,
                                        (long long)c.num_sms * 8);
    CB_CUDA(launch_shs_grid(A, kgrad, dr, dlat, !r_eq, K, std::max(grid, 1),
                            c.stream), st);

    // longitude sums
    double *fg = nullptr;
    st = dbuf(c, "fgrid", (size_t)npar * nlat * nlon, &fg);
    if (!st.ok())
        return st;
    if (use_fft)
    {
        cufftHandle h;
        st = plan(c, CUFFT_Z2D, (int)nlon, (long long)npar * nlat, &h);
        if (!st.ok())
            return st;
        cufftResult r = cufftExecZ2D(h, reinterpret_cast<cufftDoubleComplex *>(lc),
                                     fg);
        if (r != CUFFT_SUCCESS)
        {
            st.code = CHARM_EFUNCARG;
            st.msg = "cuFFT Z2D failed (code " + std::to_string((int)r) + ")";
            return st;
        }
    }
    else
    {
        double *dlon_arr = nullptr;
        st = dbuf(c, "lon", nlon, &dlon_arr);
        if (!st.ok())
            return st;
        CB_CUDA(cudaMemcpyAsync(dlon_arr, pnt->lon, nlon * 8,
                                cudaMemcpyHostToDevice, c.stream), st);
        CB_CUDA(launch_lon_direct(npar, (int)nlat, (int)nlon, (long long)nmax,
                                  lc, ldf, dlon_arr, fg, c.stream), st);
    }
    for (int q = 0; q < npar; q++)
        CB_CUDA(cudaMemcpyAsync(f[q], fg + (size_t)q * nlat * nlon,
                                nlat * nlon * 8, cudaMemcpyDeviceToHost,
                                c.stream), st);
    return finish(c, d_status);
}

// ---------------------------------------------------------------------------
// Scattered synthesis
// ---------------------------------------------------------------------------
Status shs_sctr(Context &c, const charm_point *pnt, const charm_shc *shcs,
                unsigned long nmax, int kgrad, int dr, int dlat, int dlon,
                double **f)
{
    Status st;
    const size_t npt = pnt->nlat;
    bool r_eq = true;
    for (size_t i = 0; i < npt; i++)
        if (!nearly_equal(pnt->r[i], shcs->r, charm_glob_threshold))
        {
            r_eq = false;
            break;
        }
    double mur;
    int dorder, npar;
    mur_dorder(shcs, kgrad, dr, dlat, dlon, &mur, &dorder, &npar);
    bool need_en = (kgrad > 0) || (dlat > 0);
    double2 *ab = nullptr, *en = nullptr;
    double *dm = nullptr;
    st = tables(c, (long long)nmax, need_en, &ab, &en, &dm);
    if (!st.ok())
        return st;
    const long long Ts = (long long)(shcs->nmax + 1) * (shcs->nmax + 2) / 2;
    const long long T = (long long)(nmax + 1) * (nmax + 2) / 2;
    double *dcs_raw = nullptr;
    double2 *dcs = nullptr;
    st = dbuf(c, "shc_in", (size_t)(2 * Ts), &dcs_raw);
    if (!st.ok())
        return st;
    st = dbuf(c, "cs", (size_t)T, &dcs);
    if (!st.ok())
        return st;
    st = upload_tri(c, shcs->c, shcs->nmax, dcs_raw);
    if (!st.ok())
        return st;
    st = upload_tri(c, shcs->s, shcs->nmax, dcs_raw + Ts);
    if (!st.ok())
        return st;
    CB_CUDA(launch_interleave((long long)nmax, (long long)shcs->nmax, dcs_raw,
                              dcs_raw + Ts, dcs, c.stream), st);
    double *dpts = nullptr;
    st = dbuf(c, "sctr_pts", 3 * npt, &dpts);
    if (!st.ok())
        return st;
    CB_CUDA(cudaMemcpyAsync(dpts, pnt->lat, npt * 8, cudaMemcpyHostToDevice,
                            c.stream), st);
    CB_CUDA(cudaMemcpyAsync(dpts + npt, pnt->lon, npt * 8,
                            cudaMemcpyHostToDevice, c.stream), st);
    if (!r_eq)
        CB_CUDA(cudaMemcpyAsync(dpts + 2 * npt, pnt->r, npt * 8,
                                cudaMemcpyHostToDevice, c.stream), st);
    double *fo = nullptr;
    st = dbuf(c, "sctr_f", (size_t)npar * npt, &fo);
    if (!st.ok())
        return st;
    unsigned *d_status;
    unsigned long long *d_counter;
    st = status_words(c, &d_status, &d_counter);
    if (!st.ok())
        return st;
    const int K = choose_k(kgrad, dlat, (long long)npt);
    SctrArgs A{};
    A.nmax = (long long)nmax;
    A.npoint = (long long)npt;
    A.ntiles = ((long long)npt + 32 * K - 1) / (32 * K);
    A.ab = ab;
    A.cs = dcs;
    A.en = en;
    A.dm = dm;
    A.lat = dpts;
    A.lon = dpts + npt;
    A.r = dpts + 2 * npt;
    A.R = shcs->r;
    A.f = fo;
    A.mur = mur;
    A.dlon = dlon;
    A.polar_thr = polar_threshold(nmax);
    A.counter = d_counter;
    A.status = d_status;
    int grid = (int)std::min<long long>((A.ntiles + 3) / 4,
                                        (long long)c.num_sms * 8);
    CB_CUDA(launch_sctr(A, kgrad, dr, dlat, !r_eq, K, std::max(grid, 1),
                        c.stream), st);
    for (int q = 0; q < npar; q++)
        CB_CUDA(cudaMemcpyAsync(f[q], fo + (size_t)q * npt, npt * 8,
                                cudaMemcpyDeviceToHost, c.stream), st);
    return finish(c, d_status);
}

} // namespace

// ---------------------------------------------------------------------------
// Public engine entry points
// ---------------------------------------------------------------------------
Status shs_point(const charm_point *pnt, const charm_shc *shcs,
                 unsigned long nmax, int kgrad, int dr, int dlat, int dlon,
                 double **f)
{
    std::lock_guard<std::mutex> lock(g_ctx.mtx);
    Status st = init(g_ctx);
    if (!st.ok())
        return st;
    if (pnt->type == CHARM_CRD_POINT_SCATTERED)
        return shs_sctr(g_ctx, pnt, shcs, nmax, kgrad, dr, dlat, dlon, f);
    return shs_grid(g_ctx, pnt, shcs, nmax, kgrad, dr, dlat, dlon, f);
}

Status sha_point(const charm_point *pnt, const double *f, unsigned long nmax,
                 charm_shc *shcs)
{
    std::lock_guard<std::mutex> lock(g_ctx.mtx);
    Context &c = g_ctx;
    Status st = init(c);
    if (!st.ok())
        return st;
    const size_t nlat = pnt->nlat, nlon = pnt->nlon;
    const double r0 = pnt->r[0];
    const unsigned long nmax_grd = pnt->type == CHARM_CRD_POINT_GRID_GL
                                       ? nlat - 1
                                       : (nlat - 2) / 2;
    // quadrature constant, src/sha/sha_point.c:313-322
    double cq = 0.0;
    if (pnt->type == CHARM_CRD_POINT_GRID_GL ||
        pnt->type == CHARM_CRD_POINT_GRID_DH1)
        cq = PI / (double)(nmax_grd + 1);
    else
        cq = PI / (double)(2 * nmax_grd + 2);
    cq *= 1.0 / (4.0 * PI) * (r0 / shcs->mu);

    Pairs P;
    grid_pairs(pnt, charm_glob_threshold2, true, P);
    const int np = (int)P.row_n.size();
    size_t geo_bytes = (size_t)np * (4 * 8 + 2 * 4);
    void *hp = nullptr;
    st = pinned(c, geo_bytes, &hp);
    if (!st.ok())
        return st;
    double *ht = static_cast<double *>(hp);
    double *hu = ht + np;
    double *hcn = hu + np;
    double *hcs = hcn + np;
    int *hrn = reinterpret_cast<int *>(hcs + np);
    int *hrs = hrn + np;
    for (int p = 0; p < np; p++)
    {
        double la = pnt->lat[P.row_n[p]];
        ht[p] = std::sin(la);
        hu[p] = std::cos(la);
        hcn[p] = cq * pnt->w[P.row_n[p]];
        hcs[p] = P.row_s[p] >= 0 ? cq * pnt->w[P.row_s[p]] : 0.0;
        hrn[p] = P.row_n[p];
        hrs[p] = P.row_s[p];
    }
    void *dgeo = nullptr;
    st = buf(c, "geo", geo_bytes, &dgeo);
    if (!st.ok())
        return st;
    CB_CUDA(cudaMemcpyAsync(dgeo, hp, geo_bytes, cudaMemcpyHostToDevice,
                            c.stream), st);
    const double *dt = static_cast<const double *>(dgeo);
    const double *du = dt + np;
    const double *dcn = du + np;
    const double *dcsw = dcn + np;
    const int *drn = reinterpret_cast<const int *>(dcsw + np);
    const int *drs = drn + np;

    double2 *ab = nullptr, *en = nullptr;
    double *dm = nullptr;
    st = tables(c, (long long)nmax, false, &ab, &en, &dm);
    if (!st.ok())
        return st;

    // grid upload and r2c along the parallels
    double *fg = nullptr;
    st = dbuf(c, "fgrid", nlat * nlon, &fg);
    if (!st.ok())
        return st;
    CB_CUDA(cudaMemcpyAsync(fg, f, nlat * nlon * 8, cudaMemcpyHostToDevice,
                            c.stream), st);
    const int ldF = (int)(nlon / 2 + 1);
    double2 *F = nullptr;
    st = dbuf(c, "lumped", nlat * (size_t)ldF, &F);
    if (!st.ok())
        return st;
    cufftHandle h;
    st = plan(c, CUFFT_D2Z, (int)nlon, (long long)nlat, &h);
    if (!st.ok())
        return st;
    if (cufftExecD2Z(h, fg, reinterpret_cast<cufftDoubleComplex *>(F)) !=
        CUFFT_SUCCESS)
    {
        st.code = CHARM_EFUNCARG;
        st.msg = "cuFFT D2Z failed";
        return st;
    }

    double *psx = nullptr;
    int *pse = nullptr;
    st = dbuf(c, "psx", (size_t)(nmax + 1) * np, &psx);
    if (!st.ok())
        return st;
    st = dbuf(c, "pse", (size_t)(nmax + 1) * np, &pse);
    if (!st.ok())
        return st;
    CB_CUDA(launch_sectorial((long long)nmax, np, du, nullptr, 0, 0, dm, psx,
                             pse, c.stream), st);

    unsigned *d_status;
    unsigned long long *d_counter;
    st = status_words(c, &d_status, &d_counter);
    if (!st.ok())
        return st;
    const int K = choose_k(0, 0, np);
    const int ntiles = (np + 32 * K - 1) / (32 * K);
    const long long T = (long long)(nmax + 1) * (nmax + 2) / 2;
    long long slots = (long long)c.num_sms * 8 * 4;
    long long G = std::max<long long>(1, (2 * slots + nmax) / (nmax + 1));
    G = std::min<long long>(G, ntiles);
    int tpg = (int)((ntiles + G - 1) / G);
    G = (ntiles + tpg - 1) / tpg;
    double2 *part = nullptr;
    st = dbuf(c, "sha_part", (size_t)G * T, &part);
    if (!st.ok())
        return st;
    ShaGridArgs A{};
    A.nmax = (long long)nmax;
    A.npairs = np;
    A.ntiles = ntiles;
    A.ngroups = (int)G;
    A.tiles_per_group = tpg;
    A.nitems = (long long)(nmax + 1) * G;
    A.ab = ab;
    A.psx = psx;
    A.pse = pse;
    A.t = dt;
    A.u = du;
    A.row_n = drn;
    A.row_s = drs;
    A.cw_n = dcn;
    A.cw_s = dcsw;
    A.F = F;
    A.ldF = ldF;
    A.part = part;
    A.polar_thr = polar_threshold(nmax);
    A.counter = d_counter;
    A.status = d_status;
    int grid = (int)std::min<long long>((A.nitems + 3) / 4,
                                        (long long)c.num_sms * 8);
    CB_CUDA(launch_sha_grid(A, K, std::max(grid, 1), c.stream), st);

    // rescaling from r0 to shcs->r (src/sha/sha_point.c:1088-1108 with
    // src/shc/shc_rescale.c)
    const unsigned long sn = shcs->nmax;
    double *dres = nullptr;
    std::vector<double> res;
    if (!nearly_equal(shcs->r, r0, charm_glob_threshold))
    {
        double mu_ratio = shcs->mu / shcs->mu;
        double r_ratio = r0 / shcs->r;
        res.resize(sn + 1);
        double tmp2 = mu_ratio * r_ratio;
        res[0] = mu_ratio;
        for (unsigned long n = 1; n <= sn; n++)
        {
            res[n] = tmp2;
            tmp2 *= r_ratio;
        }
        st = dbuf(c, "sha_rescale", sn + 1, &dres);
        if (!st.ok())
            return st;
        CB_CUDA(cudaMemcpyAsync(dres, res.data(), (sn + 1) * 8,
                                cudaMemcpyHostToDevice, c.stream), st);
    }
    const long long Ts = (long long)(sn + 1) * (sn + 2) / 2;
    double *dout = nullptr;
    st = dbuf(c, "shc_out", (size_t)(2 * Ts), &dout);
    if (!st.ok())
        return st;
    CB_CUDA(launch_sha_reduce((long long)nmax, (long long)sn, (int)G, T, part,
                              dres, dout, dout + Ts, c.stream), st);
    st = download_tri(c, dout, sn, shcs->c);
    if (!st.ok())
        return st;
    st = download_tri(c, dout + Ts, sn, shcs->s);
    if (!st.ok())
        return st;
    return finish(c, d_status);
}

Status quad_nodes(int type, unsigned long nmax, double *lat, double *w)
{
    std::lock_guard<std::mutex> lock(g_ctx.mtx);
    Context &c = g_ctx;
    Status st = init(c);
    if (!st.ok())
        return st;
    size_t nlat = type == CHARM_CRD_POINT_GRID_GL ? nmax + 1 : 2 * (nmax + 1);
    double *d = nullptr;
    st = dbuf(c, "crd", 2 * nlat, &d);
    if (!st.ok())
        return st;
    CB_CUDA(cudaMemsetAsync(d, 0, 2 * nlat * 8, c.stream), st);
    unsigned *d_status;
    unsigned long long *d_counter;
    st = status_words(c, &d_status, &d_counter);
    if (!st.ok())
        return st;
    if (type == CHARM_CRD_POINT_GRID_GL)
        CB_CUDA(launch_gl_nodes(nmax, d, d + nlat, d_status, c.stream), st);
    else
        CB_CUDA(launch_dh_nodes(nmax, d, d + nlat, c.stream), st);
    CB_CUDA(cudaMemcpyAsync(lat, d, nlat * 8, cudaMemcpyDeviceToHost, c.stream),
            st);
    CB_CUDA(cudaMemcpyAsync(w, d + nlat, nlat * 8, cudaMemcpyDeviceToHost,
                            c.stream), st);
    st = finish(c, d_status);
    if (!st.ok() && type == CHARM_CRD_POINT_GRID_GL)
        st.msg = "Error in computing latitudes of the Gauss--Legendre grid.  "
                 "Either the maximum number of iterations was exceeded or at "
                 "least one latitude was detected to be not a real number.";
    return st;
}

void shutdown()
{
    std::lock_guard<std::mutex> lock(g_ctx.mtx);
    Context &c = g_ctx;
    if (!c.ready)
        return;
    cudaStreamSynchronize(c.stream);
    for (auto &kv : c.plans)
        cufftDestroy(kv.second);
    c.plans.clear();
    for (auto &kv : c.bufs)
        if (kv.second.p)
            cudaFree(kv.second.p);
    c.bufs.clear();
    if (c.pinned)
        cudaFreeHost(c.pinned);
    c.pinned = nullptr;
    c.pinned_bytes = 0;
    c.tab_nmax = -1;
    c.ready = false;
}

} // namespace cb
