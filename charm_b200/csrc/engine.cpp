// Host runtime of charm_b200 (see engine.h).
//
// One process-wide context, bound to the device it was set up on (one
// device per process): a compute stream and a copy stream (the host-array
// calls copy their grids and coefficients in bands there, ordered against
// the kernels by events), grow-only device buffers, cached recurrence
// tables per maximum degree, cached row-transform plans (rfft.cu, every
// row length up to 147456 points; no library FFT), a pinned staging
// area for the small per-call arrays and a ring of pinned buffers through
// which host threads copy pageable host arrays.
// Calls are serialised by a mutex.  Every call ends with a synchronisation
// of its streams and a check of the device status word written by the
// kernels.
#include "engine.h"

#include <cuda_runtime.h>

#include <sched.h>
#include <unistd.h>

#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
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

// Every a[i] nearly_equal to ref: an exact scan first (the common case, a
// grid on one sphere), the element-wise test only when that fails.
bool all_nearly_equal(const double *a, size_t n, double ref, double eps)
{
    bool exact = true;
    for (size_t i = 0; i < n; i++)
        exact &= (a[i] == ref);
    if (exact)
        return true;
    for (size_t i = 0; i < n; i++)
        if (!nearly_equal(a[i], ref, eps))
            return false;
    return true;
}

struct DevBuf
{
    void *p = nullptr;
    size_t bytes = 0;
};

constexpr int TAB_SLOTS = 3;
// bands of the host-array calls' copies (at most 6 of each kind)
constexpr int SHS_LAT_BANDS = 4;   // synthesis: grid rows down
constexpr int SHA_LAT_BANDS = 4;   // analysis: grid rows up
constexpr int SHS_ORD_BANDS = 4;   // synthesis: coefficients up
constexpr int SHA_ORD_BANDS = 4;   // analysis: coefficients down
constexpr int EV_LAT0 = 0, EV_ORD0 = 6, EV_START = 15;

struct Context
{
    bool ready = false;
    int device = -1;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    // host <-> device copies of grid bands, overlapped with the kernels on
    // `stream` (events order the two)
    cudaStream_t copy_stream = nullptr;
    // events between the compute and copy streams of the banded host-array
    // calls: EV_LAT0.. the bands of latitude tiles, EV_ORD0.. the bands of
    // orders, EV_START the start of the copy stream after the work already
    // on the compute stream
    cudaEvent_t band_ev[16] = {};
    // page-locked copy of the device status word read at the end of a call
    unsigned *h_status = nullptr;
    std::map<std::string, DevBuf> bufs;
    void *pinned = nullptr;
    size_t pinned_bytes = 0;
    // ring of page-locked buffers for copies of pageable host arrays
    // (stage_h2d / stage_d2h); ring_ev[b] marks the last copy on buffer b
    void *ring[4] = {};
    cudaEvent_t ring_ev[4] = {};
    // recurrence tables of up to TAB_SLOTS maximum degrees (least recently
    // used slot rewritten), so that calls alternating between a few
    // degrees, e.g. syntheses and analyses of other degrees, rebuild
    // nothing
    long long tab_nmax[TAB_SLOTS] = {-1, -1, -1};
    unsigned long long tab_used[TAB_SLOTS] = {};
    unsigned long long tab_clock = 0;
    // bumped whenever a cached device buffer is (re)allocated or a cached
    // table is rewritten: a captured graph reads these by address, so it
    // replays only while the epoch it was made in lasts
    unsigned long long epoch = 0;
    long long tab32_nmax = -1;   // single-precision tables of this degree
    long long tcp_nmax = -1;     // padded ct_n rows of the tensor-core path
    long long cell_nmax = -1;    // per-degree tables of the cell kernels
    // stream capture into a CUDA graph (batch_graph_create): host
    // synchronisations are skipped, small host uploads go through pinned
    // buffers owned by the graph
    bool capturing = false;
    std::vector<void *> capture_pins;
    // autotuned latitude pairs per lane of the synthesis kernel, per
    // (kgrad, dr, dlat, r != R, nmax, pairs); value and the measured ms of
    // each candidate
    std::map<std::tuple<int, int, int, int, long long, int>,
             std::pair<int, std::vector<std::pair<int, float>>>>
        tuned;
    // quadrature nodes and weights by (grid type, nmax), host copies of
    // the last few grids built (they are deterministic; forward modelling
    // builds the same grids at every call)
    std::map<std::pair<int, unsigned long>, std::vector<double>> nodes;
    std::vector<std::pair<int, unsigned long>> nodes_order;
    std::map<long long, RfftArgs> rffts;   // row transforms by row length
    std::map<long long, void *> rfft_mem;  // their tables
    std::recursive_mutex mtx;
    // optional per-kernel timing (CUDA events on the library stream)
    bool timing = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
    double timer_ms[TIMER_COUNT] = {};
    unsigned long long timer_n[TIMER_COUNT] = {};
    unsigned long long launches = 0;   // kernels of this library
    // launches of library kernels (none: every transform is this
    // library's own)
    unsigned long long fft_execs = 0;
};

Context g_ctx;

cudaEvent_t ev_get(Context &c)
{
    if (!c.ev_pool.empty())
    {
        cudaEvent_t e = c.ev_pool.back();
        c.ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Brackets one launch: counts it and, when timing is on, records a pair of
// events that finish() turns into elapsed milliseconds.
struct Scope
{
    Context &c;
    int id;
    bool lib;
    cudaEvent_t a = nullptr;
    Scope(Context &cc, int timer, bool library_kernel = true)
        : c(cc), id(timer), lib(library_kernel)
    {
        if (c.timing)
        {
            a = ev_get(c);
            cudaEventRecord(a, c.stream);
        }
    }
    ~Scope()
    {
        if (lib)
            c.launches++;
        else
            c.fft_execs++;
        if (c.timing)
        {
            cudaEvent_t b = ev_get(c);
            cudaEventRecord(b, c.stream);
            c.pending.push_back({id, {a, b}});
        }
    }
};

void resolve_timers(Context &c)
{
    for (auto &pe : c.pending)
    {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, pe.second.first, pe.second.second) ==
            cudaSuccess)
        {
            c.timer_ms[pe.first] += ms;
            c.timer_n[pe.first] += 1;
        }
        c.ev_pool.push_back(pe.second.first);
        c.ev_pool.push_back(pe.second.second);
    }
    c.pending.clear();
    cudaGetLastError();
}

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

#define CB_TRY(expr)                                                          \
    do                                                                        \
    {                                                                         \
        Status s_ = (expr);                                                   \
        if (!s_.ok())                                                         \
            return s_;                                                        \
    } while (0)

Status init(Context &c)
{
    Status st;
    int dev = 0;
    CB_CUDA(cudaGetDevice(&dev), st);
    if (c.ready)
    {
        if (dev == c.device)
            return st;
        // The streams, events, cached buffers, tables, transform plans and
        // kernel attributes of the context belong to the device it was set
        // up on: one device per process (one process per GPU, as the
        // replicas run).
        st.code = CHARM_EFUNCARG;
        st.msg = "charm_b200 serves one device per process: it was set up on "
                 "device " + std::to_string(c.device) +
                 " and is now called with device " + std::to_string(dev) +
                 " current.";
        return st;
    }
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
    if (!c.copy_stream)
        CB_CUDA(cudaStreamCreateWithFlags(&c.copy_stream,
                                          cudaStreamNonBlocking), st);
    for (cudaEvent_t &e : c.band_ev)
        if (!e)
            CB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), st);
    if (!c.h_status)
    {
        void *hp = nullptr;
        CB_CUDA(cudaHostAlloc(&hp, 64, cudaHostAllocDefault), st);
        c.h_status = static_cast<unsigned *>(hp);
    }
    c.ready = true;
    return st;
}

Status buf(Context &c, const std::string &name, size_t bytes, void **out)
{
    Status st;
    DevBuf &b = c.bufs[name];
    if (b.bytes < bytes && c.capturing)
    {
        st.code = CHARM_EFUNCARG;
        st.msg = "device buffer \"" + name + "\" grew during graph capture";
        return st;
    }
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
        c.epoch++;
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
    if (c.capturing)
    {
        // a buffer of its own, read by the graph at every replay
        void *p = nullptr;
        CB_CUDA(cudaMallocHost(&p, std::max<size_t>(bytes, 16)), st);
        c.capture_pins.push_back(p);
        *out = p;
        return st;
    }
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

// ---------------------------------------------------------------------------
// Pageable host arrays
// ---------------------------------------------------------------------------
// A copy between pageable host memory and the device runs through the
// driver's own staging, serially and at a fraction of the page-locked rate
// (numpy arrays, as PyHarm passes them, are pageable).  Such arrays are
// copied here through a ring of page-locked buffers instead: host threads
// copy chunk i between the caller's array and a ring buffer while the copy
// engine moves chunk i - 1.

constexpr int RING_N = 4;
constexpr size_t RING_CHUNK = (size_t)8 << 20;

// Host threads that copy one block of memory together: the caller takes
// the first slice and the workers the others.
class CopyPool
{
  public:
    explicit CopyPool(int workers) : n_(workers)
    {
        for (int k = 0; k < n_; k++)
            std::thread([this, k] { run(k + 1); }).detach();
    }

    void copy(void *dst, const void *src, size_t bytes)
    {
        if (n_ == 0 || bytes < ((size_t)1 << 20))
        {
            std::memcpy(dst, src, bytes);
            return;
        }
        {
            std::lock_guard<std::mutex> l(mu_);
            dst_ = static_cast<char *>(dst);
            src_ = static_cast<const char *>(src);
            bytes_ = bytes;
            pending_ = n_;
            gen_++;
        }
        go_.notify_all();
        slice(0, dst_, src_, bytes);
        std::unique_lock<std::mutex> l(mu_);
        done_.wait(l, [this] { return pending_ == 0; });
    }

  private:
    void slice(int k, char *d, const char *s, size_t bytes) const
    {
        const size_t parts = (size_t)n_ + 1;
        size_t a = (bytes * k / parts) & ~(size_t)63;
        size_t b = k + 1 == (int)parts ? bytes
                                       : (bytes * (k + 1) / parts) & ~(size_t)63;
        if (b > a)
            std::memcpy(d + a, s + a, b - a);
    }

    void run(int k)
    {
        unsigned long seen = 0;
        for (;;)
        {
            char *d;
            const char *s;
            size_t bytes;
            {
                std::unique_lock<std::mutex> l(mu_);
                go_.wait(l, [&] { return gen_ != seen; });
                seen = gen_;
                d = dst_;
                s = src_;
                bytes = bytes_;
            }
            slice(k, d, s, bytes);
            std::lock_guard<std::mutex> l(mu_);
            if (--pending_ == 0)
                done_.notify_one();
        }
    }

    const int n_;
    std::mutex mu_;
    std::condition_variable go_, done_;
    char *dst_ = nullptr;
    const char *src_ = nullptr;
    size_t bytes_ = 0;
    unsigned long gen_ = 0;
    int pending_ = 0;
};

// The pool of this process (made again in a forked child, which has none
// of the parent's threads): one worker per usable core beyond the
// caller's, at most seven.
CopyPool &copy_pool()
{
    static CopyPool *pool = nullptr;
    static pid_t owner = 0;
    if (!pool || owner != getpid())
    {
        int ncpu = 1;
        cpu_set_t set;
        if (sched_getaffinity(0, sizeof(set), &set) == 0)
            ncpu = CPU_COUNT(&set);
        pool = new CopyPool(std::max(0, std::min(7, ncpu - 1)));
        owner = getpid();
    }
    return *pool;
}

bool is_pageable(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess)
    {
        cudaGetLastError();
        return true;
    }
    return a.type == cudaMemoryTypeUnregistered;
}

Status ring_ready(Context &c)
{
    Status st;
    for (int b = 0; b < RING_N; b++)
    {
        if (!c.ring[b])
            CB_CUDA(cudaMallocHost(&c.ring[b], RING_CHUNK), st);
        if (!c.ring_ev[b])
            CB_CUDA(cudaEventCreateWithFlags(&c.ring_ev[b],
                                             cudaEventDisableTiming), st);
    }
    return st;
}

// Host to device on stream q (the compute stream when null); a pageable
// source is read through the ring (the caller may change it once this
// returns).  `pageable` < 0 asks the driver about src; callers that copy
// one array in several pieces decide once, for the whole array, and pass
// 0 or 1.
Status stage_h2d(Context &c, void *dst, const void *src, size_t bytes,
                 cudaStream_t q = nullptr, int pageable = -1)
{
    Status st;
    if (!q)
        q = c.stream;
    if (bytes == 0)
        return st;
    if (pageable < 0)
        pageable = is_pageable(src) ? 1 : 0;
    if (!pageable)
    {
        CB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, q),
                st);
        return st;
    }
    CB_TRY(ring_ready(c));
    char *d = static_cast<char *>(dst);
    const char *s = static_cast<const char *>(src);
    for (size_t off = 0, i = 0; off < bytes; off += RING_CHUNK, i++)
    {
        const int b = (int)(i % RING_N);
        const size_t len = std::min(RING_CHUNK, bytes - off);
        // the buffer's previous copy has read it
        CB_CUDA(cudaEventSynchronize(c.ring_ev[b]), st);
        copy_pool().copy(c.ring[b], s + off, len);
        CB_CUDA(cudaMemcpyAsync(d + off, c.ring[b], len,
                                cudaMemcpyHostToDevice, q), st);
        CB_CUDA(cudaEventRecord(c.ring_ev[b], q), st);
    }
    return st;
}

// Device to host after the work already on stream q (the compute stream
// when null); returns when the host array holds the data.  A pageable
// destination is written through the ring.
Status stage_d2h(Context &c, void *dst, const void *src, size_t bytes,
                 cudaStream_t q = nullptr, int pageable = -1)
{
    Status st;
    if (!q)
        q = c.stream;
    if (bytes == 0)
        return st;
    if (pageable < 0)
        pageable = is_pageable(dst) ? 1 : 0;
    if (!pageable)
    {
        CB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, q),
                st);
        CB_CUDA(cudaStreamSynchronize(q), st);
        return st;
    }
    CB_TRY(ring_ready(c));
    char *d = static_cast<char *>(dst);
    const char *s = static_cast<const char *>(src);
    const size_t nch = (bytes + RING_CHUNK - 1) / RING_CHUNK;
    auto issue = [&](size_t i) -> Status {
        Status s2;
        const int b = (int)(i % RING_N);
        const size_t off = i * RING_CHUNK;
        // an earlier copy out of this buffer, possibly on another stream,
        // has read it
        CB_CUDA(cudaStreamWaitEvent(q, c.ring_ev[b], 0), s2);
        CB_CUDA(cudaMemcpyAsync(c.ring[b], s + off,
                                std::min(RING_CHUNK, bytes - off),
                                cudaMemcpyDeviceToHost, q), s2);
        CB_CUDA(cudaEventRecord(c.ring_ev[b], q), s2);
        return s2;
    };
    for (size_t i = 0; i < std::min<size_t>(RING_N, nch); i++)
        CB_TRY(issue(i));
    for (size_t i = 0; i < nch; i++)
    {
        const int b = (int)(i % RING_N);
        const size_t off = i * RING_CHUNK;
        CB_CUDA(cudaEventSynchronize(c.ring_ev[b]), st);
        copy_pool().copy(d + off, c.ring[b],
                         std::min(RING_CHUNK, bytes - off));
        if (i + RING_N < nch)
            CB_TRY(issue(i + RING_N));
    }
    return st;
}

// Upload of a small host array; while capturing through a graph-owned
// pinned copy (the graph reads it at every replay).
Status h2d_small(Context &c, void *dst, const void *src, size_t bytes)
{
    Status st;
    if (!c.capturing)
    {
        CB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice,
                                c.stream), st);
        return st;
    }
    void *hp = nullptr;
    CB_TRY(pinned(c, bytes, &hp));
    std::memcpy(hp, src, bytes);
    CB_CUDA(cudaMemcpyAsync(dst, hp, bytes, cudaMemcpyHostToDevice, c.stream),
            st);
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

// S_m = P_mm(u) / u^m = sqrt(3) prod_{k=1}^{m-1} d_k
// (src/leg/leg_func_prepare.c), in extended precision, m = 0..nmax.
void host_smm(long long nmax, double *smm)
{
    long double s = 1.0L;
    smm[0] = 1.0;
    for (long long m = 1; m <= nmax; m++)
    {
        if (m == 1)
            s = sqrtl(3.0L);
        else
            s *= sqrtl((long double)(2 * m + 1) / (long double)(2 * m));
        smm[m] = (double)s;
    }
}

// Recurrence tables of the rescaled recurrence (leg.cuh, tables.cu), built
// once per maximum degree and kept on the device.
struct Tabs
{
    double2 *tb = nullptr;
    double *tc = nullptr;
    double *tmul = nullptr;
    int ldmul = 0;
    double *sg = nullptr;
    double *dm = nullptr;
};

Status tables(Context &c, long long nmax, Tabs *tab)
{
    Status st;
    long long T = (nmax + 1) * (nmax + 2) / 2;
    tab->ldmul = (int)((nmax + 1 + 63) / 64);
    int slot = -1;
    for (int k = 0; k < TAB_SLOTS; k++)
        if (c.tab_nmax[k] == nmax)
            slot = k;
    const bool hit = slot >= 0;
    if (!hit)
    {
        slot = 0;
        for (int k = 1; k < TAB_SLOTS; k++)
            if (c.tab_used[k] < c.tab_used[slot])
                slot = k;
    }
    c.tab_used[slot] = ++c.tab_clock;
    const std::string sfx = slot ? "#" + std::to_string(slot) : "";
    CB_TRY(dbuf(c, "tab_b" + sfx, (size_t)T, &tab->tb));
    CB_TRY(dbuf(c, "tab_c" + sfx, (size_t)T, &tab->tc));
    CB_TRY(dbuf(c, "tab_mul" + sfx, (size_t)(nmax + 1) * tab->ldmul,
                &tab->tmul));
    CB_TRY(dbuf(c, "tab_sg" + sfx, (size_t)(2 * (nmax + 1)), &tab->sg));
    CB_TRY(dbuf(c, "tab_dm" + sfx, (size_t)(nmax + 1), &tab->dm));
    if (hit)
        return st;
    // the slot is rewritten: invalid until the rebuild below completes
    c.tab_nmax[slot] = -1;
    c.epoch++;
    std::vector<double> r, ri, dmh;
    host_r_ri_dm(nmax, r, ri, dmh);
    std::vector<double> smm(nmax + 1);
    host_smm(nmax, smm.data());
    double *dr = nullptr, *dri = nullptr, *dsm = nullptr;
    CB_TRY(dbuf(c, "tab_r", r.size(), &dr));
    CB_TRY(dbuf(c, "tab_ri", ri.size(), &dri));
    CB_TRY(dbuf(c, "tab_smm", smm.size(), &dsm));
    CB_CUDA(cudaMemcpyAsync(dr, r.data(), r.size() * 8, cudaMemcpyHostToDevice,
                            c.stream), st);
    CB_CUDA(cudaMemcpyAsync(dri, ri.data(), ri.size() * 8,
                            cudaMemcpyHostToDevice, c.stream), st);
    CB_CUDA(cudaMemcpyAsync(dsm, smm.data(), smm.size() * 8,
                            cudaMemcpyHostToDevice, c.stream), st);
    CB_CUDA(cudaMemcpyAsync(tab->dm, dmh.data(), dmh.size() * 8,
                            cudaMemcpyHostToDevice, c.stream), st);
    {
        Scope sc(c, TIMER_TABLES);
        CB_CUDA(launch_tables(nmax, dr, dri, dsm, tab->tb, tab->tc, tab->tmul,
                              tab->ldmul, tab->sg, c.stream), st);
    }
    // the host vectors must outlive the copies
    CB_CUDA(cudaStreamSynchronize(c.stream), st);
    c.tab_nmax[slot] = nmax;
    return st;
}

// Shape of the transform of grid rows of length L (rfft.cu): the complex
// length H (L / 2 for even rows, L for odd rows), the FFT length M, the
// cluster size C (CTAs per row, each holding M / C values) and the passes
// of the per-CTA FFT, or false when no plan exists (M / C would exceed
// 9216 even with clusters of 16, i.e. H above 73728).
bool rfft_shape(long long L, RfftArgs *out)
{
    constexpr long long MC_MAX = 9216;   // values in one CTA's shared memory
    RfftArgs A{};
    A.M = 0;
    A.C = 1;
    A.V = 16;
    auto smooth = [](long long n, int *a, int *b) {
        *a = *b = 0;
        while (n > 1 && n % 2 == 0)
        {
            n /= 2;
            (*a)++;
        }
        while (n > 1 && n % 3 == 0)
        {
            n /= 3;
            (*b)++;
        }
        return n == 1;
    };
    // smallest 2^a 3^b >= need with a >= 6 (every per-CTA plan starts with
    // two radix-8 passes and keeps its strides multiples of 8), <= MC_MAX
    auto local_len = [&](long long need) {
        long long best = 0;
        for (long long p2 = 64; p2 <= MC_MAX; p2 *= 2)
            for (long long m = p2; m <= MC_MAX; m *= 3)
                if (m >= need && (best == 0 || m < best))
                    best = m;
        return best;
    };
    if (L < 1)
    {
        *out = A;
        return false;
    }
    const bool odd = (L % 2) != 0;
    const long long H = odd ? L : L / 2;
    int a = 0, b = 0;
    long long Mc = 0;
    if (!odd && smooth(H, &a, &b) && a >= 6 && H <= MC_MAX)
    {
        A.direct = 1;
        A.M = (int)H;
        Mc = H;
    }
    else
    {
        // Bluestein: M = C Mc >= 2H - 1, the smallest M, then the fewest
        // CTAs per row
        const long long need = 2 * H - 1;
        long long bestM = 0;
        for (int C = 1; C <= 16; C *= 2)
        {
            const long long m = local_len((need + C - 1) / C);
            if (m > 0 && (bestM == 0 || C * m < bestM))
            {
                bestM = C * m;
                A.C = C;
                Mc = m;
            }
        }
        if (bestM == 0)
        {
            *out = A;
            return false;
        }
        A.direct = 0;
        A.M = (int)bestM;
    }
    smooth(Mc, &a, &b);
    A.H = (int)H;
    A.odd = odd ? 1 : 0;
    // passes of the per-CTA FFT of length Mc: radix 8, then 4, then 2
    // (powers of two), then 3
    int p8 = a / 3, p4 = 0, p2 = 0;
    if (a % 3 == 2)
        p4 = 1;
    else if (a % 3 == 1)
    {
        if (p8 > 0)
        {
            p8--;
            p4 = 2;
        }
        else
            p2 = 1;
    }
    A.npass = make_int4(p8, p4, p2, b);
    *out = A;
    return true;
}

// Transform of grid rows of length L (rfft.cu), set up once per length:
// fails with CHARM_EFUNCARG when no plan exists for L (rfft_shape) or the
// plan's cluster shape cannot be scheduled on this device.
Status row_fft(Context &c, long long L, const RfftArgs **out)
{
    Status st;
    *out = nullptr;
    auto it = c.rffts.find(L);
    if (it != c.rffts.end())
    {
        *out = &it->second;
        return st;
    }
    RfftArgs A{};
    if (!rfft_shape(L, &A))
    {
        st.code = CHARM_EFUNCARG;
        st.msg = "no longitude transform for grid rows of " +
                 std::to_string(L) +
                 " points (the limit is 147456 points per row).";
        return st;
    }
    const long long H = A.H;
    const size_t nM = (size_t)A.M, nH = (size_t)H;
    // the largest transform of either width, so that no later plan needs
    // a different limit
    CB_CUDA(rfft_set_smem(rfft_smem_bytes(9216)), st);
    void *mem = nullptr;
    cudaError_t ce = cudaSuccess;
    if (A.C > 1)
    {
        const int Mc = A.M / A.C;
        if (rfftc_max_clusters(A.C, Mc) < 1)
        {
            st.code = CHARM_EFUNCARG;
            st.msg = "the longitude transform of rows of " +
                     std::to_string(L) + " points needs clusters of " +
                     std::to_string(A.C) +
                     " CTAs, which this device cannot schedule.";
            return st;
        }
        // tw (Mc), twM (M), w (H), bh (M), ht (H + 1)
        const size_t n_tab = (size_t)Mc + nM + nH + nM + nH + 1;
        CB_CUDA(cudaMalloc(&mem, n_tab * sizeof(double2)), st);
        double2 *tw = static_cast<double2 *>(mem);
        double2 *twM = tw + Mc;
        double2 *w = twM + nM;
        double2 *bh = w + nH;
        double2 *ht = bh + nM;
        A.bh = bh;
        ce = launch_rfftc_tables(A, tw, twM, w, ht, bh, c.stream);
        c.launches += 3;
    }
    else
    {
        const size_t n_tab = nM + (A.direct ? 0 : nH + nM) + nH + 1;
        CB_CUDA(cudaMalloc(&mem, n_tab * sizeof(double2)), st);
        double2 *tw = static_cast<double2 *>(mem);
        double2 *w = A.direct ? nullptr : tw + nM;
        double2 *bh = A.direct ? nullptr : w + nH;
        double2 *ht = A.direct ? tw + nM : bh + nM;
        A.tw = tw;
        A.w = w;
        A.bh = bh;
        A.ht = ht;
        ce = launch_rfft_tables(A, tw, w, ht, bh, c.stream);
        c.launches += A.direct ? 1 : 2;
    }
    if (ce == cudaSuccess)
        ce = cudaStreamSynchronize(c.stream);
    if (ce != cudaSuccess)
    {
        cudaFree(mem);
        st.code = CHARM_EFUNCARG;
        st.msg = std::string("row transform set-up failed: ") +
                 cudaGetErrorString(ce);
        return st;
    }
    c.rffts[L] = A;
    c.rfft_mem[L] = mem;
    *out = &c.rffts[L];
    return st;
}

// Quarter-length plan for synthesis rows of length L = 4 Lq (DH2 grids:
// L = 4 (nmax + 1)), or nullptr: two complex DFTs of length Lq per row
// (rfft.cu, k_rfft_inv4), used where the half-length plan `half` needs
// M = 9216 and Lq has the compile-time Bluestein plan M = 4608 (two CTAs
// per SM instead of one).  Cached under the key -L.
Status row_fft_quarter(Context &c, long long L, const RfftArgs *half,
                       const RfftArgs **out)
{
    Status st;
    *out = nullptr;
    if (!half || half->M != 9216 || half->C != 1 || half->odd || L % 4 != 0)
        return st;
    auto it = c.rffts.find(-L);
    if (it != c.rffts.end())
    {
        *out = it->second.M > 0 ? &it->second : nullptr;
        return st;
    }
    const long long Lq = L / 4;
    RfftArgs A{};
    if (!rfft_shape(2 * Lq, &A) || A.direct || A.M != 4608 || A.C != 1)
    {
        A.M = 0;
        c.rffts[-L] = A;
        return st;
    }
    const size_t nM = (size_t)A.M, nH = (size_t)A.H;
    const size_t n_tab = nM + nH + nM + (nH + 1) + nH;
    void *mem = nullptr;
    CB_CUDA(cudaMalloc(&mem, n_tab * sizeof(double2)), st);
    double2 *tw = static_cast<double2 *>(mem);
    double2 *w = tw + nM;
    double2 *bh = w + nH;
    double2 *ht = bh + nM;
    double2 *w4 = ht + nH + 1;
    A.tw = tw;
    A.w = w;
    A.bh = bh;
    A.ht = ht;
    A.w4 = w4;
    A.quarter = 1;
    cudaError_t ce = rfft_set_smem(rfft_smem_bytes(9216));
    if (ce == cudaSuccess)
        ce = launch_rfft_tables(A, tw, w, ht, bh, c.stream);
    if (ce == cudaSuccess)
        ce = launch_rfft_w4(A.H, w4, c.stream);
    if (ce == cudaSuccess)
        ce = cudaStreamSynchronize(c.stream);
    if (ce != cudaSuccess)
    {
        cudaFree(mem);
        st.code = CHARM_EFUNCARG;
        st.msg = std::string("row transform set-up failed: ") +
                 cudaGetErrorString(ce);
        return st;
    }
    c.launches += 3;
    c.rffts[-L] = A;
    c.rfft_mem[-L] = mem;
    *out = &c.rffts[-L];
    return st;
}

// The plan of a synthesis launch whose spectra stop at kmax: the
// quarter-length one where it was set up and applies (kmax below its
// length), else the half-length one.
const RfftArgs *synth_plan(const RfftArgs *half, const RfftArgs *quarter,
                           long long kmax)
{
    return (quarter && kmax < quarter->H) ? quarter : half;
}

// Triangle pointer of a charm_shc whose columns c[m] lie contiguously as in
// src/shc/shc_init_chunk.c:126-145 (every charm_shc built by CHarm's
// constructors), else null.
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

Status upload_tri(Context &c, double *const *cols, unsigned long shc_nmax,
                  double *dst)
{
    Status st;
    const double *base = contiguous_tri(cols, shc_nmax);
    size_t T = (size_t)(shc_nmax + 1) * (shc_nmax + 2) / 2;
    if (base)
        return stage_h2d(c, dst, base, T * 8);
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
        // a page-locked destination is copied asynchronously (the call's
        // final synchronisation waits for it); a pageable one through the
        // ring, which returns when the copy is done
        if (!is_pageable(base))
        {
            CB_CUDA(cudaMemcpyAsync(const_cast<double *>(base), src, T * 8,
                                    cudaMemcpyDeviceToHost, c.stream), st);
            return st;
        }
        return stage_d2h(c, const_cast<double *>(base), src, T * 8);
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

// Index of column m (C_mm) in an order-major triangle of degree N (CHarm's
// layout, src/shc/shc_init_chunk.c:126-145).
long long tri_start(long long N, long long m)
{
    return (m * (2 * N + 3 - m)) / 2;
}

// The columns m_lo <= m < m_hi of a charm_shc's host columns into a device
// triangle of degree shc_nmax, on stream st (pg: the host triangle is
// pageable, copied through the ring).
Status upload_tri_orders(Context &c, double *const *cols,
                         unsigned long shc_nmax, double *dst, long long m_lo,
                         long long m_hi, cudaStream_t st, int pg)
{
    Status s2;
    if (m_hi <= m_lo)
        return s2;
    const long long N = (long long)shc_nmax;
    const double *base = contiguous_tri(cols, shc_nmax);
    if (base)
    {
        const long long i0 = tri_start(N, m_lo), i1 = tri_start(N, m_hi);
        return stage_h2d(c, dst + i0, base + i0, (size_t)(i1 - i0) * 8, st,
                         pg);
    }
    for (long long m = m_lo; m < m_hi; m++)
        CB_CUDA(cudaMemcpyAsync(dst + tri_start(N, m), cols[m],
                                (size_t)(N + 1 - m) * 8,
                                cudaMemcpyHostToDevice, st),
                s2);
    return s2;
}

// The columns m_lo <= m < m_hi of a device triangle of degree shc_nmax into
// a charm_shc's host columns, on stream st (pg: the host triangle is
// pageable, copied through the ring).
Status download_tri_orders(Context &c, const double *src,
                           unsigned long shc_nmax, double *const *cols,
                           long long m_lo, long long m_hi, cudaStream_t st,
                           int pg)
{
    Status s2;
    if (m_hi <= m_lo)
        return s2;
    const long long N = (long long)shc_nmax;
    const double *base = contiguous_tri(cols, shc_nmax);
    if (base)
    {
        const long long i0 = tri_start(N, m_lo), i1 = tri_start(N, m_hi);
        double *dst = const_cast<double *>(base) + i0;
        // page-locked: asynchronous on st; pageable: through the ring,
        // done when this returns
        if (!pg)
        {
            CB_CUDA(cudaMemcpyAsync(dst, src + i0, (size_t)(i1 - i0) * 8,
                                    cudaMemcpyDeviceToHost, st),
                    s2);
            return s2;
        }
        return stage_d2h(c, dst, src + i0, (size_t)(i1 - i0) * 8, st, 1);
    }
    for (long long m = m_lo; m < m_hi; m++)
        CB_CUDA(cudaMemcpyAsync(cols[m], src + tri_start(N, m),
                                (size_t)(N + 1 - m) * 8,
                                cudaMemcpyDeviceToHost, st),
                s2);
    return s2;
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

// src/misc/misc_arr_chck_symm.c with centre 0
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

// Latitude pairs of a grid: evaluated rows and mirror rows (-1 when none),
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
    size_t nlatdo = symm ? (pnt_nlat + 1 - (even ? 1 : 0)) / 2 : nlat;
    P.row_n.clear();
    P.row_s.clear();
    for (size_t ipv = 0; ipv < nlatdo; ipv++)
    {
        int s;
        if (!symm)
            s = 0;
        else if (quad)
            s = (dh && ipv == 0) ? 0 : (ipv < equator ? 1 : 0);
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

// Latitude pairs per lane of the analysis kernel.  Wider tiles amortise
// the per-degree beta load and the transpose-reduce over more latitudes but
// lower the resident warps (sha_grid.cu); CHARM_B200_SHA_K (1, 2, 4, 6 or
// 8) overrides the choice for tuning.
int choose_k_sha(long long npairs)
{
    static const int forced = [] {
        const char *e = std::getenv("CHARM_B200_SHA_K");
        int k = e ? std::atoi(e) : 0;
        return (k == 1 || k == 2 || k == 4 || k == 6 || k == 8) ? k : 0;
    }();
    if (forced)
        return forced;
    if (npairs < 64)
        return 1;
    if (npairs < 1024)
        return 2;
    return 4;
}

// Autotuner of the synthesis kernel's latitude pairs per lane (the tile is
// 32 K pairs): on the first call of a problem shape every candidate runs
// once on the call's own data, timed with CUDA events on the library
// stream, and the fastest is kept for the process.  The sums of a latitude
// pair do not depend on K, so the choice changes no result.  Shapes with
// nmax < 256 and CHARM_B200_AUTOTUNE=0 keep the built-in choice.
bool autotune_on()
{
    static const bool on = [] {
        const char *e = std::getenv("CHARM_B200_AUTOTUNE");
        return !(e && std::strcmp(e, "0") == 0);
    }();
    return on;
}

// True when tune_shs_k launches nothing for this shape (tuned already, or
// not tuned at all), so that the call's coefficients need not all be on
// the device before its first synthesis launch.
bool shs_k_settled(Context &c, int kgrad, int dr, int dlat, bool rr,
                   long long nmax, int np)
{
    const auto key = std::make_tuple(kgrad, dr, dlat, rr ? 1 : 0, nmax, np);
    return c.tuned.count(key) > 0 || !autotune_on() || nmax < 256;
}

Status tune_shs_k(Context &c, const ShsGridArgs &A0, int kgrad, int dr,
                  int dlat, bool rr, int np, int *K)
{
    Status st;
    const auto key = std::make_tuple(kgrad, dr, dlat, rr ? 1 : 0, A0.nmax, np);
    auto it = c.tuned.find(key);
    if (it != c.tuned.end())
    {
        *K = it->second.first;
        return st;
    }
    if (!autotune_on() || A0.nmax < 256 || A0.nsets > 0)
        return st;
    std::vector<int> cands = kgrad >= 1 || dlat > 0 ? std::vector<int>{1, 2}
                                                    : std::vector<int>{1, 2, 4};
    cudaEvent_t e0 = ev_get(c), e1 = ev_get(c);
    std::vector<std::pair<int, float>> meas;
    int best = *K;
    float best_ms = 0.0f;
    // one untimed launch first (first-use costs of the module, caches)
    cands.insert(cands.begin(), *K);
    bool warm = true;
    for (int k : cands)
    {
        ShsGridArgs A = A0;
        A.ntiles = (np + 32 * k - 1) / (32 * k);
        A.nitems = (long long)(A.nmax + 1) * A.ntiles;
        const int grid = (int)std::min<long long>((A.nitems + 3) / 4,
                                                  (long long)c.num_sms * 8);
        CB_CUDA(cudaMemsetAsync(A.counter, 0, sizeof(unsigned long long),
                                c.stream), st);
        CB_CUDA(cudaEventRecord(e0, c.stream), st);
        CB_CUDA(launch_shs_grid(A, kgrad, dr, dlat, rr, k, std::max(grid, 1),
                                c.stream), st);
        CB_CUDA(cudaEventRecord(e1, c.stream), st);
        CB_CUDA(cudaEventSynchronize(e1), st);
        float ms = 0.0f;
        CB_CUDA(cudaEventElapsedTime(&ms, e0, e1), st);
        c.launches++;
        if (warm)
        {
            warm = false;
            continue;
        }
        meas.emplace_back(k, ms);
        if (best_ms == 0.0f || ms < best_ms)
        {
            best_ms = ms;
            best = k;
        }
    }
    c.ev_pool.push_back(e0);
    c.ev_pool.push_back(e1);
    CB_CUDA(cudaMemsetAsync(A0.counter, 0, sizeof(unsigned long long),
                            c.stream), st);
    c.tuned[key] = std::make_pair(best, meas);
    *K = best;
    return st;
}

Status finish(Context &c, unsigned *d_status)
{
    Status st;
    if (c.capturing)
        return st;   // read by batch_graph_launch after each replay
    // into page-locked memory, so the copy is queued like a kernel and the
    // one synchronisation below covers both
    *c.h_status = 0u;
    CB_CUDA(cudaMemcpyAsync(c.h_status, d_status, sizeof(unsigned),
                            cudaMemcpyDeviceToHost, c.stream), st);
    CB_CUDA(cudaStreamSynchronize(c.stream), st);
    const unsigned h_status = *c.h_status;
    if (c.timing)
        resolve_timers(c);
    if (h_status)
    {
        st.code = CHARM_EFUNCARG;
        st.msg = "A GPU kernel reported an internal error (status " +
                 std::to_string(h_status) + ").";
        if (h_status == DEV_ERR_TC_RANGE)
            st.msg = "The split-precision synthesis met a Legendre value "
                     "outside its fixed-point range (status " +
                     std::to_string(h_status) + ").";
    }
    return st;
}

Status status_words(Context &c, unsigned **d_status,
                    unsigned long long **d_counter)
{
    Status st;
    void *p = nullptr;
    CB_TRY(buf(c, "status", 256, &p));
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
void mur_dorder(double mu, double R, int kgrad, int dr, int dlat, int dlon,
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
    double rpow = R;
    for (int i = 1; i <= *dorder; i++)
        rpow *= R;
    *mur = mu / rpow;
}

// Coefficients entering a synthesis: host columns (CHarm's charm_shc) or a
// device-resident triangle of degree nmax_shc.
struct CoefIn
{
    unsigned long nmax;
    double mu, r;
    double *const *hc = nullptr, *const *hs = nullptr;
    const double *dc = nullptr, *ds = nullptr;
};

Status coef_to_device(Context &c, const CoefIn &in, unsigned long nmax,
                      const Tabs &tab, double2 **dcs)
{
    Status st;
    const long long Ts = (long long)(in.nmax + 1) * (in.nmax + 2) / 2;
    const long long T = (long long)(nmax + 1) * (nmax + 2) / 2;
    CB_TRY(dbuf(c, "cs", (size_t)T, dcs));
    const double *src_c = in.dc, *src_s = in.ds;
    if (!src_c)
    {
        double *raw = nullptr;
        CB_TRY(dbuf(c, "shc_in", (size_t)(2 * Ts), &raw));
        CB_TRY(upload_tri(c, in.hc, in.nmax, raw));
        CB_TRY(upload_tri(c, in.hs, in.nmax, raw + Ts));
        src_c = raw;
        src_s = raw + Ts;
    }
    Scope sc(c, TIMER_PREP);
    CB_CUDA(launch_scale_cs((long long)nmax, (long long)in.nmax, src_c, src_s,
                            tab.tc, *dcs, c.stream), st);
    return st;
}

// ---------------------------------------------------------------------------
// Grid synthesis
// ---------------------------------------------------------------------------
// Rows of the latitude pairs [p0, p1) as two contiguous ranges: north rows
// [r[0], r[1]) and mirror rows [r[2], r[3]) (empty when there are none).
// False when they do not form two disjoint contiguous ranges.
bool band_rows(const Pairs &P, int p0, int p1, int nlat, int r[4])
{
    int nmin = nlat, nmx = -1, nn = 0, smin = nlat, smx = -1, ns = 0;
    for (int p = p0; p < p1; p++)
    {
        const int a = P.row_n[p], b = P.row_s[p];
        if (a >= 0 && a < nlat)
        {
            nmin = std::min(nmin, a);
            nmx = std::max(nmx, a);
            nn++;
        }
        if (b >= 0 && b < nlat)
        {
            smin = std::min(smin, b);
            smx = std::max(smx, b);
            ns++;
        }
    }
    if (nn == 0 || nmx - nmin + 1 != nn)
        return false;
    r[0] = nmin;
    r[1] = nmx + 1;
    r[2] = r[3] = 0;
    if (ns > 0)
    {
        if (smx - smin + 1 != ns || !(smx < nmin || smin > nmx))
            return false;
        r[2] = smin;
        r[3] = smx + 1;
    }
    return true;
}

// Bands of consecutive tiles (or tile groups) for the overlap of the grid's
// host copies with the kernels: nb bands of units [u0, u1) of `units`, each
// unit covering `per` latitude pairs; their row ranges in `rows`.  Returns
// the number of bands, 1 when the rows do not split into contiguous
// ranges.
int grid_bands(const Pairs &P, int nlat, int units, int per, int nb,
               std::vector<std::array<int, 6>> &bands)
{
    const int np = (int)P.row_n.size();
    bands.clear();
    nb = std::max(1, std::min(nb, units));
    if (nb < 2)
        return 1;
    for (int b = 0; b < nb; b++)
    {
        const int u0 = (int)((long long)b * units / nb);
        const int u1 = (int)((long long)(b + 1) * units / nb);
        const int p0 = std::min(np, u0 * per), p1 = std::min(np, u1 * per);
        int r[4];
        if (p1 <= p0 || !band_rows(P, p0, p1, nlat, r))
        {
            bands.clear();
            return 1;
        }
        bands.push_back({u0, u1, r[0], r[1], r[2], r[3]});
    }
    return nb;
}

Status shs_grid(Context &c, const charm_point *pnt, const CoefIn &in,
                unsigned long nmax, int kgrad, int dr, int dlat, int dlon,
                double **f, double *d_f)
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
    // src/shs/shs_grd_point_fft_check.c:30-55
    double dlon_step = nlon > 1 ? pnt->lon[1] - pnt->lon[0] : 0.0;
    bool use_fft = (nlon >= 1) && ((nlon - 1) / 2 >= nmax) &&
                   nearly_equal(pnt->lon[0], 0.0, thr) &&
                   nearly_equal(pnt->lon[nlon - 1] + dlon_step, 2.0 * PI, thr);

    // r == R everywhere selects the faster kernels (shs_r_eq_rref.c)
    const bool r_eq = all_nearly_equal(pnt->r, nlat, in.r, thr);
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
    mur_dorder(in.mu, in.r, kgrad, dr, dlat, dlon, &mur, &dorder, &npar);

    // per-pair geometry, staged through pinned memory (one upload)
    size_t geo_bytes = (size_t)np * (3 * 8 + 2 * 4);
    void *hp = nullptr;
    CB_TRY(pinned(c, geo_bytes, &hp));
    double *ht = static_cast<double *>(hp);
    double *hu = ht + np;
    double *hrho = hu + np;
    int *hrn = reinterpret_cast<int *>(hrho + np);
    int *hrs = hrn + np;
    for (int p = 0; p < np; p++)
    {
        double la = pnt->lat[P.row_n[p]];
        sincos(la, &ht[p], &hu[p]);
        hrho[p] = r_eq ? 1.0 : in.r / pnt->r[P.row_n[p]];
        hrn[p] = P.row_n[p];
        hrs[p] = P.row_s[p];
    }
    void *dgeo = nullptr;
    CB_TRY(buf(c, "geo", geo_bytes, &dgeo));
    CB_CUDA(cudaMemcpyAsync(dgeo, hp, geo_bytes, cudaMemcpyHostToDevice,
                            c.stream), st);
    const double *dt = static_cast<const double *>(dgeo);
    const double *du = dt + np;
    const double *drho = du + np;
    const int *drn = reinterpret_cast<const int *>(drho + np);
    const int *drs = drn + np;

    Tabs tab;
    CB_TRY(tables(c, (long long)nmax, &tab));
    // Host coefficients of a call whose grid goes to the host are uploaded
    // later, in bands of orders overlapped with the synthesis of the first
    // band of latitudes (when the call runs in bands), else all now.
    double2 *dcs = nullptr;
    double *raw = nullptr;
    const long long Ts = (long long)(in.nmax + 1) * (in.nmax + 2) / 2;
    bool coef_later =
        !in.dc && !d_f &&
        shs_k_settled(c, kgrad, dr, dlat, !r_eq, (long long)nmax, np);
    if (coef_later)
    {
        CB_TRY(dbuf(c, "cs", (size_t)((nmax + 1) * (nmax + 2) / 2), &dcs));
        CB_TRY(dbuf(c, "shc_in", (size_t)(2 * Ts), &raw));
    }
    else
        CB_TRY(coef_to_device(c, in, nmax, tab, &dcs));

    // lumped coefficients
    const int ldf = use_fft ? (int)(nlon / 2 + 1) : (int)(nmax + 1);
    double2 *lc = nullptr;
    CB_TRY(dbuf(c, "lumped", (size_t)npar * nlat * ldf, &lc));
    double *fg = d_f;
    // the even-row transform stores pairs of doubles: a device output that
    // is not on a 16-byte boundary is written through the aligned staging
    // grid and copied once
    double *f_dev_unaligned = nullptr;
    if (fg && use_fft && nlon % 2 == 0 &&
        reinterpret_cast<uintptr_t>(fg) % 16 != 0)
    {
        f_dev_unaligned = fg;
        fg = nullptr;
    }
    if (!fg)
        CB_TRY(dbuf(c, "fgrid", (size_t)npar * nlat * nlon, &fg));
    const RfftArgs *rf = nullptr, *rfq = nullptr;
    if (use_fft)
    {
        CB_TRY(row_fft(c, (long long)nlon, &rf));
        CB_TRY(row_fft_quarter(c, (long long)nlon, rf, &rfq));
    }
    unsigned *d_status;
    unsigned long long *d_counter;
    CB_TRY(status_words(c, &d_status, &d_counter));

    int K = choose_k(kgrad, dlat, np);
    int ntiles = (np + 32 * K - 1) / (32 * K);
    ShsGridArgs A{};
    A.nmax = (long long)nmax;
    A.npairs = np;
    A.ntiles = ntiles;
    A.nitems = (long long)(nmax + 1) * ntiles;
    A.tb = tab.tb;
    A.tmul = tab.tmul;
    A.ldmul = tab.ldmul;
    A.sg = tab.sg;
    A.cs = dcs;
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
    // autotuned tile (first call of this shape)
    {
        int Kt = K;
        CB_TRY(tune_shs_k(c, A, kgrad, dr, dlat, !r_eq, np, &Kt));
        if (Kt != K)
        {
            K = Kt;
            ntiles = (np + 32 * K - 1) / (32 * K);
            A.ntiles = ntiles;
            A.nitems = (long long)(nmax + 1) * ntiles;
        }
    }

    // Host output through the row transform: bands of latitude tiles, each
    // band's rows copied to the host (copy stream) while the next band is
    // synthesised; the sums of every item are the same as in one launch.
    std::vector<std::array<int, 6>> bands;
    const int nband =
        (!d_f && rf) ? grid_bands(P, (int)nlat, ntiles, 32 * K,
                                  ntiles >= 6 ? SHS_LAT_BANDS : 2, bands)
                     : 1;
    if (coef_later && nband <= 1)
    {
        // no bands: every coefficient now
        CB_TRY(upload_tri(c, in.hc, in.nmax, raw));
        CB_TRY(upload_tri(c, in.hs, in.nmax, raw + Ts));
        Scope sc(c, TIMER_PREP);
        CB_CUDA(launch_scale_cs((long long)nmax, (long long)in.nmax, raw,
                                raw + Ts, tab.tc, dcs, c.stream),
                st);
        coef_later = false;
    }
    if (nband > 1)
    {
        unsigned long long *bcnt = nullptr;
        CB_TRY(dbuf(c, "band_counters", 16, &bcnt));
        CB_CUDA(cudaMemsetAsync(bcnt, 0, 16 * sizeof(unsigned long long),
                                c.stream), st);
        // orders in up to SHS_ORD_BANDS bands of about equal numbers of
        // coefficients
        std::vector<long long> mb{0};
        if (coef_later)
        {
            const long long T = (long long)(nmax + 1) * (nmax + 2) / 2;
            for (int k = 1; k < SHS_ORD_BANDS; k++)
            {
                long long m = mb.back();
                while (m <= (long long)nmax &&
                       tri_start((long long)nmax, m) < k * T / SHS_ORD_BANDS)
                    m++;
                if (m > mb.back() && m <= (long long)nmax)
                    mb.push_back(m);
            }
            // the copy stream starts after everything before it on the
            // stream; band k of the orders: copy (copy stream), then scale
            CB_CUDA(cudaEventRecord(c.band_ev[EV_START], c.stream), st);
            CB_CUDA(cudaStreamWaitEvent(c.copy_stream, c.band_ev[EV_START], 0), st);
        }
        mb.push_back((long long)nmax + 1);
        const int nob = (int)mb.size() - 1;
        if (coef_later)
            for (int k = 0; k < nob; k++)
            {
                CB_TRY(upload_tri_orders(c, in.hc, in.nmax, raw, mb[k],
                                         mb[k + 1], c.copy_stream, 0));
                CB_TRY(upload_tri_orders(c, in.hs, in.nmax, raw + Ts, mb[k],
                                         mb[k + 1], c.copy_stream, 0));
                CB_CUDA(cudaEventRecord(c.band_ev[EV_ORD0 + k], c.copy_stream),
                        st);
            }
        for (int b = 0; b < nband; b++)
        {
            const auto &bd = bands[b];
            // the first band synthesises each band of orders as soon as its
            // coefficients are on the device
            const bool split = b == 0 && coef_later;
            for (int k = 0; k < (split ? nob : 1); k++)
            {
                if (split)
                {
                    CB_CUDA(cudaStreamWaitEvent(c.stream, c.band_ev[EV_ORD0 + k],
                                                0),
                            st);
                    Scope sc(c, TIMER_PREP);
                    CB_CUDA(launch_scale_cs_orders(
                                (long long)nmax, (long long)in.nmax, raw,
                                raw + Ts, tab.tc, dcs, mb[k], mb[k + 1],
                                c.stream),
                            st);
                }
                ShsGridArgs Ab = A;
                Ab.tile0 = bd[0];
                Ab.ntiles = bd[1] - bd[0];
                Ab.m0 = split ? mb[k] : 0;
                Ab.nitems = (long long)(split ? mb[k + 1] - mb[k]
                                              : (long long)nmax + 1) *
                            Ab.ntiles;
                Ab.counter = bcnt + (split ? 8 + k : b);
                const int gb = (int)std::min<long long>(
                    (Ab.nitems + 3) / 4, (long long)c.num_sms * 8);
                Scope sc(c, TIMER_SHS);
                CB_CUDA(launch_shs_grid(Ab, kgrad, dr, dlat, !r_eq, K,
                                        std::max(gb, 1), c.stream), st);
            }
            for (int q = 0; q < npar; q++)
                for (int h = 0; h < 2; h++)
                {
                    const int r0 = bd[2 + 2 * h], r1 = bd[3 + 2 * h];
                    if (r1 <= r0)
                        continue;
                    RfftArgs R = *synth_plan(rf, rfq, (long long)nmax);
                    R.nrows = r1 - r0;
                    R.x = fg + ((size_t)q * nlat + r0) * nlon;
                    R.ldx = (long long)nlon;
                    R.X = lc + ((size_t)q * nlat + r0) * ldf;
                    R.ldX = ldf;
                    R.kmax = (int)nmax;
                    Scope sc(c, TIMER_FFT);
                    CB_CUDA(launch_rfft(R, true, c.stream), st);
                }
            CB_CUDA(cudaEventRecord(c.band_ev[EV_LAT0 + b], c.stream), st);
            CB_CUDA(cudaStreamWaitEvent(c.copy_stream, c.band_ev[EV_LAT0 + b],
                                        0),
                    st);
            for (int q = 0; q < npar; q++)
                for (int h = 0; h < 2; h++)
                {
                    const int r0 = bd[2 + 2 * h], r1 = bd[3 + 2 * h];
                    if (r1 > r0)
                        CB_CUDA(cudaMemcpyAsync(
                                    f[q] + (size_t)r0 * nlon,
                                    fg + ((size_t)q * nlat + r0) * nlon,
                                    (size_t)(r1 - r0) * nlon * 8,
                                    cudaMemcpyDeviceToHost, c.copy_stream),
                                st);
                }
        }
        CB_CUDA(cudaStreamSynchronize(c.copy_stream), st);
        return finish(c, d_status);
    }

    int grid = (int)std::min<long long>((A.nitems + 3) / 4,
                                        (long long)c.num_sms * 8);
    {
        Scope sc(c, TIMER_SHS);
        CB_CUDA(launch_shs_grid(A, kgrad, dr, dlat, !r_eq, K,
                                std::max(grid, 1), c.stream), st);
    }

    // longitude sums into the output grid(s)
    if (rf)
    {
        RfftArgs R = *synth_plan(rf, rfq, (long long)nmax);
        R.nrows = (long long)npar * nlat;
        R.x = fg;
        R.ldx = (long long)nlon;
        R.X = lc;
        R.ldX = ldf;
        R.kmax = (int)nmax;
        Scope sc(c, TIMER_FFT);
        CB_CUDA(launch_rfft(R, true, c.stream), st);
    }
    else
    {
        double *dlon_arr = nullptr;
        CB_TRY(dbuf(c, "lon", nlon, &dlon_arr));
        CB_CUDA(cudaMemcpyAsync(dlon_arr, pnt->lon, nlon * 8,
                                cudaMemcpyHostToDevice, c.stream), st);
        Scope sc(c, TIMER_LON);
        CB_CUDA(launch_lon_direct(npar, (int)nlat, (int)nlon, (long long)nmax,
                                  lc, ldf, dlon_arr, fg, c.stream), st);
    }
    if (f_dev_unaligned)
        CB_CUDA(cudaMemcpyAsync(f_dev_unaligned, fg,
                                (size_t)npar * nlat * nlon * 8,
                                cudaMemcpyDeviceToDevice, c.stream), st);
    if (!d_f)
        for (int q = 0; q < npar; q++)
            CB_CUDA(cudaMemcpyAsync(f[q], fg + (size_t)q * nlat * nlon,
                                    nlat * nlon * 8, cudaMemcpyDeviceToHost,
                                    c.stream), st);
    return finish(c, d_status);
}

// ---------------------------------------------------------------------------
// Scattered synthesis
// ---------------------------------------------------------------------------
Status shs_sctr(Context &c, const charm_point *pnt, const CoefIn &in,
                unsigned long nmax, int kgrad, int dr, int dlat, int dlon,
                double **f, double *d_f)
{
    Status st;
    const size_t npt = pnt->nlat;
    const bool r_eq =
        all_nearly_equal(pnt->r, npt, in.r, charm_glob_threshold);
    double mur;
    int dorder, npar;
    mur_dorder(in.mu, in.r, kgrad, dr, dlat, dlon, &mur, &dorder, &npar);
    Tabs tab;
    CB_TRY(tables(c, (long long)nmax, &tab));
    double2 *dcs = nullptr;
    CB_TRY(coef_to_device(c, in, nmax, tab, &dcs));
    double *dpts = nullptr;
    CB_TRY(dbuf(c, "sctr_pts", 3 * npt, &dpts));
    CB_TRY(stage_h2d(c, dpts, pnt->lat, npt * 8));
    CB_TRY(stage_h2d(c, dpts + npt, pnt->lon, npt * 8));
    if (!r_eq)
        CB_TRY(stage_h2d(c, dpts + 2 * npt, pnt->r, npt * 8));
    double *fo = d_f;
    if (!fo)
        CB_TRY(dbuf(c, "sctr_f", (size_t)npar * npt, &fo));
    unsigned *d_status;
    unsigned long long *d_counter;
    CB_TRY(status_words(c, &d_status, &d_counter));
    const int K = choose_k(kgrad, dlat, (long long)npt);
    SctrArgs A{};
    A.nmax = (long long)nmax;
    A.npoint = (long long)npt;
    A.ntiles = ((long long)npt + 32 * K - 1) / (32 * K);
    A.tb = tab.tb;
    A.tmul = tab.tmul;
    A.ldmul = tab.ldmul;
    A.sg = tab.sg;
    A.cs = dcs;
    A.dm = tab.dm;
    A.lat = dpts;
    A.lon = dpts + npt;
    A.r = dpts + 2 * npt;
    A.R = in.r;
    A.f = fo;
    A.mur = mur;
    A.dlon = dlon;
    A.polar_thr = polar_threshold(nmax);
    A.counter = d_counter;
    A.status = d_status;
    int grid = (int)std::min<long long>((A.ntiles + 3) / 4,
                                        (long long)c.num_sms * 8);
    {
        Scope sc(c, TIMER_SCTR);
        CB_CUDA(launch_sctr(A, kgrad, dr, dlat, !r_eq, K, std::max(grid, 1),
                            c.stream), st);
    }
    if (!d_f)
        for (int q = 0; q < npar; q++)
        {
            if (!is_pageable(f[q]))
                CB_CUDA(cudaMemcpyAsync(f[q], fo + (size_t)q * npt, npt * 8,
                                        cudaMemcpyDeviceToHost, c.stream),
                        st);
            else
                CB_TRY(stage_d2h(c, f[q], fo + (size_t)q * npt, npt * 8));
        }
    return finish(c, d_status);
}

// Grid checks, latitude pairs and their geometry on the device for the
// batched syntheses: FFT longitudes are required; r may vary by latitude
// (pairs only where the mirror row has the same radius).
struct BatchGeo
{
    Pairs P;
    int np = 0;
    bool r_eq = true;
    const double *dt = nullptr;   // t[np], u[np], rho[np], row_n, row_s
};

Status batch_geometry(Context &c, const charm_point *pnt, unsigned long N,
                      double R, BatchGeo *G)
{
    Status st;
    const double thr = charm_glob_threshold, thr2 = charm_glob_threshold2;
    const size_t nlat = pnt->nlat, nlon = pnt->nlon;
    if (pnt->type == CHARM_CRD_POINT_GRID && nlon > 1)
    {
        double step = pnt->lon[1] - pnt->lon[0];
        for (size_t j = 1; j < nlon; j++)
            if (!(step > 0.0) ||
                !nearly_equal(step, pnt->lon[j] - pnt->lon[j - 1], thr2))
            {
                st.code = CHARM_EFUNCARG;
                st.msg = "\"pnt->lon\" is not a linearly increasing array "
                         "within the \"threshold2\".";
                return st;
            }
    }
    double dlon_step = nlon > 1 ? pnt->lon[1] - pnt->lon[0] : 0.0;
    const bool use_fft = (nlon >= 1) && ((nlon - 1) / 2 >= N) &&
                         nearly_equal(pnt->lon[0], 0.0, thr) &&
                         nearly_equal(pnt->lon[nlon - 1] + dlon_step, 2.0 * PI,
                                      thr);
    if (!use_fft)
    {
        st.code = CHARM_EFUNCARG;
        st.msg = "The batched synthesis needs a grid with FFT longitudes "
                 "(0, 2 pi / nlon, ..., nlon > 2 nmax).";
        return st;
    }
    const bool r_eq = all_nearly_equal(pnt->r, nlat, R, thr);
    Pairs &P = G->P;
    grid_pairs(pnt, thr2, true, P);
    if (!r_eq)
        for (size_t p = 0; p < P.row_n.size(); p++)
            if (P.row_s[p] >= 0 && P.row_s[p] < (int)nlat &&
                pnt->r[P.row_s[p]] != pnt->r[P.row_n[p]])
            {
                grid_pairs(pnt, thr2, false, P);
                break;
            }
    const int np = (int)P.row_n.size();
    size_t geo_bytes = (size_t)np * (3 * 8 + 2 * 4);
    void *hp = nullptr;
    CB_TRY(pinned(c, geo_bytes, &hp));
    double *ht = static_cast<double *>(hp);
    double *hu = ht + np;
    double *hrho = hu + np;
    int *hrn = reinterpret_cast<int *>(hrho + np);
    int *hrs = hrn + np;
    for (int p = 0; p < np; p++)
    {
        double la = pnt->lat[P.row_n[p]];
        sincos(la, &ht[p], &hu[p]);
        hrho[p] = r_eq ? 1.0 : R / pnt->r[P.row_n[p]];
        hrn[p] = P.row_n[p];
        hrs[p] = P.row_s[p];
    }
    void *dgeo = nullptr;
    CB_TRY(buf(c, "geo", geo_bytes, &dgeo));
    CB_CUDA(cudaMemcpyAsync(dgeo, hp, geo_bytes, cudaMemcpyHostToDevice,
                            c.stream), st);
    const double *dt = static_cast<const double *>(dgeo);

    G->np = np;
    G->r_eq = r_eq;
    G->dt = dt;
    return st;
}

// ---------------------------------------------------------------------------
// Batched synthesis: many coefficient sets on one grid
// ---------------------------------------------------------------------------
// All sets share the grid, its geometry, the recurrence tables of the
// largest degree and one persistent launch per derivative kind; each work
// item (set, order, latitude tile) stops at its set's own nmax.  kgrad 0:
// potential, 1: grad1, 2: grad2, 3: all ten quantities (potential, grad1
// x y z, grad2 xx xy xz yy yz zz, in CHarm's output order) per set.
Status shs_batch(Context &c, const charm_point *pnt, size_t nsets,
                 const unsigned long *nmax_v, const unsigned long *shc_nmax_v,
                 const double *mu_v, double R, const double *const *d_c,
                 const double *const *d_s, int kgrad, double *const *d_f)
{
    Status st;
    const double thr = charm_glob_threshold, thr2 = charm_glob_threshold2;
    const size_t nlat = pnt->nlat, nlon = pnt->nlon;
    unsigned long N = 0;
    for (size_t j = 0; j < nsets; j++)
        N = std::max(N, nmax_v[j]);
    BatchGeo G;
    CB_TRY(batch_geometry(c, pnt, N, R, &G));
    const Pairs &P = G.P;
    const int np = G.np;
    const bool r_eq = G.r_eq;
    const double *dt = G.dt;
    (void)thr;
    (void)thr2;
    (void)P;

    Tabs tab;
    CB_TRY(tables(c, (long long)N, &tab));
    const long long T = (long long)(N + 1) * (N + 2) / 2;
    double2 *cs_all = nullptr;
    CB_TRY(dbuf(c, "batch_cs", (size_t)nsets * T, &cs_all));
    for (size_t j = 0; j < nsets; j++)
    {
        Scope sc(c, TIMER_PREP);
        CB_CUDA(launch_scale_cs_set((long long)N, (long long)nmax_v[j],
                                    (long long)shc_nmax_v[j], d_c[j], d_s[j],
                                    tab.tc, cs_all + (size_t)j * T, c.stream),
                st);
    }
    const RfftArgs *rf = nullptr, *rfq = nullptr;
    CB_TRY(row_fft(c, (long long)nlon, &rf));
    CB_TRY(row_fft_quarter(c, (long long)nlon, rf, &rfq));
    const int ldf = (int)(nlon / 2 + 1);
    const size_t grid_sz = nlat * nlon;
    unsigned *d_status;
    unsigned long long *d_counter;
    CB_TRY(status_words(c, &d_status, &d_counter));

    // derivative kinds of this call and where their components go in the
    // caller's per-set output (CHarm's order after its pointer reordering,
    // src/shs/shs_point_gradn.c:133-165)
    struct Kind
    {
        int kgrad, npar, base;
        int slot[6];
    };
    std::vector<Kind> kinds;
    const Kind K0{0, 1, 0, {0}};
    const Kind K1{1, 3, 0, {1, 2, 0}};
    const Kind K2{2, 6, 0, {3, 4, 1, 5, 2, 0}};
    if (kgrad == 0 || kgrad == 3)
        kinds.push_back(K0);
    if (kgrad == 1 || kgrad == 3)
    {
        kinds.push_back(K1);
        kinds.back().base = kgrad == 3 ? 1 : 0;
    }
    if (kgrad == 2 || kgrad == 3)
    {
        kinds.push_back(K2);
        kinds.back().base = kgrad == 3 ? 4 : 0;
    }
    const int ncomp = kgrad == 3 ? 10 : kinds[0].npar;
    for (const Kind &kd : kinds)
    {
        const int kg = kd.kgrad, npar = kd.npar;
        const int dd = kg;   // grad kinds: dr = dlat = dlon = kgrad
        // sets per launch, bounded by the lumped-coefficient buffer (8 GB)
        const size_t per_set = (size_t)npar * nlat * ldf * sizeof(double2);
        size_t bsz = std::max<size_t>(1, ((size_t)8 << 30) / per_set);
        bsz = std::min(bsz, nsets);
        double2 *lc = nullptr;
        CB_TRY(dbuf(c, "batch_lumped", bsz * per_set / sizeof(double2), &lc));
        BatchSet *dsets = nullptr;
        CB_TRY(dbuf(c, "batch_sets", bsz, &dsets));
        std::vector<BatchSet> hsets(bsz);
        const int K = choose_k(kg, dd, np);
        const int ntiles = (np + 32 * K - 1) / (32 * K);
        for (size_t j0 = 0; j0 < nsets; j0 += bsz)
        {
            const size_t nb = std::min(bsz, nsets - j0);
            long long items = 0;
            for (size_t b = 0; b < nb; b++)
            {
                const size_t j = j0 + b;
                double mur;
                int dorder, npar_j;
                mur_dorder(mu_v[j], R, kg, dd, dd, dd, &mur, &dorder,
                           &npar_j);
                hsets[b].nmax = (long long)nmax_v[j];
                hsets[b].item0 = items;
                hsets[b].cs = cs_all + j * T;
                hsets[b].out = lc + b * (per_set / sizeof(double2));
                hsets[b].mur = mur;
                hsets[b].polar_thr = polar_threshold(nmax_v[j]);
                items += (long long)(nmax_v[j] + 1) * ntiles;
            }
            CB_TRY(h2d_small(c, dsets, hsets.data(), nb * sizeof(BatchSet)));
            CB_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(unsigned long long),
                                    c.stream), st);
            ShsGridArgs A{};
            A.nmax = (long long)N;
            A.npairs = np;
            A.ntiles = ntiles;
            A.nitems = items;
            A.tb = tab.tb;
            A.tmul = tab.tmul;
            A.ldmul = tab.ldmul;
            A.sg = tab.sg;
            A.t = dt;
            A.u = dt + np;
            A.rho = dt + 2 * np;
            A.row_n = reinterpret_cast<const int *>(dt + 3 * np);
            A.row_s = A.row_n + np;
            A.nlat = (int)nlat;
            A.ldf = ldf;
            A.fft_pack = 1;
            A.dlon = dd;
            A.counter = d_counter;
            A.status = d_status;
            A.sets = dsets;
            A.nsets = (int)nb;
            int grid = (int)std::min<long long>((items + 3) / 4,
                                                (long long)c.num_sms * 8);
            {
                Scope sc(c, TIMER_SHS);
                CB_CUDA(launch_shs_grid(A, kg, dd, dd, !r_eq, K,
                                        std::max(grid, 1), c.stream), st);
            }
            // longitude transforms, component by component into the
            // caller's output slots
            for (size_t b = 0; b < nb; b++)
                for (int q = 0; q < npar; q++)
                {
                    double *dst = d_f[j0 + b] +
                                  (size_t)(kd.base + kd.slot[q]) * grid_sz;
                    double2 *src = lc + b * (per_set / sizeof(double2)) +
                                   (size_t)q * nlat * ldf;
                    if (rf->odd || reinterpret_cast<uintptr_t>(dst) % 16 == 0)
                    {
                        RfftArgs R2 = *synth_plan(
                            rf, rfq, (long long)nmax_v[j0 + b]);
                        R2.nrows = (long long)nlat;
                        R2.x = dst;
                        R2.ldx = (long long)nlon;
                        R2.X = src;
                        R2.ldX = ldf;
                        // orders above this set's degree are not written
                        // by the kernel (the buffer is reused): the row
                        // transform takes them as zero
                        R2.kmax = (int)nmax_v[j0 + b];
                        Scope sc(c, TIMER_FFT);
                        CB_CUDA(launch_rfft(R2, true, c.stream), st);
                    }
                    else
                    {
                        st.code = CHARM_EFUNCARG;
                        st.msg = "batched synthesis outputs must start on "
                                 "a 16-byte boundary";
                        return st;
                    }
                }
            // the set descriptors and the lumped buffer are reused by the
            // next sub-batch: wait for this one (stream order suffices
            // inside a captured graph, whose uploads have their own copies)
            if (!c.capturing)
                CB_CUDA(cudaStreamSynchronize(c.stream), st);
        }
    }
    (void)ncomp;
    return finish(c, d_status);
}

// ---------------------------------------------------------------------------
// Batched synthesis with the degree sums on the tensor cores (shs_tc.cu)
// ---------------------------------------------------------------------------
// The potential of up to SHS_TC_SETS sets per launch: their coefficients
// are cut into INT8 digit tiles once per call, one persistent launch forms
// the lumped coefficients of all sets for every (order, 128-pair tile) and
// the row transforms follow per set.  Same grids and outputs as
// shs_batch's kgrad 0.
// kgrad 0: the potential, SHS_TC_SETS sets per launch; kgrad 1, 2 or 3:
// the gradient families (shs_tc.cu), SHS_TC_GRAD_SETS sets per launch, of
// which grad1 (kgrad 1), grad2 (2) or all ten quantities (3) are written,
// in the batched FP64 path's component order.
Status shs_batch_tc(Context &c, const charm_point *pnt, size_t nsets,
                    const unsigned long *nmax_v,
                    const unsigned long *shc_nmax_v, const double *mu_v,
                    double R, const double *const *d_c,
                    const double *const *d_s, double *const *d_f,
                    int kgrad = 0)
{
    Status st;
    const bool grad = kgrad != 0;
    const size_t per_launch = grad ? SHS_TC_GRAD_SETS : SHS_TC_SETS;
    const size_t nlat = pnt->nlat, nlon = pnt->nlon;
    unsigned long N = 0;
    for (size_t j = 0; j < nsets; j++)
        N = std::max(N, nmax_v[j]);
    if (polar_threshold(N) >= 0.0)
    {
        st.code = CHARM_EFUNCARG;
        st.msg = "The split-precision batched synthesis does not apply the "
                 "polar optimisation; switch it off.";
        return st;
    }
    BatchGeo G;
    CB_TRY(batch_geometry(c, pnt, N, R, &G));
    const int np = G.np;
    const double *dt = G.dt;

    Tabs tab;
    CB_TRY(tables(c, (long long)N, &tab));
    const int ld = tab.ldmul * 64;
    double *btp = nullptr;
    CB_TRY(dbuf(c, "tc_btab", (size_t)(N + 1) * ld * 2, &btp));
    double *ctp = btp + (size_t)(N + 1) * ld;
    if (c.tcp_nmax != (long long)N)
    {
        c.epoch++;
        Scope sc(c, TIMER_TABLES);
        CB_CUDA(launch_tc_ctab((long long)N, ld, tab.tb, tab.tc, btp, ctp,
                               c.stream), st);
        c.tcp_nmax = (long long)N;
    }
    // sets in order of decreasing degree, so that each launch of up to
    // SHS_TC_SETS sets stops at a degree close to all of its sets'
    std::vector<size_t> ord(nsets);
    for (size_t j = 0; j < nsets; j++)
        ord[j] = j;
    std::stable_sort(ord.begin(), ord.end(), [&](size_t a, size_t b) {
        return nmax_v[a] > nmax_v[b];
    });
    // chunks of 64 degrees per order, and where each order's tiles start
    // (for the largest degree; a launch of lower degree uses a prefix of
    // the same layout rebuilt for its own degree)
    std::vector<long long> h0(N + 2);
    auto chunk_layout = [&](unsigned long Ng) {
        h0[0] = 0;
        for (unsigned long m = 0; m <= Ng; m++)
            h0[m + 1] = h0[m] + (long long)((Ng - m + 64) / 64);
        return h0[Ng + 1];
    };
    const long long nchunks = chunk_layout(N);
    long long *d_chunk0 = nullptr;
    CB_TRY(dbuf(c, "tc_chunk0", h0.size(), &d_chunk0));
    int *d_ecol = nullptr;
    CB_TRY(dbuf(c, "tc_ecol", (size_t)(N + 1) * 32, &d_ecol));
    void *bdig = nullptr;
    CB_TRY(buf(c, "tc_bdig", (size_t)nchunks * shs_tc_chunk_bytes(), &bdig));

    const RfftArgs *rf = nullptr, *rfq = nullptr;
    CB_TRY(row_fft(c, (long long)nlon, &rf));
    CB_TRY(row_fft_quarter(c, (long long)nlon, rf, &rfq));
    const int ldf = (int)(nlon / 2 + 1);
    const size_t per_q = nlat * (size_t)ldf;
    const size_t per_set = (grad ? 10 : 1) * per_q;
    const size_t bsz = std::min<size_t>(nsets, per_launch);
    double2 *lc = nullptr;
    CB_TRY(dbuf(c, "batch_lumped", bsz * per_set, &lc));
    // lumped array q of a set -> component slot of the caller's output
    // (V; grad1 l r p -> y z x; grad2 ll lr lp rr rp pp -> yy yz xy zz xz
    // xx, CHarm's order after src/shs/shs_point_gradn.c:133-165), or -1
    int slot[10];
    for (int q = 0; q < 10; q++)
        slot[q] = -1;
    {
        const int s1[3] = {1, 2, 0}, s2[6] = {3, 4, 1, 5, 2, 0};
        if (kgrad == 0 || kgrad == 3)
            slot[0] = 0;
        for (int q = 0; q < 3; q++)
            if (kgrad == 1 || kgrad == 3)
                slot[1 + q] = (kgrad == 3 ? 1 : 0) + s1[q];
        for (int q = 0; q < 6; q++)
            if (kgrad == 2 || kgrad == 3)
                slot[4 + q] = (kgrad == 3 ? 4 : 0) + s2[q];
    }
    const size_t grid_sz = nlat * nlon;
    unsigned *d_status;
    unsigned long long *d_counter;
    CB_TRY(status_words(c, &d_status, &d_counter));
    const int ntiles = (np + 127) / 128;
    double *seed_x = nullptr;
    CB_TRY(dbuf(c, "tc_seed_x", (size_t)(N + 1) * np, &seed_x));
    int2 *seed_e = nullptr;
    CB_TRY(dbuf(c, "tc_seed_e", (size_t)(N + 1) * np, &seed_e));

    for (size_t j0 = 0; j0 < nsets; j0 += per_launch)
    {
        const int nb = (int)std::min<size_t>(per_launch, nsets - j0);
        const unsigned long Ng = nmax_v[ord[j0]];   // largest of the launch
        chunk_layout(Ng);
        CB_TRY(h2d_small(c, d_chunk0, h0.data(),
                         (Ng + 2) * sizeof(long long)));
        ShsTcPrep P{};
        P.nmax = (long long)Ng;
        P.nsets = nb;
        for (int b = 0; b < nb; b++)
        {
            const size_t jj = ord[j0 + b];
            P.set_nmax[b] = (long long)nmax_v[jj];
            P.shc_nmax[b] = (long long)shc_nmax_v[jj];
            P.c[b] = d_c[jj];
            P.s[b] = d_s[jj];
        }
        P.chunk0 = d_chunk0;
        P.ecol = d_ecol;
        P.bdig = static_cast<unsigned char *>(bdig);
        P.status = d_status;
        P.grad = grad ? 1 : 0;
        {
            Scope sc(c, TIMER_PREP);
            CB_CUDA(launch_tc_prep(P, c.stream), st);
        }
        CB_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(unsigned long long),
                                c.stream), st);
        ShsTcArgs A{};
        A.nmax = (long long)N;
        A.nmax_sets = (long long)Ng;
        A.npairs = np;
        A.ntiles = ntiles;
        A.nitems = (long long)(Ng + 1) * ntiles;
        A.tmul = tab.tmul;
        A.ldmul = tab.ldmul;
        A.sg = tab.sg;
        A.btp = btp;
        A.ctp = ctp;
        A.bdig = static_cast<const unsigned char *>(bdig);
        A.chunk0 = d_chunk0;
        A.ecol = d_ecol;
        A.t = dt;
        A.u = dt + np;
        A.rho = dt + 2 * np;
        A.row_n = reinterpret_cast<const int *>(dt + 3 * np);
        A.row_s = A.row_n + np;
        A.nlat = (int)nlat;
        A.ldf = ldf;
        A.nsets = nb;
        for (int b = 0; b < nb; b++)
        {
            A.out[b] = lc + (size_t)b * per_set;
            A.mur[b] = mu_v[ord[j0 + b]] / R;
        }
        A.counter = d_counter;
        A.status = d_status;
        A.seed_x = seed_x;
        A.seed_e = seed_e;
        A.grad = grad ? 1 : 0;
        A.Rref = R;
        if (j0 == 0)
        {
            Scope sc(c, TIMER_PREP);
            CB_CUDA(launch_tc_seeds(A, !G.r_eq, seed_x, seed_e, c.stream), st);
        }
        const int grid = (int)std::min<long long>(A.nitems,
                                                  (long long)c.num_sms);
        {
            Scope sc(c, TIMER_SHS);
            CB_CUDA(launch_shs_tc(A, !G.r_eq, std::max(grid, 1), c.stream),
                    st);
        }
        for (int b = 0; b < nb; b++)
        {
            const size_t jj = ord[j0 + b];
            for (int q = 0; q < (grad ? 10 : 1); q++)
            {
                const int sl = grad ? slot[q] : 0;
                if (sl < 0)
                    continue;
                double *dst = d_f[jj] + (size_t)sl * grid_sz;
                double2 *src = lc + (size_t)b * per_set + (size_t)q * per_q;
                if (rf->odd || reinterpret_cast<uintptr_t>(dst) % 16 == 0)
                {
                    RfftArgs R2 = *synth_plan(rf, rfq, (long long)nmax_v[jj]);
                    R2.nrows = (long long)nlat;
                    R2.x = dst;
                    R2.ldx = (long long)nlon;
                    R2.X = src;
                    R2.ldX = ldf;
                    R2.kmax = (int)nmax_v[jj];
                    Scope sc(c, TIMER_FFT);
                    CB_CUDA(launch_rfft(R2, true, c.stream), st);
                }
                else
                {
                    st.code = CHARM_EFUNCARG;
                    st.msg = "batched synthesis outputs must start on a "
                             "16-byte boundary";
                    return st;
                }
            }
        }
        // the digit tiles and the lumped buffer are reused by the next group
        // (stream order suffices inside a captured graph)
        if (!c.capturing)
            CB_CUDA(cudaStreamSynchronize(c.stream), st);
    }
    return finish(c, d_status);
}

// ---------------------------------------------------------------------------
// Single-precision mode (f32.cu): potential on FFT grids, r = R
// ---------------------------------------------------------------------------
// Tables (a_nm, b_nm) in float and S_m in double, built once per nmax.
Status tables_f32(Context &c, long long nmax, float4 **ab, double **smm)
{
    Status st;
    const long long T = (nmax + 1) * (nmax + 2) / 2;
    CB_TRY(dbuf(c, "tab32_ab", (size_t)T, ab));
    CB_TRY(dbuf(c, "tab32_smm", (size_t)(nmax + 1), smm));
    if (c.tab32_nmax == nmax)
        return st;
    std::vector<double> r, ri, dmh, hs(nmax + 1);
    host_r_ri_dm(nmax, r, ri, dmh);
    host_smm(nmax, hs.data());
    double *dr = nullptr, *dri = nullptr;
    CB_TRY(dbuf(c, "tab32_r", r.size(), &dr));
    CB_TRY(dbuf(c, "tab32_ri", ri.size(), &dri));
    CB_CUDA(cudaMemcpyAsync(dr, r.data(), r.size() * 8,
                            cudaMemcpyHostToDevice, c.stream), st);
    CB_CUDA(cudaMemcpyAsync(dri, ri.data(), ri.size() * 8,
                            cudaMemcpyHostToDevice, c.stream), st);
    CB_CUDA(cudaMemcpyAsync(*smm, hs.data(), hs.size() * 8,
                            cudaMemcpyHostToDevice, c.stream), st);
    {
        Scope sc(c, TIMER_TABLES);
        CB_CUDA(launch_tables_f32(nmax, dr, dri, *ab, c.stream), st);
    }
    // the host vectors must outlive the copies
    CB_CUDA(cudaStreamSynchronize(c.stream), st);
    c.tab32_nmax = nmax;
    return st;
}

// Checks shared by both directions: equally spaced longitudes starting at
// 0 with a shared-memory row transform, orders up to nmax resolvable, and
// every row on the sphere r = R.
Status f32_grid_checks(Context &c, const charm_point *pnt, unsigned long nmax,
                       double R, const RfftArgs **rf)
{
    Status st;
    if (nmax > 2200)
    {
        // the scaled-seed renormalisation every 16 degrees keeps the float
        // recurrence in range up to this degree
        st.code = CHARM_EFUNCARG;
        st.msg = "The single-precision mode serves nmax <= 2200.";
        return st;
    }
    const size_t nlat = pnt->nlat, nlon = pnt->nlon;
    const double thr = charm_glob_threshold;
    double step = nlon > 1 ? pnt->lon[1] - pnt->lon[0] : 0.0;
    bool fft = nlon >= 2 && (nlon - 1) / 2 >= nmax &&
               nearly_equal(pnt->lon[0], 0.0, thr) &&
               nearly_equal(pnt->lon[nlon - 1] + step, 2.0 * PI, thr);
    for (size_t j = 1; fft && j < nlon; j++)
        if (!nearly_equal(step, pnt->lon[j] - pnt->lon[j - 1],
                          charm_glob_threshold2))
            fft = false;
    *rf = nullptr;
    if (fft && nlon % 2 == 0)
        CB_TRY(row_fft(c, (long long)nlon, rf));
    if (!*rf || (*rf)->C > 1)
    {
        st.code = CHARM_EFUNCARG;
        st.msg = "The single-precision mode needs a grid whose longitudes "
                 "0, 2 pi / nlon, ... admit the shared-memory row transform "
                 "(even nlon, nlon / 2 + 1 > nmax).";
        return st;
    }
    for (size_t i = 0; i < nlat; i++)
        if (!nearly_equal(pnt->r[i], R, thr))
        {
            st.code = CHARM_EFUNCARG;
            st.msg = "The single-precision mode needs every grid row on the "
                     "sphere of the coefficients' radius (r = R).";
            return st;
        }
    return st;
}

Status shs_grid_f32(Context &c, const charm_point *pnt, unsigned long shc_nmax,
                    double mu, double R, const float *d_c, const float *d_s,
                    unsigned long nmax, float *d_f)
{
    Status st;
    const size_t nlat = pnt->nlat, nlon = pnt->nlon;
    const RfftArgs *rf = nullptr;
    CB_TRY(f32_grid_checks(c, pnt, nmax, R, &rf));
    if (reinterpret_cast<uintptr_t>(d_f) % 8 != 0)
    {
        st.code = CHARM_EFUNCARG;
        st.msg = "The grid values must start on an 8-byte boundary.";
        return st;
    }
    Pairs P;
    grid_pairs(pnt, charm_glob_threshold2, true, P);
    const int np = (int)P.row_n.size();
    size_t geo_bytes = (size_t)np * (2 * 8 + 2 * 4);
    void *hp = nullptr;
    CB_TRY(pinned(c, geo_bytes, &hp));
    double *ht = static_cast<double *>(hp);
    double *hu = ht + np;
    int *hrn = reinterpret_cast<int *>(hu + np);
    int *hrs = hrn + np;
    for (int p = 0; p < np; p++)
    {
        double la = pnt->lat[P.row_n[p]];
        sincos(la, &ht[p], &hu[p]);
        hrn[p] = P.row_n[p];
        hrs[p] = P.row_s[p];
    }
    void *dgeo = nullptr;
    CB_TRY(buf(c, "geo", geo_bytes, &dgeo));
    CB_CUDA(cudaMemcpyAsync(dgeo, hp, geo_bytes, cudaMemcpyHostToDevice,
                            c.stream), st);
    float4 *ab = nullptr;
    double *smm = nullptr;
    CB_TRY(tables_f32(c, (long long)nmax, &ab, &smm));
    const long long T = (long long)(nmax + 1) * (nmax + 2) / 2;
    float4 *abcs = nullptr;
    CB_TRY(dbuf(c, "abcs32", (size_t)(2 * T), &abcs));
    {
        Scope sc(c, TIMER_PREP);
        CB_CUDA(launch_pack_cs_f32((long long)nmax, (long long)shc_nmax, d_c,
                                   d_s, ab, abcs, c.stream), st);
    }
    const int ldf = (int)(nlon / 2 + 1);
    double2 *lc = nullptr;
    CB_TRY(dbuf(c, "lumped", nlat * (size_t)ldf, &lc));
    unsigned *d_status;
    unsigned long long *d_counter;
    CB_TRY(status_words(c, &d_status, &d_counter));
    const int K = np >= 4096 ? 8 : (np >= 128 ? 4 : 2);
    ShsF32Args A{};
    A.nmax = (long long)nmax;
    A.npairs = np;
    A.ntiles = (np + 32 * K - 1) / (32 * K);
    A.nitems = (long long)(nmax + 1) * A.ntiles;
    A.abcs = abcs;
    A.smm = smm;
    A.t = static_cast<const double *>(dgeo);
    A.u = A.t + np;
    A.row_n = reinterpret_cast<const int *>(A.u + np);
    A.row_s = A.row_n + np;
    A.nlat = (int)nlat;
    A.ldf = ldf;
    A.out = lc;
    A.mur = mu / R;
    A.polar_thr = polar_threshold(nmax);
    A.counter = d_counter;
    A.status = d_status;
    int grid = (int)std::min<long long>((A.nitems + 3) / 4,
                                        (long long)c.num_sms * 8);
    {
        Scope sc(c, TIMER_SHS);
        CB_CUDA(launch_shs_grid_f32(A, K, std::max(grid, 1), c.stream), st);
    }
    RfftArgs R2 = *rf;
    R2.nrows = (long long)nlat;
    R2.x = reinterpret_cast<double *>(d_f);
    R2.ldx = (long long)nlon;
    R2.X = lc;
    R2.ldX = ldf;
    R2.kmax = (int)nmax;
    R2.f32_rows = 1;
    {
        Scope sc(c, TIMER_FFT);
        CB_CUDA(launch_rfft(R2, true, c.stream), st);
    }
    return finish(c, d_status);
}

Status sha_grid_f32(Context &c, const charm_point *pnt, const float *d_f,
                    unsigned long nmax, double mu, double R,
                    unsigned long shc_nmax, float *d_c, float *d_s)
{
    Status st;
    const size_t nlat = pnt->nlat, nlon = pnt->nlon;
    const double r0 = pnt->r[0];
    const RfftArgs *rf = nullptr;
    CB_TRY(f32_grid_checks(c, pnt, nmax, r0, &rf));
    if (reinterpret_cast<uintptr_t>(d_f) % 8 != 0)
    {
        st.code = CHARM_EFUNCARG;
        st.msg = "The grid values must start on an 8-byte boundary.";
        return st;
    }
    const unsigned long nmax_grd = pnt->type == CHARM_CRD_POINT_GRID_GL
                                       ? nlat - 1
                                       : (nlat - 2) / 2;
    // quadrature constant, src/sha/sha_point.c:313-322
    double cq = (pnt->type == CHARM_CRD_POINT_GRID_DH2)
                    ? PI / (double)(2 * nmax_grd + 2)
                    : PI / (double)(nmax_grd + 1);
    cq *= 1.0 / (4.0 * PI) * (r0 / mu);
    Pairs P;
    grid_pairs(pnt, charm_glob_threshold2, true, P);
    const int np = (int)P.row_n.size();
    size_t geo_bytes = (size_t)np * (4 * 8 + 2 * 4);
    void *hp = nullptr;
    CB_TRY(pinned(c, geo_bytes, &hp));
    double *ht = static_cast<double *>(hp);
    double *hu = ht + np;
    double *hcn = hu + np;
    double *hcs = hcn + np;
    int *hrn = reinterpret_cast<int *>(hcs + np);
    int *hrs = hrn + np;
    for (int p = 0; p < np; p++)
    {
        double la = pnt->lat[P.row_n[p]];
        sincos(la, &ht[p], &hu[p]);
        hcn[p] = cq * pnt->w[P.row_n[p]];
        hcs[p] = P.row_s[p] >= 0 ? cq * pnt->w[P.row_s[p]] : 0.0;
        hrn[p] = P.row_n[p];
        hrs[p] = P.row_s[p];
    }
    void *dgeo = nullptr;
    CB_TRY(buf(c, "geo", geo_bytes, &dgeo));
    CB_CUDA(cudaMemcpyAsync(dgeo, hp, geo_bytes, cudaMemcpyHostToDevice,
                            c.stream), st);
    float4 *ab = nullptr;
    double *smm = nullptr;
    CB_TRY(tables_f32(c, (long long)nmax, &ab, &smm));
    const int ldF = (int)(nlon / 2 + 1);
    double2 *F = nullptr;
    CB_TRY(dbuf(c, "lumped", nlat * (size_t)ldF, &F));
    RfftArgs R2 = *rf;
    R2.nrows = (long long)nlat;
    R2.x = const_cast<double *>(reinterpret_cast<const double *>(d_f));
    R2.ldx = (long long)nlon;
    R2.X = F;
    R2.ldX = ldF;
    R2.kmax = (int)nmax;
    R2.f32_rows = 1;
    {
        Scope sc(c, TIMER_FFT);
        CB_CUDA(launch_rfft(R2, false, c.stream), st);
    }
    unsigned *d_status;
    unsigned long long *d_counter;
    CB_TRY(status_words(c, &d_status, &d_counter));
    const int K = np >= 4096 ? 8 : (np >= 128 ? 4 : 2);
    const int ntiles = (np + 32 * K - 1) / (32 * K);
    const long long T = (long long)(nmax + 1) * (nmax + 2) / 2;
    long long slots = (long long)c.num_sms * 8 * 4;
    long long G = std::max<long long>(1, (2 * slots + nmax) / (nmax + 1));
    G = std::min<long long>(G, ntiles);
    int tpg = (int)((ntiles + G - 1) / G);
    G = (ntiles + tpg - 1) / tpg;
    float2 *part = nullptr;
    CB_TRY(dbuf(c, "sha_part32", (size_t)G * T, &part));
    ShaF32Args A{};
    A.nmax = (long long)nmax;
    A.npairs = np;
    A.ntiles = ntiles;
    A.ngroups = (int)G;
    A.tiles_per_group = tpg;
    A.nitems = (long long)(nmax + 1) * G;
    A.ab = ab;
    A.smm = smm;
    A.t = static_cast<const double *>(dgeo);
    A.u = A.t + np;
    A.cw_n = A.u + np;
    A.cw_s = A.cw_n + np;
    A.row_n = reinterpret_cast<const int *>(A.cw_s + np);
    A.row_s = A.row_n + np;
    A.F = F;
    A.ldF = ldF;
    A.part = part;
    A.polar_thr = polar_threshold(nmax);
    A.counter = d_counter;
    A.status = d_status;
    int grid = (int)std::min<long long>((A.nitems + 3) / 4,
                                        (long long)c.num_sms * 8);
    {
        Scope sc(c, TIMER_SHA);
        CB_CUDA(launch_sha_grid_f32(A, K, std::max(grid, 1), c.stream), st);
    }
    // rescaling from r0 to the coefficients' radius (as sha_grid)
    double *dres = nullptr;
    std::vector<double> res;
    if (!nearly_equal(R, r0, charm_glob_threshold))
    {
        double r_ratio = r0 / R;
        res.resize(nmax + 1);
        double tmp2 = r_ratio;
        res[0] = 1.0;
        for (unsigned long n = 1; n <= nmax; n++)
        {
            res[n] = tmp2;
            tmp2 *= r_ratio;
        }
        CB_TRY(dbuf(c, "sha_rescale", nmax + 1, &dres));
        CB_CUDA(cudaMemcpyAsync(dres, res.data(), (nmax + 1) * 8,
                                cudaMemcpyHostToDevice, c.stream), st);
    }
    {
        Scope sc(c, TIMER_PREP);
        CB_CUDA(launch_sha_reduce_f32((long long)nmax, (long long)shc_nmax,
                                      (int)G, T, part, dres, d_c, d_s,
                                      c.stream), st);
    }
    return finish(c, d_status);
}

// ---------------------------------------------------------------------------
// Adjoint of the scattered synthesis with respect to the coefficients
// ---------------------------------------------------------------------------
// C_nm = (GM/R) sum_i g_i (R/r_i)^(n+1) P_nm(sin lat_i) cos(m lon_i), S_nm
// with sin: the transpose of shs_sctr's potential (dorder 0), computed by
// the analysis kernel with points as amplitude source.
Status sctr_adjoint(Context &c, const charm_point *pnt, const double *g_host,
                    const double *d_g, unsigned long nmax, double mu,
                    double R, unsigned long shc_nmax, double *const *hc,
                    double *const *hs, double *d_c, double *d_s)
{
    Status st;
    const size_t npt = pnt->nlat;
    const bool r_eq = all_nearly_equal(pnt->r, npt, R, charm_glob_threshold);
    Tabs tab;
    CB_TRY(tables(c, (long long)nmax, &tab));
    double *dpts = nullptr;
    CB_TRY(dbuf(c, "sctr_pts", 3 * npt + (d_g ? 0 : npt), &dpts));
    CB_CUDA(cudaMemcpyAsync(dpts, pnt->lat, npt * 8, cudaMemcpyHostToDevice,
                            c.stream), st);
    CB_CUDA(cudaMemcpyAsync(dpts + npt, pnt->lon, npt * 8,
                            cudaMemcpyHostToDevice, c.stream), st);
    if (!r_eq)
        CB_CUDA(cudaMemcpyAsync(dpts + 2 * npt, pnt->r, npt * 8,
                                cudaMemcpyHostToDevice, c.stream), st);
    const double *gw = d_g;
    if (!gw)
    {
        CB_CUDA(cudaMemcpyAsync(dpts + 3 * npt, g_host, npt * 8,
                                cudaMemcpyHostToDevice, c.stream), st);
        gw = dpts + 3 * npt;
    }
    unsigned *d_status;
    unsigned long long *d_counter;
    CB_TRY(status_words(c, &d_status, &d_counter));
    const int K = choose_k_sha((long long)npt);
    const long long ntiles = ((long long)npt + 32 * K - 1) / (32 * K);
    const long long T = (long long)(nmax + 1) * (nmax + 2) / 2;
    long long slots = (long long)c.num_sms * 8 * 4;
    long long G = std::max<long long>(1, (2 * slots + nmax) / (nmax + 1));
    G = std::min<long long>(G, ntiles);
    long long tpg = (ntiles + G - 1) / G;
    G = (ntiles + tpg - 1) / tpg;
    double2 *part = nullptr;
    CB_TRY(dbuf(c, "sha_part", (size_t)G * T, &part));
    ShaGridArgs A{};
    A.nmax = (long long)nmax;
    A.npairs = (int)npt;
    A.ntiles = (int)ntiles;
    A.ngroups = (int)G;
    A.tiles_per_group = (int)tpg;
    A.nitems = (long long)(nmax + 1) * G;
    A.tb = tab.tb;
    A.tmul = tab.tmul;
    A.ldmul = tab.ldmul;
    A.sg = tab.sg;
    A.part = part;
    A.polar_thr = polar_threshold(nmax);
    A.counter = d_counter;
    A.status = d_status;
    A.lat = dpts;
    A.lon = dpts + npt;
    A.r = dpts + 2 * npt;
    A.g = gw;
    A.R = R;
    int grid = (int)std::min<long long>((A.nitems + 3) / 4,
                                        (long long)c.num_sms * 8);
    {
        Scope sc(c, TIMER_SCTR);
        CB_CUDA(launch_sha_points(A, r_eq ? 1 : 2, K, std::max(grid, 1),
                                  c.stream), st);
    }
    const long long Ts = (long long)(shc_nmax + 1) * (shc_nmax + 2) / 2;
    double *oc = d_c, *os = d_s;
    if (!oc)
    {
        double *dout = nullptr;
        CB_TRY(dbuf(c, "shc_out", (size_t)(2 * Ts), &dout));
        oc = dout;
        os = dout + Ts;
    }
    {
        Scope sc(c, TIMER_PREP);
        CB_CUDA(launch_sha_reduce((long long)nmax, (long long)shc_nmax,
                                  (int)G, T, part, tab.tc, nullptr, mu / R,
                                  oc, os, c.stream), st);
    }
    if (!d_c)
    {
        CB_TRY(download_tri(c, oc, shc_nmax, hc));
        CB_TRY(download_tri(c, os, shc_nmax, hs));
    }
    return finish(c, d_status);
}

// ---------------------------------------------------------------------------
// Grid analysis
// ---------------------------------------------------------------------------
// pair0 / pair1: with pair1 >= 0, only the latitude pairs [pair0, pair1)
// of the grid's pairing (grid_pairs) enter the sums (a band of one
// latitude-band-sharded analysis; device grids only).
Status sha_grid(Context &c, const charm_point *pnt, const double *f_host,
                const double *d_fin, unsigned long nmax, double mu, double R,
                unsigned long shc_nmax, double *const *hc, double *const *hs,
                double *d_c, double *d_s, int pair0 = 0, int pair1 = -1)
{
    Status st;
    const size_t nlat = pnt->nlat, nlon = pnt->nlon;
    const double r0 = pnt->r[0];
    const unsigned long nmax_grd = pnt->type == CHARM_CRD_POINT_GRID_GL
                                       ? nlat - 1
                                       : (nlat - 2) / 2;
    // quadrature constant, src/sha/sha_point.c:313-322
    double cq = (pnt->type == CHARM_CRD_POINT_GRID_DH2)
                    ? PI / (double)(2 * nmax_grd + 2)
                    : PI / (double)(nmax_grd + 1);
    cq *= 1.0 / (4.0 * PI) * (r0 / mu);

    Pairs P;
    grid_pairs(pnt, charm_glob_threshold2, true, P);
    const bool band = pair1 >= 0;
    // rows of the band's northern and southern members, [lo, hi)
    int band_n0 = 0, band_n1 = 0, band_s0 = 0, band_s1 = 0;
    if (band)
    {
        if (!d_fin || pair0 < 0 || pair0 > pair1 ||
            pair1 > (int)P.row_n.size())
        {
            st.code = CHARM_EFUNCARG;
            st.msg = "latitude band [" + std::to_string(pair0) + ", " +
                     std::to_string(pair1) + ") outside the grid's " +
                     std::to_string(P.row_n.size()) +
                     " latitude pairs (or a host grid)";
            return st;
        }
        P.row_n.assign(P.row_n.begin() + pair0, P.row_n.begin() + pair1);
        P.row_s.assign(P.row_s.begin() + pair0, P.row_s.begin() + pair1);
        band_n0 = band_s0 = (int)nlat;
        for (size_t p = 0; p < P.row_n.size(); p++)
        {
            band_n0 = std::min(band_n0, P.row_n[p]);
            band_n1 = std::max(band_n1, P.row_n[p] + 1);
            if (P.row_s[p] >= 0 && P.row_s[p] < (int)nlat)
            {
                band_s0 = std::min(band_s0, P.row_s[p]);
                band_s1 = std::max(band_s1, P.row_s[p] + 1);
            }
        }
        if (P.row_n.empty())
        {
            // an empty band contributes nothing
            const size_t T = (size_t)(shc_nmax + 1) * (shc_nmax + 2) / 2;
            CB_CUDA(cudaMemsetAsync(d_c, 0, T * 8, c.stream), st);
            CB_CUDA(cudaMemsetAsync(d_s, 0, T * 8, c.stream), st);
            CB_CUDA(cudaStreamSynchronize(c.stream), st);
            return st;
        }
    }
    const int np = (int)P.row_n.size();
    size_t geo_bytes = (size_t)np * (4 * 8 + 2 * 4);
    void *hp = nullptr;
    CB_TRY(pinned(c, geo_bytes, &hp));
    double *ht = static_cast<double *>(hp);
    double *hu = ht + np;
    double *hcn = hu + np;
    double *hcs = hcn + np;
    int *hrn = reinterpret_cast<int *>(hcs + np);
    int *hrs = hrn + np;
    for (int p = 0; p < np; p++)
    {
        double la = pnt->lat[P.row_n[p]];
        sincos(la, &ht[p], &hu[p]);
        hcn[p] = cq * pnt->w[P.row_n[p]];
        hcs[p] = P.row_s[p] >= 0 ? cq * pnt->w[P.row_s[p]] : 0.0;
        hrn[p] = P.row_n[p];
        hrs[p] = P.row_s[p];
    }
    void *dgeo = nullptr;
    CB_TRY(buf(c, "geo", geo_bytes, &dgeo));
    CB_CUDA(cudaMemcpyAsync(dgeo, hp, geo_bytes, cudaMemcpyHostToDevice,
                            c.stream), st);
    const double *dt = static_cast<const double *>(dgeo);
    const double *du = dt + np;
    const double *dcn = du + np;
    const double *dcsw = dcn + np;
    const int *drn = reinterpret_cast<const int *>(dcsw + np);
    const int *drs = drn + np;

    Tabs tab;
    CB_TRY(tables(c, (long long)nmax, &tab));

    // work decomposition: K latitude pairs per lane, tiles of 32 K pairs,
    // groups of tiles whose partial sums are added in fixed order
    unsigned *d_status;
    unsigned long long *d_counter;
    CB_TRY(status_words(c, &d_status, &d_counter));
    const int K = choose_k_sha(np);
    const int ntiles = (np + 32 * K - 1) / (32 * K);
    const long long T = (long long)(nmax + 1) * (nmax + 2) / 2;
    long long slots = (long long)c.num_sms * 8 * 4;
    long long G = std::max<long long>(1, (2 * slots + nmax) / (nmax + 1));
    G = std::min<long long>(G, ntiles);
    // a host grid is analysed in bands of tiles, overlapped with its copy:
    // groups of single tiles (within 512 MB of partial sums) keep each
    // band's launch balanced (shorter work items)
    if (!d_fin)
        G = std::max<long long>(
            G, std::min<long long>(ntiles, (512LL << 20) / (16 * T)));
    int tpg = (int)((ntiles + G - 1) / G);
    G = (ntiles + tpg - 1) / tpg;
    double2 *part = nullptr;
    CB_TRY(dbuf(c, "sha_part", (size_t)G * T, &part));

    // grid on the device and r2c along the parallels
    const double *fg = d_fin;
    double *fdev = nullptr;
    if (!fg)
    {
        CB_TRY(dbuf(c, "fgrid", nlat * nlon, &fdev));
        fg = fdev;
    }
    const int ldF = (int)(nlon / 2 + 1);
    double2 *F = nullptr;
    CB_TRY(dbuf(c, "lumped", nlat * (size_t)ldF, &F));
    // the transform loads pairs of doubles: a device grid that is not on a
    // 16-byte boundary is copied once into the aligned staging grid
    if (d_fin && reinterpret_cast<uintptr_t>(d_fin) % 16 != 0)
    {
        double *al = nullptr;
        CB_TRY(dbuf(c, "fgrid", nlat * nlon, &al));
        CB_CUDA(cudaMemcpyAsync(al, d_fin, nlat * nlon * 8,
                                cudaMemcpyDeviceToDevice, c.stream), st);
        fg = al;
    }
    const RfftArgs *rf = nullptr;
    CB_TRY(row_fft(c, (long long)nlon, &rf));
    if (rf->odd)
    {
        st.code = CHARM_EFUNCARG;
        st.msg = "analysis grids have an even number of longitudes";
        return st;
    }
    auto rows_fft = [&](int r0, int r1) -> Status {
        Status s2;
        RfftArgs R = *rf;
        R.nrows = (long long)(r1 - r0);
        R.x = const_cast<double *>(fg) + (size_t)r0 * nlon;
        R.ldx = (long long)nlon;
        R.X = F + (size_t)r0 * ldF;
        R.ldX = ldF;
        R.kmax = (int)nmax;
        Scope sc(c, TIMER_FFT);
        CB_CUDA(launch_rfft(R, false, c.stream), s2);
        return s2;
    };

    ShaGridArgs A{};
    A.nmax = (long long)nmax;
    A.npairs = np;
    A.ntiles = ntiles;
    A.ngroups = (int)G;
    A.tiles_per_group = tpg;
    A.nitems = (long long)(nmax + 1) * G;
    A.tb = tab.tb;
    A.tmul = tab.tmul;
    A.ldmul = tab.ldmul;
    A.sg = tab.sg;
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

    // rescaling from r0 to the coefficients' radius
    // (src/sha/sha_point.c:1088-1108 with src/shc/shc_rescale.c)
    const unsigned long sn = shc_nmax;
    double *dres = nullptr;
    std::vector<double> res;
    if (!nearly_equal(R, r0, charm_glob_threshold))
    {
        double mu_ratio = mu / mu;
        double r_ratio = r0 / R;
        res.resize(sn + 1);
        double tmp2 = mu_ratio * r_ratio;
        res[0] = mu_ratio;
        for (unsigned long n = 1; n <= sn; n++)
        {
            res[n] = tmp2;
            tmp2 *= r_ratio;
        }
        CB_TRY(dbuf(c, "sha_rescale", sn + 1, &dres));
        CB_CUDA(cudaMemcpyAsync(dres, res.data(), (sn + 1) * 8,
                                cudaMemcpyHostToDevice, c.stream), st);
    }
    const long long Ts = (long long)(sn + 1) * (sn + 2) / 2;
    double *oc = d_c, *os = d_s;
    if (!oc)
    {
        double *dout = nullptr;
        CB_TRY(dbuf(c, "shc_out", (size_t)(2 * Ts), &dout));
        oc = dout;
        os = dout + Ts;
    }

    // Host input through the row transform: bands of tile groups; band b's
    // rows are copied (copy stream) while band b - 1 is transformed and
    // analysed.  The partial sums of every group are the same as in one
    // launch.  With host outputs the last band runs in bands of orders,
    // each reduced and copied to the host (copy stream) while the next one
    // is analysed.
    std::vector<std::array<int, 6>> bands;
    const int nband = (fdev && rf) ? grid_bands(P, (int)nlat, (int)G,
                                                32 * K * tpg,
                                                G >= 3 ? SHA_LAT_BANDS : 2,
                                                bands)
                                   : 1;
    bool ordered = false;
    if (nband > 1)
    {
        // orders of the last band in up to SHA_ORD_BANDS bands of about
        // equal numbers of coefficients
        std::vector<long long> mb{0};
        if (!d_c)
        {
            const int nob = SHA_ORD_BANDS;
            for (int k = 1; k < nob; k++)
            {
                long long m = mb.back();
                while (m <= (long long)nmax &&
                       tri_start((long long)nmax, m) < k * T / nob)
                    m++;
                if (m > mb.back() && m <= (long long)nmax)
                    mb.push_back(m);
            }
        }
        mb.push_back((long long)nmax + 1);
        const int nob = (int)mb.size() - 1;
        unsigned long long *bcnt = nullptr;
        CB_TRY(dbuf(c, "band_counters", 16, &bcnt));
        CB_CUDA(cudaMemsetAsync(bcnt, 0, 16 * sizeof(unsigned long long),
                                c.stream), st);
        // the copy stream starts after everything before it on the stream
        // (buffers in use by an earlier call)
        CB_CUDA(cudaEventRecord(c.band_ev[EV_START], c.stream), st);
        CB_CUDA(cudaStreamWaitEvent(c.copy_stream, c.band_ev[EV_START], 0), st);
        for (int b = 0; b < nband; b++)
        {
            const auto &bd = bands[b];
            for (int h = 0; h < 2; h++)
            {
                const int r0 = bd[2 + 2 * h], r1 = bd[3 + 2 * h];
                if (r1 > r0)
                    CB_CUDA(cudaMemcpyAsync(fdev + (size_t)r0 * nlon,
                                            f_host + (size_t)r0 * nlon,
                                            (size_t)(r1 - r0) * nlon * 8,
                                            cudaMemcpyHostToDevice,
                                            c.copy_stream),
                            st);
            }
            CB_CUDA(cudaEventRecord(c.band_ev[EV_LAT0 + b], c.copy_stream), st);
            CB_CUDA(cudaStreamWaitEvent(c.stream, c.band_ev[EV_LAT0 + b], 0),
                    st);
            for (int h = 0; h < 2; h++)
            {
                const int r0 = bd[2 + 2 * h], r1 = bd[3 + 2 * h];
                if (r1 > r0)
                    CB_TRY(rows_fft(r0, r1));
            }
            const bool split = b == nband - 1 && nob > 1;
            for (int k = 0; k < (split ? nob : 1); k++)
            {
                ShaGridArgs Ab = A;
                Ab.group0 = bd[0];
                Ab.ngroups = bd[1] - bd[0];
                Ab.m0 = split ? mb[k] : 0;
                Ab.nitems = (long long)(split ? mb[k + 1] - mb[k]
                                              : (long long)nmax + 1) *
                            Ab.ngroups;
                Ab.counter = bcnt + (split ? nband + k : b);
                const int gb = (int)std::min<long long>(
                    (Ab.nitems + 3) / 4, (long long)c.num_sms * 8);
                {
                    Scope sc(c, TIMER_SHA);
                    CB_CUDA(launch_sha_grid(Ab, K, std::max(gb, 1), c.stream),
                            st);
                }
                if (split)
                {
                    // these orders are complete: their coefficients (with
                    // the zero orders above nmax after the last band)
                    const long long m_hi =
                        k == nob - 1 ? (long long)sn + 1 : mb[k + 1];
                    Scope sc(c, TIMER_PREP);
                    CB_CUDA(launch_sha_reduce_orders(
                                (long long)nmax, (long long)sn, (int)G, T,
                                part, tab.tc, dres, 1.0, oc, os, mb[k], m_hi,
                                c.stream),
                            st);
                    CB_CUDA(cudaEventRecord(c.band_ev[EV_ORD0 + k], c.stream), st);
                }
            }
            if (split)
            {
                // the copies after every launch, so that a copy to pageable
                // memory, which returns only when it is done, holds back no
                // launch
                for (int k = 0; k < nob; k++)
                {
                    const long long m_hi =
                        k == nob - 1 ? (long long)sn + 1 : mb[k + 1];
                    CB_CUDA(cudaStreamWaitEvent(c.copy_stream,
                                                c.band_ev[EV_ORD0 + k], 0),
                            st);
                    CB_TRY(download_tri_orders(c, oc, sn, hc, mb[k], m_hi,
                                               c.copy_stream, 0));
                    CB_TRY(download_tri_orders(c, os, sn, hs, mb[k], m_hi,
                                               c.copy_stream, 0));
                }
                ordered = true;
            }
        }
    }
    else
    {
        if (fdev)
            CB_CUDA(cudaMemcpyAsync(fdev, f_host, nlat * nlon * 8,
                                    cudaMemcpyHostToDevice, c.stream), st);
        if (band)
        {
            CB_TRY(rows_fft(band_n0, band_n1));
            if (band_s1 > band_s0)
                CB_TRY(rows_fft(band_s0, band_s1));
        }
        else
            CB_TRY(rows_fft(0, (int)nlat));
        int grid = (int)std::min<long long>((A.nitems + 3) / 4,
                                            (long long)c.num_sms * 8);
        Scope sc(c, TIMER_SHA);
        CB_CUDA(launch_sha_grid(A, K, std::max(grid, 1), c.stream), st);
    }

    if (ordered)
    {
        CB_CUDA(cudaStreamSynchronize(c.copy_stream), st);
        return finish(c, d_status);
    }
    {
        Scope sc(c, TIMER_PREP);
        CB_CUDA(launch_sha_reduce((long long)nmax, (long long)sn, (int)G, T,
                                  part, tab.tc, dres, 1.0, oc, os, c.stream),
                st);
    }
    if (!d_c)
    {
        CB_TRY(download_tri(c, oc, sn, hc));
        CB_TRY(download_tri(c, os, sn, hs));
    }
    // res must stay alive until the copy ran: finish() synchronises
    return finish(c, d_status);
}

// ---------------------------------------------------------------------------
// Cells: block means (cell.cu)
// ---------------------------------------------------------------------------
// src/misc/misc_arr_chck_lin_incr.c with first = 0, every_nth = 1: the
// array starts at its minimum and increases by one positive step
bool lin_incr(const double *a, size_t n, double eps)
{
    if (n < 2)
        return true;
    double mn = a[0];
    for (size_t j = 1; j < n; j++)
        mn = std::min(mn, a[j]);
    if (!nearly_equal(a[0], mn, eps))
        return false;
    const double step = a[1] - a[0];
    if (step <= 0.0)
        return false;
    for (size_t j = 1; j < n; j++)
        if (!nearly_equal(step, a[j] - a[j - 1], eps))
            return false;
    return true;
}

// src/crd/crd_check_cells.c:14-40
Status check_cells(const charm_cell *cell)
{
    Status st;
    for (size_t i = 0; i < cell->nlat; i++)
        if (cell->latmax[i] <= cell->latmin[i])
        {
            st.code = CHARM_EFUNCARG;
            st.msg = "Minimum cell latitudes must be smaller than maximum "
                     "cell latitudes.";
            return st;
        }
    for (size_t j = 0; j < cell->nlon; j++)
        if (cell->lonmin[j] >= cell->lonmax[j])
        {
            st.code = CHARM_EFUNCARG;
            st.msg = "Minimum cell longitudes must be smaller than maximum "
                     "cell longitudes.";
            return st;
        }
    return st;
}

// src/shs/shs_cell_check_grd_lons.c:14-85: constant steps of lonmin and
// lonmax, equal to each other; returns the step (the cell width)
Status cell_grd_lons(const charm_cell *cell, double *dlon)
{
    Status st;
    const double thr2 = charm_glob_threshold2;
    if (cell->nlon > 1)
    {
        if (!lin_incr(cell->lonmin, cell->nlon, thr2))
        {
            st.code = CHARM_EFUNCARG;
            st.msg = "\"cell->lonmin\" is not a linearly increasing array of "
                     "cells within the \"threshold2\".";
            return st;
        }
        if (!lin_incr(cell->lonmax, cell->nlon, thr2))
        {
            st.code = CHARM_EFUNCARG;
            st.msg = "\"cell->lonmax\" is not a linearly increasing array of "
                     "cells within the \"threshold2\".";
            return st;
        }
        if (!nearly_equal(cell->lonmin[1] - cell->lonmin[0],
                          cell->lonmax[1] - cell->lonmax[0], thr2))
        {
            st.code = CHARM_EFUNCARG;
            st.msg = "The difference \"cell->lonmin[1] - cell->lonmin[0]\" "
                     "has to be equal to \"cell->lonmax[1] - "
                     "cell->lonmax[0]\".";
            return st;
        }
        *dlon = cell->lonmin[1] - cell->lonmin[0];
    }
    else
        *dlon = cell->lonmax[0] - cell->lonmin[0];
    return st;
}

struct CellTabs
{
    double2 *hn = nullptr;
    double4 *zn = nullptr;
    double *gm = nullptr;
};

// Per-degree tables of the cell kernels, built once per maximum degree:
// (h_n, 1 / (n + 1)) and g_n of src/leg/leg_func_gm_hm.c:14-45, and the
// un-normalised zonal recurrence (e_n+1, f_n+1) of src/leg/leg_pol_en_fn.c
// with 1 / sqrt(2n + 1).
Status cell_tables(Context &c, long long nmax, CellTabs *ct)
{
    Status st;
    const size_t L = (size_t)nmax + 1;
    CB_TRY(dbuf(c, "cell_hn", L, &ct->hn));
    CB_TRY(dbuf(c, "cell_zn", L, &ct->zn));
    CB_TRY(dbuf(c, "cell_gm", L, &ct->gm));
    if (c.cell_nmax == nmax)
        return st;
    std::vector<double> r, ri, dmh;
    host_r_ri_dm(nmax, r, ri, dmh);
    std::vector<double2> hn(L);
    std::vector<double4> zn(L);
    std::vector<double> gm(L, 0.0);
    for (long long n = 0; n <= nmax; n++)
    {
        hn[n] = make_double2((double)(n - 2) / (double)(n + 1),
                             1.0 / (double)(n + 1));
        if (n == 0)
            zn[n] = make_double4(0.0, 0.0, 0.0, 0.0);
        else
        {
            const long long k = n + 1;
            zn[n] = make_double4((double)(2 * k - 1) / (double)k,
                                 (double)(k - 1) / (double)k, ri[2 * n + 1],
                                 0.0);
        }
        if (n >= 3)
            gm[n] = 1.0 / (double)(2 * n + 2) * r[n] * r[2 * n + 1] *
                    r[2 * n - 1] * ri[n - 1];
    }
    CB_CUDA(cudaMemcpyAsync(ct->hn, hn.data(), L * sizeof(double2),
                            cudaMemcpyHostToDevice, c.stream), st);
    CB_CUDA(cudaMemcpyAsync(ct->zn, zn.data(), L * sizeof(double4),
                            cudaMemcpyHostToDevice, c.stream), st);
    CB_CUDA(cudaMemcpyAsync(ct->gm, gm.data(), L * sizeof(double),
                            cudaMemcpyHostToDevice, c.stream), st);
    // the host vectors must outlive the copies
    CB_CUDA(cudaStreamSynchronize(c.stream), st);
    c.cell_nmax = nmax;
    return st;
}

// Cell-row pairs of a grid (shs_cell_grd.c:52-110 with crd_grd_check_symm.c
// for cell grids; sha_cell.c:140-205 picks nlatdo the same way): rows
// 0..nlatdo-1, each with its mirror nlat-1-i when the grid is symmetric,
// except the middle row of an odd grid.  A mirror with another radius gets
// a pair of its own (the rows of a pair share the radius ratio).
void cell_pairs(const charm_cell *cell, bool split_radii, Pairs &P)
{
    const size_t nlat = cell->nlat;
    const bool even = nlat % 2 == 0;
    bool symm = nlat > 1;
    for (size_t i = 0; i < nlat && symm; i++)
        if (!nearly_equal(cell->latmin[i], -cell->latmax[nlat - i - 1],
                          charm_glob_threshold2))
            symm = false;
    const size_t nlatdo = symm ? (nlat + 1 - (even ? 1 : 0)) / 2 : nlat;
    P.row_n.clear();
    P.row_s.clear();
    std::vector<int> extra;
    for (size_t i = 0; i < nlatdo; i++)
    {
        const bool s = symm && !(!even && i == nlatdo - 1);
        int mi = s ? (int)(nlat - 1 - i) : -1;
        if (mi >= 0 && split_radii && cell->r[mi] != cell->r[i])
        {
            extra.push_back(mi);
            mi = -1;
        }
        P.row_n.push_back((int)i);
        P.row_s.push_back(mi);
    }
    for (int e : extra)
    {
        P.row_n.push_back(e);
        P.row_s.push_back(-1);
    }
}

// Geometry [8][np] of the pairs (CellArgs::geo) with the block-mean scale
// mur / ((sin latmax - sin latmin) dlon) of each pair's northern row
// (src/shs/shs_grd_fft.c:83-92 uses it for the mirror row too)
Status cell_geometry(Context &c, const charm_cell *cell, const Pairs &P,
                     double R, bool rr, double mur, double dlon, double **dgeo,
                     int **drows)
{
    Status st;
    const int np = (int)P.row_n.size();
    const size_t bytes = (size_t)np * (8 * 8 + 2 * 4);
    void *hp = nullptr;
    CB_TRY(pinned(c, bytes, &hp));
    double *h = static_cast<double *>(hp);
    int *hr = reinterpret_cast<int *>(h + 8 * (size_t)np);
    for (int p = 0; p < np; p++)
    {
        const int i = P.row_n[p];
        const double la1 = cell->latmin[i], la2 = cell->latmax[i];
        const double t1 = std::sin(la1), t2 = std::sin(la2);
        h[0 * np + p] = t1;
        h[1 * np + p] = std::cos(la1);
        h[2 * np + p] = t2;
        h[3 * np + p] = std::cos(la2);
        h[4 * np + p] = rr ? R / cell->r[i] : 1.0;
        h[5 * np + p] = mur / ((t2 - t1) * dlon);
        h[6 * np + p] = la1;
        h[7 * np + p] = la2;
        hr[p] = P.row_n[p];
        hr[np + p] = P.row_s[p];
    }
    void *d = nullptr;
    CB_TRY(buf(c, "geo", bytes, &d));
    CB_CUDA(cudaMemcpyAsync(d, hp, bytes, cudaMemcpyHostToDevice, c.stream),
            st);
    *dgeo = static_cast<double *>(d);
    *drows = reinterpret_cast<int *>(*dgeo + 8 * (size_t)np);
    return st;
}

Status shs_cell_grid(Context &c, const charm_cell *cell, const CoefIn &in,
                     unsigned long nmax, double *f_host, double *d_f)
{
    Status st;
    const double thr = charm_glob_threshold;
    const size_t nlat = cell->nlat, nlon = cell->nlon;
    double dlon = 0.0;
    CB_TRY(cell_grd_lons(cell, &dlon));
    // src/shs/shs_grd_cell_fft_check.c:17-60
    const bool use_fft =
        nlon > 1 && (nlon - 1) / 2 >= nmax &&
        nearly_equal(cell->lonmin[0], 0.0, thr) &&
        nearly_equal(cell->lonmax[nlon - 1], 2.0 * PI, thr) &&
        nearly_equal(cell->lonmin[1], cell->lonmax[0], thr);
    CB_TRY(check_cells(cell));

    // radius ratios R / r (shs_cell_grd.c:650-668); exactly 1 when r == R
    bool rr = false;
    for (size_t i = 0; i < nlat; i++)
        rr |= cell->r[i] != in.r;
    Pairs P;
    cell_pairs(cell, rr, P);
    const int np = (int)P.row_n.size();
    double *dgeo = nullptr;
    int *drows = nullptr;
    CB_TRY(cell_geometry(c, cell, P, in.r, rr, in.mu / in.r, dlon, &dgeo,
                         &drows));

    Tabs tab;
    CB_TRY(tables(c, (long long)nmax, &tab));
    CellTabs ctab;
    CB_TRY(cell_tables(c, (long long)nmax, &ctab));
    double2 *dcs = nullptr;
    CB_TRY(coef_to_device(c, in, nmax, tab, &dcs));
    double *imm = nullptr;
    CB_TRY(dbuf(c, "cell_imm", (size_t)np * (nmax + 1), &imm));

    const int ldf = use_fft ? (int)(nlon / 2 + 1) : (int)(nmax + 1);
    double2 *lc = nullptr;
    CB_TRY(dbuf(c, "lumped", (size_t)nlat * ldf, &lc));
    double *fg = d_f;
    double *f_dev_unaligned = nullptr;
    if (fg && use_fft && nlon % 2 == 0 &&
        reinterpret_cast<uintptr_t>(fg) % 16 != 0)
    {
        f_dev_unaligned = fg;
        fg = nullptr;
    }
    if (!fg)
        CB_TRY(dbuf(c, "fgrid", nlat * nlon, &fg));
    const RfftArgs *rf = nullptr, *rfq = nullptr;
    if (use_fft)
    {
        CB_TRY(row_fft(c, (long long)nlon, &rf));
        CB_TRY(row_fft_quarter(c, (long long)nlon, rf, &rfq));
    }
    unsigned *d_status;
    unsigned long long *d_counter;
    CB_TRY(status_words(c, &d_status, &d_counter));

    CellArgs A{};
    A.nmax = (long long)nmax;
    A.npairs = np;
    // two adjacent pairs per lane when the rows are aligned (each pair of
    // rows shares a boundary) and there are enough pairs
    bool shared = np >= 512;
    for (int p = 0; shared && p + 1 < np; p += 2)
        shared = cell->latmin[P.row_n[p]] == cell->latmax[P.row_n[p + 1]];
    A.ntiles = shared ? (np + 63) / 64 : (np + 31) / 32;
    A.nitems = (long long)(nmax + 1) * A.ntiles;
    A.tb = tab.tb;
    A.tc = tab.tc;
    A.tmul = tab.tmul;
    A.ldmul = tab.ldmul;
    A.sg = tab.sg;
    A.dm = tab.dm;
    A.gm = ctab.gm;
    A.cs = dcs;
    A.hn = ctab.hn;
    A.zn = ctab.zn;
    A.geo = dgeo;
    A.imm = imm;
    A.row_n = drows;
    A.row_s = drows + np;
    A.dlon = dlon;
    A.fft = use_fft ? 1 : 0;
    A.ldf = ldf;
    A.out = lc;
    A.polar_thr = polar_threshold(nmax);
    A.counter = d_counter;
    A.status = d_status;
    {
        Scope sc(c, TIMER_PREP);
        CB_CUDA(launch_cell_imm(A, c.stream), st);
    }
    {
        const int grid = (int)std::min<long long>((A.nitems + 3) / 4,
                                                  (long long)c.num_sms * 8);
        Scope sc(c, TIMER_SHS);
        CB_CUDA(launch_shs_cell(A, rr, shared, std::max(grid, 1), c.stream),
                st);
    }
    if (rf)
    {
        RfftArgs R = *synth_plan(rf, rfq, (long long)nmax);
        R.nrows = (long long)nlat;
        R.x = fg;
        R.ldx = (long long)nlon;
        R.X = lc;
        R.ldX = ldf;
        R.kmax = (int)nmax;
        Scope sc(c, TIMER_FFT);
        CB_CUDA(launch_rfft(R, true, c.stream), st);
    }
    else
    {
        // sums at the cell centres lon0 + j dlon (shs_grd_lr.c:145-190)
        std::vector<double> lon(nlon);
        const double lon0 = (cell->lonmin[0] + cell->lonmax[0]) / 2.0;
        for (size_t j = 0; j < nlon; j++)
            lon[j] = lon0 + (double)j * dlon;
        double *dlon_arr = nullptr;
        CB_TRY(dbuf(c, "lon", nlon, &dlon_arr));
        CB_CUDA(cudaMemcpyAsync(dlon_arr, lon.data(), nlon * 8,
                                cudaMemcpyHostToDevice, c.stream), st);
        {
            Scope sc(c, TIMER_LON);
            CB_CUDA(launch_lon_direct(1, (int)nlat, (int)nlon,
                                      (long long)nmax, lc, ldf, dlon_arr, fg,
                                      c.stream), st);
        }
        // lon must outlive the copy
        CB_CUDA(cudaStreamSynchronize(c.stream), st);
    }
    if (f_dev_unaligned)
        CB_CUDA(cudaMemcpyAsync(f_dev_unaligned, fg, nlat * nlon * 8,
                                cudaMemcpyDeviceToDevice, c.stream), st);
    if (!d_f)
        CB_CUDA(cudaMemcpyAsync(f_host, fg, nlat * nlon * 8,
                                cudaMemcpyDeviceToHost, c.stream), st);
    return finish(c, d_status);
}

// src/shs/shs_cell_sctr.c: one cell per (latmin, latmax, lonmin, lonmax, r)
Status shs_cell_sctr(Context &c, const charm_cell *cell, const CoefIn &in,
                     unsigned long nmax, double *f_host, double *d_f)
{
    Status st;
    CB_TRY(check_cells(cell));
    const size_t n = cell->ncell;
    bool rr = false;
    for (size_t i = 0; i < n; i++)
        rr |= cell->r[i] != in.r;
    Pairs P;
    for (size_t i = 0; i < n; i++)
    {
        P.row_n.push_back((int)i);
        P.row_s.push_back(-1);
    }
    double *dgeo = nullptr;
    int *drows = nullptr;
    CB_TRY(cell_geometry(c, cell, P, in.r, rr, in.mu / in.r, 1.0, &dgeo,
                         &drows));
    std::vector<double> lh(2 * n);
    for (size_t i = 0; i < n; i++)
    {
        lh[i] = cell->lonmin[i] + cell->lonmax[i];
        lh[n + i] = cell->lonmax[i] - cell->lonmin[i];
    }
    double *dl = nullptr;
    CB_TRY(dbuf(c, "cell_lon", 2 * n, &dl));
    CB_CUDA(cudaMemcpyAsync(dl, lh.data(), 2 * n * 8, cudaMemcpyHostToDevice,
                            c.stream), st);

    Tabs tab;
    CB_TRY(tables(c, (long long)nmax, &tab));
    CellTabs ctab;
    CB_TRY(cell_tables(c, (long long)nmax, &ctab));
    double2 *dcs = nullptr;
    CB_TRY(coef_to_device(c, in, nmax, tab, &dcs));
    double *fo = d_f;
    if (!fo)
        CB_TRY(dbuf(c, "fgrid", n, &fo));
    unsigned *d_status;
    unsigned long long *d_counter;
    CB_TRY(status_words(c, &d_status, &d_counter));

    CellArgs A{};
    A.nmax = (long long)nmax;
    A.npairs = (int)n;
    A.ntiles = (int)((n + 31) / 32);
    A.nitems = A.ntiles;
    A.tb = tab.tb;
    A.tc = tab.tc;
    A.tmul = tab.tmul;
    A.ldmul = tab.ldmul;
    A.sg = tab.sg;
    A.dm = tab.dm;
    A.gm = ctab.gm;
    A.cs = dcs;
    A.hn = ctab.hn;
    A.zn = ctab.zn;
    A.geo = dgeo;
    A.polar_thr = polar_threshold(nmax);
    A.counter = d_counter;
    A.status = d_status;
    A.lonsum = dl;
    A.dlonc = dl + n;
    A.fout = fo;
    A.mur = in.mu / in.r;
    {
        const int grid = (int)std::min<long long>((A.nitems + 3) / 4,
                                                  (long long)c.num_sms * 8);
        Scope sc(c, TIMER_SCTR);
        CB_CUDA(launch_shs_cell_sctr(A, rr, std::max(grid, 1), c.stream), st);
    }
    if (!d_f)
        CB_CUDA(cudaMemcpyAsync(f_host, fo, n * 8, cudaMemcpyDeviceToHost,
                                c.stream), st);
    // lh must outlive its copy: finish() synchronises
    return finish(c, d_status);
}

// src/sha/sha_cell.c:37-1487 (CHARM_SHA_CELL_AQ)
Status sha_cell_grid(Context &c, const charm_cell *cell, const double *f_host,
                     const double *d_fin, unsigned long nmax, double mu,
                     double R, unsigned long shc_nmax, double *const *hc,
                     double *const *hs, double *d_c, double *d_s)
{
    Status st;
    const double thr = charm_glob_threshold;
    const size_t nlat = cell->nlat, nlon = cell->nlon;
    auto fail = [&](const char *msg) {
        st.code = CHARM_EFUNCARG;
        st.msg = msg;
        return st;
    };
    const double r0 = cell->r[0];
    for (size_t i = 1; i < nlat; i++)
        if (!nearly_equal(cell->r[i], r0, thr))
            return fail("All spherical radii in \"cell->r\" must be equal.");
    if (!nearly_equal(cell->latmax[0], PI / 2.0, thr))
        return fail("\"cell->latmax[0]\" has to be equal to \"PI / 2.0\" "
                    "within the \"threshold\".");
    if (nlat < nmax + 1)
        return fail("Not enough data in the latitudinal direction.  The "
                    "required minimum is \"nmax + 1\".");
    if (!nearly_equal(cell->latmin[nlat - 1], -PI / 2.0, thr))
        return fail("\"cell->latmin[cell->nlat - 1]\" has to be equal to "
                    "\"-PI / 2.0\" within the \"threshold\".");
    for (size_t i = 0; i + 1 < nlat; i++)
        if (!nearly_equal(cell->latmin[i], cell->latmax[i + 1], thr))
            return fail("The grid cells are not nicely aligned in the "
                        "latitudinal direction.  It must hold that "
                        "\"cell->latmin[i] == cell->latmax[i + 1]\" for all "
                        "\"i = 0, 1, ..., cell->nlat - 2\" with "
                        "\"cell->nlat > 1\".");
    if (nlon < 2 * nmax + 1)
        return fail("Not enough data in the longitudinal direction.  The "
                    "required minimum is \"2 * nmax + 1\".");
    if (!nearly_equal(cell->lonmin[0], 0.0, thr))
        return fail("\"cell->lonmin[0]\" has to be equal to \"0.0\" within "
                    "the \"threshold\".");
    if (!nearly_equal(cell->lonmax[nlon - 1], 2.0 * PI, thr))
        return fail("\"cell->lonmax[cell->nlon - 1]\" has to be equal to "
                    "\"2.0 * PI\" within the \"threshold\".");
    double dlon = 0.0;
    CB_TRY(cell_grd_lons(cell, &dlon));
    if (nlon > 1 && !nearly_equal(cell->lonmin[1], cell->lonmax[0], thr))
        return fail("The grid cells are not nicely aligned in the "
                    "longitudinal direction.  It must hold that "
                    "\"cell->lonmin[j + 1] == cell->lonmax[j]\" for all "
                    "\"j = 0, 1, ..., cell->nlon - 2\" with "
                    "\"cell->nlon > 1\".");
    CB_TRY(check_cells(cell));

    Pairs P;
    cell_pairs(cell, false, P);
    const int np = (int)P.row_n.size();
    double *dgeo = nullptr;
    int *drows = nullptr;
    CB_TRY(cell_geometry(c, cell, P, R, false, 1.0, dlon, &dgeo, &drows));
    Tabs tab;
    CB_TRY(tables(c, (long long)nmax, &tab));
    CellTabs ctab;
    CB_TRY(cell_tables(c, (long long)nmax, &ctab));
    double *imm = nullptr;
    CB_TRY(dbuf(c, "cell_imm", (size_t)np * (nmax + 1), &imm));

    // block means on the device and r2c along the rows
    const double *fg = d_fin;
    if (!fg || reinterpret_cast<uintptr_t>(fg) % 16 != 0)
    {
        double *fdev = nullptr;
        CB_TRY(dbuf(c, "fgrid", nlat * nlon, &fdev));
        if (fg)
            CB_CUDA(cudaMemcpyAsync(fdev, fg, nlat * nlon * 8,
                                    cudaMemcpyDeviceToDevice, c.stream), st);
        else
            CB_CUDA(cudaMemcpyAsync(fdev, f_host, nlat * nlon * 8,
                                    cudaMemcpyHostToDevice, c.stream), st);
        fg = fdev;
    }
    const int ldF = (int)(nlon / 2 + 1);
    double2 *F = nullptr;
    CB_TRY(dbuf(c, "lumped", nlat * (size_t)ldF, &F));
    // even rows of 64 cells or more: the forward row transform of rfft.cu;
    // odd and short rows: the direct DFT
    const RfftArgs *rf = nullptr;
    if (nlon % 2 == 0 && nlon >= 64)
        CB_TRY(row_fft(c, (long long)nlon, &rf));
    {
        Scope sc(c, TIMER_FFT);
        if (rf)
        {
            RfftArgs Rg = *rf;
            Rg.nrows = (long long)nlat;
            Rg.x = const_cast<double *>(fg);
            Rg.ldx = (long long)nlon;
            Rg.X = F;
            Rg.ldX = ldF;
            Rg.kmax = (int)nmax;
            CB_CUDA(launch_rfft(Rg, false, c.stream), st);
        }
        else
            CB_CUDA(launch_dft_rows_fwd((long long)nlat, (long long)nlon,
                                        (int)nmax, fg, (long long)nlon, F,
                                        ldF, c.stream), st);
    }

    unsigned *d_status;
    unsigned long long *d_counter;
    CB_TRY(status_words(c, &d_status, &d_counter));
    const long long T = (long long)(nmax + 1) * (nmax + 2) / 2;
    // two cell-row pairs per lane once there are enough of them; adjacent
    // ones (pairs 2l, 2l + 1) when each such pair of rows shares a
    // boundary, which the kernel then carries once
    const int K = np >= 512 ? 2 : 1;
    bool shared = K == 2;
    for (int p = 0; shared && p + 1 < np; p += 2)
        shared = cell->latmin[P.row_n[p]] == cell->latmax[P.row_n[p + 1]];
    const int ntiles = (np + 32 * K - 1) / (32 * K);
    const long long slots = (long long)c.num_sms * 8 * 4;
    long long G = std::max<long long>(1, (2 * slots + nmax) / (nmax + 1));
    G = std::min<long long>(G, ntiles);
    const int tpg = (int)((ntiles + G - 1) / G);
    G = (ntiles + tpg - 1) / tpg;
    double2 *part = nullptr;
    CB_TRY(dbuf(c, "sha_part", (size_t)G * T, &part));

    CellArgs A{};
    A.nmax = (long long)nmax;
    A.npairs = np;
    A.ntiles = ntiles;
    A.ngroups = (int)G;
    A.tiles_per_group = tpg;
    A.nitems = (long long)(nmax + 1) * G;
    A.tb = tab.tb;
    A.tc = tab.tc;
    A.tmul = tab.tmul;
    A.ldmul = tab.ldmul;
    A.sg = tab.sg;
    A.dm = tab.dm;
    A.gm = ctab.gm;
    A.hn = ctab.hn;
    A.zn = ctab.zn;
    A.geo = dgeo;
    A.imm = imm;
    A.row_n = drows;
    A.row_s = drows + np;
    A.dlon = dlon;
    A.polar_thr = polar_threshold(nmax);
    A.counter = d_counter;
    A.status = d_status;
    A.F = F;
    A.ldF = ldF;
    A.part = part;
    {
        Scope sc(c, TIMER_PREP);
        CB_CUDA(launch_cell_imm(A, c.stream), st);
    }
    {
        const int grid = (int)std::min<long long>((A.nitems + 3) / 4,
                                                  (long long)c.num_sms * 8);
        Scope sc(c, TIMER_SHA);
        CB_CUDA(launch_sha_cell(A, K, shared, std::max(grid, 1), c.stream),
                st);
    }

    // 1 / (4 pi) r0 / mu and the rescaling from r0 to R
    // (sha_cell.c:1420-1480, src/shc/shc_rescale.c)
    const unsigned long sn = shc_nmax;
    double *dres = nullptr;
    std::vector<double> res;
    if (!nearly_equal(R, r0, thr))
    {
        const double r_ratio = r0 / R;
        res.resize(sn + 1);
        double tmp2 = r_ratio;
        res[0] = 1.0;
        for (unsigned long n = 1; n <= sn; n++)
        {
            res[n] = tmp2;
            tmp2 *= r_ratio;
        }
        CB_TRY(dbuf(c, "sha_rescale", sn + 1, &dres));
        CB_CUDA(cudaMemcpyAsync(dres, res.data(), (sn + 1) * 8,
                                cudaMemcpyHostToDevice, c.stream), st);
    }
    const long long Ts = (long long)(sn + 1) * (sn + 2) / 2;
    double *oc = d_c, *os = d_s;
    if (!oc)
    {
        double *dout = nullptr;
        CB_TRY(dbuf(c, "shc_out", (size_t)(2 * Ts), &dout));
        oc = dout;
        os = dout + Ts;
    }
    {
        Scope sc(c, TIMER_PREP);
        CB_CUDA(launch_sha_reduce((long long)nmax, (long long)sn, (int)G, T,
                                  part, tab.tc, dres,
                                  1.0 / (4.0 * PI) * (r0 / mu), oc, os,
                                  c.stream),
                st);
    }
    if (!d_c)
    {
        CB_TRY(download_tri(c, oc, sn, hc));
        CB_TRY(download_tri(c, os, sn, hs));
    }
    return finish(c, d_status);
}

// ---------------------------------------------------------------------------
// Coefficient files streamed to the device
// ---------------------------------------------------------------------------
// A binary coefficient file (src/shc/shc_read_bin.c layout) into device
// triangles of degree shc_nmax.  The destination of a range of orders is
// contiguous in the order-major triangle, so each chunk of orders is laid
// out in a page-locked buffer exactly as on the device (the file's first
// nmax + 1 - m values of column m, zeros up to shc_nmax) and copied with one
// call; two buffers alternate, so that reading chunk k + 1 from the file
// overlaps the copy of chunk k.
Status shc_read_bin_dev_impl(Context &c, const char *path, unsigned long nmax,
                             unsigned long shc_nmax, double *d_c, double *d_s,
                             double *mu, double *r, unsigned long *nmax_file)
{
    Status st;
    FILE *fp = std::fopen(path, "rb");
    if (!fp)
    {
        st.code = CHARM_EFILEIO;
        st.msg = std::string("Couldn't open \"") + path + "\".";
        return st;
    }
    struct Closer
    {
        FILE *f;
        ~Closer() { std::fclose(f); }
    } closer{fp};
    unsigned long nf = 0;
    double hdr[2];
    if (std::fread(&nf, sizeof nf, 1, fp) != 1 ||
        std::fread(hdr, sizeof(double), 2, fp) != 2)
    {
        st.code = CHARM_EFILEIO;
        st.msg = "Failed to read the header of the coefficient file.";
        return st;
    }
    if (nmax > nf)
    {
        st.code = CHARM_EFUNCARG;
        st.msg = "Not enough coefficients in the input file for the maximum "
                 "harmonic degree \"nmax\".";
        return st;
    }
    if (nmax > shc_nmax)
    {
        st.code = CHARM_EFUNCARG;
        st.msg = "\"nmax\" cannot be larger than \"shc_nmax\".";
        return st;
    }
    *nmax_file = nf;
    *mu = hdr[0];
    *r = hdr[1];
    constexpr size_t CHUNK = 4u << 20;   // doubles per buffer (32 MB)
    void *hp = nullptr;
    CB_TRY(pinned(c, 2 * CHUNK * sizeof(double), &hp));
    double *buf[2] = {static_cast<double *>(hp),
                      static_cast<double *>(hp) + CHUNK};
    // the copy stream starts after the work already on the stream (buffers
    // the caller may still read)
    CB_CUDA(cudaEventRecord(c.band_ev[EV_START], c.stream), st);
    CB_CUDA(cudaStreamWaitEvent(c.copy_stream, c.band_ev[EV_START], 0), st);
    bool used[2] = {false, false};
    int nb = 0;
    for (int part = 0; part < 2; part++)
    {
        double *dst = part ? d_s : d_c;
        long long m = 0;
        while (m <= (long long)shc_nmax)
        {
            // orders [m, m1) of this chunk
            long long m1 = m;
            size_t len = 0;
            while (m1 <= (long long)shc_nmax &&
                   (len == 0 || len + (size_t)(shc_nmax + 1 - m1) <= CHUNK))
            {
                len += (size_t)(shc_nmax + 1 - m1);
                m1++;
            }
            if (len > CHUNK)
            {
                st.code = CHARM_EFUNCARG;
                st.msg = "A coefficient column exceeds the staging buffer.";
                return st;
            }
            const int b = nb & 1;
            if (used[b])
                CB_CUDA(cudaEventSynchronize(c.band_ev[b]), st);
            double *h = buf[b];
            size_t o = 0;
            for (long long mm = m; mm < m1; mm++)
            {
                const size_t col = (size_t)(shc_nmax + 1 - mm);
                size_t got = 0;
                if (mm <= (long long)nmax)
                {
                    got = (size_t)(nmax + 1 - mm);
                    if (std::fread(h + o, sizeof(double), got, fp) != got ||
                        (nf > nmax &&
                         std::fseek(fp, (long)((nf - nmax) * sizeof(double)),
                                    SEEK_CUR) != 0))
                    {
                        st.code = CHARM_EFILEIO;
                        st.msg = part ? "Failed to read the \"S\" coefficients."
                                      : "Failed to read the \"C\" coefficients.";
                        return st;
                    }
                }
                std::memset(h + o + got, 0, (col - got) * sizeof(double));
                o += col;
            }
            CB_CUDA(cudaMemcpyAsync(dst + tri_start((long long)shc_nmax, m), h,
                                    len * sizeof(double),
                                    cudaMemcpyHostToDevice, c.copy_stream),
                    st);
            CB_CUDA(cudaEventRecord(c.band_ev[b], c.copy_stream), st);
            used[b] = true;
            nb++;
            m = m1;
        }
        // the file position of the next part: the rest of this part's
        // columns (the file's columns m hold nf + 1 - m values; the loop
        // read the first nmax + 1 - m of the columns m <= nmax)
        if (part == 0)
        {
            const long long Tf = (long long)(nf + 1) * (nf + 2) / 2;
            const long off = (long)(sizeof(unsigned long) +
                                    2 * sizeof(double) +
                                    (size_t)Tf * sizeof(double));
            if (std::fseek(fp, off, SEEK_SET) != 0)
            {
                st.code = CHARM_EFILEIO;
                st.msg = "Failed to read the \"S\" coefficients.";
                return st;
            }
        }
    }
    CB_CUDA(cudaStreamSynchronize(c.copy_stream), st);
    return st;
}

// ---------------------------------------------------------------------------
// Spectral gravity forward modelling, global (src/gfm/gfm_sgfm.c)
// ---------------------------------------------------------------------------
// gfm_sgfm.c global_vnmc: c times the degree factor of power p and density
// order i, in CHarm's order of operations
void gfm_vnmc(unsigned long nmax, unsigned p, unsigned i, double cc,
              std::vector<double> &v)
{
    v.assign(nmax + 1, 0.0);
    const double pr = (double)p;
    for (unsigned long n = 0; n <= nmax; n++)
    {
        const double npip3 = (double)(n + i + 3);
        double snpi = npip3 / pr;
        for (unsigned pt = 1; pt < p; pt++)
            snpi *= (npip3 - (double)pt) / (pr - (double)pt);
        snpi *= 2.0 / ((2.0 * (double)n + 1.0) * npip3);
        v[n] = cc * snpi;
    }
}

// Writes the degree-n triangles (c, s) on the device as a binary
// coefficient file path-p<P>-i<I>.shcs (gfm_sgfm.c export_shcs_powers with
// the "bin" format).
Status gfm_export(Context &c, const double *dc, const double *ds,
                  unsigned long n, double mu, double r, const char *path,
                  unsigned p, unsigned pmax, unsigned i, unsigned imax)
{
    Status st;
    auto digits = [](unsigned x) {
        return x > 0 ? (int)std::ceil(std::log10((double)x)) : 1;
    };
    char name[CHARM_ERR_MAX_FILE];
    const int ret = std::snprintf(name, sizeof name, "%s-p%0*u-i%0*u.shcs",
                                  path, digits(pmax), p, digits(imax), i);
    if (ret <= 0 || (size_t)ret >= sizeof name)
    {
        st.code = CHARM_EFUNCARG;
        st.msg = "Too small string buffer for the output file name.";
        return st;
    }
    const size_t T = (size_t)(n + 1) * (n + 2) / 2;
    std::vector<double> hc(T), hs(T);
    CB_CUDA(cudaMemcpyAsync(hc.data(), dc, T * 8, cudaMemcpyDeviceToHost,
                            c.stream), st);
    CB_CUDA(cudaMemcpyAsync(hs.data(), ds, T * 8, cudaMemcpyDeviceToHost,
                            c.stream), st);
    CB_CUDA(cudaStreamSynchronize(c.stream), st);
    FILE *fp = std::fopen(name, "wb");
    if (!fp)
    {
        st.code = CHARM_EFILEIO;
        st.msg = std::string("Couldn't create \"") + name + "\".";
        return st;
    }
    const bool ok = std::fwrite(&n, sizeof n, 1, fp) == 1 &&
                    std::fwrite(&mu, 8, 1, fp) == 1 &&
                    std::fwrite(&r, 8, 1, fp) == 1 &&
                    std::fwrite(hc.data(), 8, T, fp) == T &&
                    std::fwrite(hs.data(), 8, T, fp) == T;
    std::fclose(fp);
    if (!ok)
    {
        st.code = CHARM_EFILEIO;
        st.msg = std::string("Failed to write \"") + name + "\".";
    }
    return st;
}

Status gfm_global_impl(Context &c, const GfmArgs &g)
{
    Status st;
    const bool rho_const = g.density == nullptr;
    const unsigned imax = rho_const ? 0u : g.density_order;
    // get_max_nmax(density_nmax, density_order) of gfm_sgfm.c: the largest
    // of the first density_order entries (the first entry when 0)
    unsigned long dmax = 0;
    if (!rho_const)
    {
        dmax = g.density_nmax[0];
        for (unsigned k = 1; k < g.density_order; k++)
            dmax = std::max(dmax, g.density_nmax[k]);
    }
    double cc = (2.0 * PI * std::pow(g.R, 3)) / g.mass;
    if (rho_const)
        cc *= g.rho;
    const double gm = g.G * g.mass;
    const unsigned long np = g.nmax_pot;
    const size_t Tp = (size_t)(np + 1) * (np + 2) / 2;

    // inputs and the potential accumulators on the device
    const unsigned long sn = g.shape->nmax;
    const size_t Tsh = (size_t)(sn + 1) * (sn + 2) / 2;
    double *dshape = nullptr;
    CB_TRY(dbuf(c, "gfm_shape_tri", 2 * Tsh, &dshape));
    CB_TRY(upload_tri(c, g.shape->c, sn, dshape));
    CB_TRY(upload_tri(c, g.shape->s, sn, dshape + Tsh));
    std::vector<double *> ddens(imax + 1, nullptr);
    for (unsigned i = 0; !rho_const && i <= imax; i++)
    {
        const unsigned long dn = g.density[i]->nmax;
        const size_t Td = (size_t)(dn + 1) * (dn + 2) / 2;
        CB_TRY(dbuf(c, "gfm_dens_tri" + std::to_string(i), 2 * Td,
                    &ddens[i]));
        CB_TRY(upload_tri(c, g.density[i]->c, dn, ddens[i]));
        CB_TRY(upload_tri(c, g.density[i]->s, dn, ddens[i] + Td));
    }
    double *dpot = nullptr;
    if (g.pot)
    {
        CB_TRY(dbuf(c, "gfm_pot", 2 * Tp, &dpot));
        CB_CUDA(cudaMemsetAsync(dpot, 0, 2 * Tp * 8, c.stream), st);
    }
    // the degree factors of every (power, density order), uploaded once
    const unsigned npow = g.pmax - g.pmin + 1;
    const size_t nv = (size_t)npow * (imax + 1) * (np + 1);
    std::vector<double> vh(nv, 0.0), v;
    for (unsigned p = g.pmin; p <= g.pmax; p++)
        for (unsigned i = 0; i <= imax; i++)
        {
            const unsigned long nmaxp = p * g.shape_nmax + dmax;
            gfm_vnmc(nmaxp > np ? np : nmaxp, p, i, cc, v);
            std::copy(v.begin(), v.end(),
                      vh.begin() + ((size_t)(p - g.pmin) * (imax + 1) + i) *
                                       (np + 1));
        }
    double *dv = nullptr;
    CB_TRY(dbuf(c, "gfm_v", nv, &dv));
    CB_CUDA(cudaMemcpyAsync(dv, vh.data(), nv * 8, cudaMemcpyHostToDevice,
                            c.stream), st);
    // (a pageable source: the copy has read vh when the call returns)

    // The shape and the densities of one power share its grid: one batched
    // synthesis forms all of them (sets of their own degrees, one launch)
    // when their grids and lumped coefficients (about as large again) fit
    // the budget (default: a quarter of the free
    // device memory; CHARM_B200_GFM_BATCH_BYTES overrides it, 0 turns the
    // batching off), otherwise one synthesis per set.
    const size_t nsets = 1 + (rho_const ? 0 : imax + 1);
    size_t budget = 0;
    {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) == cudaSuccess)
            budget = fr / 4;
        cudaGetLastError();
        const char *e = std::getenv("CHARM_B200_GFM_BATCH_BYTES");
        if (e && *e)
            budget = (size_t)std::strtoull(e, nullptr, 10);
    }
    for (unsigned p = g.pmin; p <= g.pmax; p++)
    {
        const unsigned long nmaxp = p * g.shape_nmax + dmax;
        const unsigned long thr = nmaxp > np ? np : nmaxp;
        charm_point *grd = charm_crd_point_gl(nmaxp, 1.0);
        if (!grd)
        {
            st.code = CHARM_EFUNCARG;
            st.msg = "Failed to compute the Gauss--Legendre grid.";
            return st;
        }
        struct Free
        {
            charm_point *q;
            ~Free() { charm_crd_point_free(q); }
        } fr{grd};
        const size_t npt = grd->npoint;
        // fields: [0] the shape, [1 + i] density i (or, for a constant
        // density, [1] the power of the shape)
        std::vector<double *> fld(std::max<size_t>(nsets, 2), nullptr);
        for (size_t k = 0; k < fld.size(); k++)
            CB_TRY(dbuf(c, "gfm_f" + std::to_string(k), npt, &fld[k]));
        std::vector<unsigned long> nm_v(nsets), sn_v(nsets);
        std::vector<double> mu_v(nsets, 1.0);
        std::vector<const double *> dc_v(nsets), ds_v(nsets);
        nm_v[0] = g.shape_nmax;
        sn_v[0] = sn;
        dc_v[0] = dshape;
        ds_v[0] = dshape + Tsh;
        for (unsigned i = 0; !rho_const && i <= imax; i++)
        {
            const unsigned long dn = g.density[i]->nmax;
            nm_v[1 + i] = g.density_nmax[i];
            sn_v[1 + i] = dn;
            dc_v[1 + i] = ddens[i];
            ds_v[1 + i] = ddens[i] + (size_t)(dn + 1) * (dn + 2) / 2;
        }
        if (nsets > 1 && nsets * npt * 16 <= budget)
            CB_TRY(shs_batch(c, grd, nsets, nm_v.data(), sn_v.data(),
                             mu_v.data(), 1.0, dc_v.data(), ds_v.data(), 0,
                             fld.data()));
        else
            for (size_t k = 0; k < nsets; k++)
            {
                CoefIn in;
                in.nmax = sn_v[k];
                in.mu = 1.0;
                in.r = 1.0;
                in.dc = dc_v[k];
                in.ds = ds_v[k];
                CB_TRY(shs_grid(c, grd, in, nm_v[k], 0, 0, 0, 0, nullptr,
                                fld[k]));
            }
        const size_t Ta = (size_t)(thr + 1) * (thr + 2) / 2;
        double *da = nullptr;
        CB_TRY(dbuf(c, "gfm_a", 2 * Ta, &da));
        double Ri = 1.0;
        for (unsigned i = 0; i <= imax; i++)
        {
            double *frho = fld[1 + i];
            if (!rho_const)
            {
                CB_CUDA(launch_gfm_power(npt, fld[0], g.R, p, Ri, frho,
                                         nullptr, c.stream), st);
                Ri *= g.R;
            }
            else
                CB_CUDA(launch_gfm_power(npt, fld[0], g.R, p, 1.0, nullptr,
                                         frho, c.stream), st);
            CB_TRY(sha_grid(c, grd, nullptr, frho, thr, 1.0, 1.0, thr,
                            nullptr, nullptr, da, da + Ta));
            if (g.hro_path)
                CB_TRY(gfm_export(c, da, da + Ta, thr, 1.0, 1.0, g.hro_path,
                                  p, g.pmax, i, imax));
            const double *dvi =
                dv + ((size_t)(p - g.pmin) * (imax + 1) + i) * (np + 1);
            CB_CUDA(launch_gfm_accum((long long)thr, (long long)np, dvi, da,
                                     da + Ta, dpot, dpot ? dpot + Tp : nullptr,
                                     g.pot_path != nullptr, c.stream),
                    st);
            if (g.pot_path)
                CB_TRY(gfm_export(c, da, da + Ta, thr, gm, g.R, g.pot_path, p,
                                  g.pmax, i, imax));
        }
    }
    if (g.pot)
    {
        CB_TRY(download_tri(c, dpot, np, g.pot->c));
        CB_TRY(download_tri(c, dpot + Tp, np, g.pot->s));
        CB_CUDA(cudaStreamSynchronize(c.stream), st);
        g.pot->mu = gm;
        g.pot->r = g.R;
    }
    return st;
}

// ---------------------------------------------------------------------------
// Allocation-free analysis (charm_b200_sha_point_dev_static)
// ---------------------------------------------------------------------------
// The same kernels as sha_grid with the row transform of rfft.cu, every
// temporary carved from the fixed device scratch of sha_static.cu and every
// host-side staging array fixed in size, so that a call allocates neither
// device, pinned nor heap memory.  Its callers cannot allocate during the
// call (device memory owned by another allocator, or a loop that must not
// synchronise the device as cudaMalloc / cudaFree do).

constexpr long long STATIC_MAX_ROWS = 8192;  // grid latitudes served

struct StaticHost
{
    double r[2 * STATIC_NMAX + 4], ri[2 * STATIC_NMAX + 4];
    double smm[STATIC_NMAX + 1];
    double rescale[STATIC_NMAX + 1];
    double geo_d[4 * STATIC_MAX_ROWS];  // t, u, cw_n, cw_s per pair
    int geo_i[2 * STATIC_MAX_ROWS];     // row_n, row_s per pair
};
StaticHost g_static_host;

// per device: the scratch address (cudaGetSymbolAddress, once) and what
// the scratch currently holds
struct StaticDev
{
    unsigned char *base = nullptr;
    long long tab_nmax = -1;
    long long fft_L = -1, fft_nmax = -1;
};
constexpr int STATIC_MAX_DEVICES = 64;
StaticDev g_static_dev[STATIC_MAX_DEVICES];

struct Carve
{
    size_t off = 0;
    size_t take(size_t bytes)
    {
        size_t o = off;
        off = (off + bytes + 255) & ~(size_t)255;
        return o;
    }
};

Status sha_point_dev_static_impl(Context &c, const charm_point *pnt,
                                 const double *d_f, unsigned long nmax,
                                 double mu, double R, unsigned long shc_nmax,
                                 double *d_c, double *d_s)
{
    Status st;
    if (c.device < 0 || c.device >= STATIC_MAX_DEVICES)
    {
        st.code = CHARM_EFUNCARG;
        st.msg = "charm_b200_sha_point_dev_static serves device ordinals "
                 "below 64 only.";
        return st;
    }
    StaticDev &sd = g_static_dev[c.device];
    if (!sd.base)
    {
        void *p = nullptr;
        cudaError_t e = static_scratch_address(&p);
        if (e != cudaSuccess || !p)
        {
            cudaGetLastError();
            st.code = CHARM_EFUNCARG;
            st.msg = std::string("cudaGetSymbolAddress of the static scratch "
                                 "failed: ") +
                     cudaGetErrorString(e);
            return st;
        }
        CB_CUDA(rfft_set_smem(rfft_smem_bytes(9216)), st);
        // recorded only once the whole set-up has succeeded, so that a
        // failed set-up is retried by the next call
        sd.base = static_cast<unsigned char *>(p);
    }
    const long long N = (long long)nmax;
    const size_t nlat = pnt->nlat, nlon = pnt->nlon;
    if (N > STATIC_NMAX)
    {
        st.code = CHARM_EFUNCARG;
        st.msg = "charm_b200_sha_point_dev_static: nmax " +
                 std::to_string(N) + " exceeds the static scratch limit of " +
                 std::to_string(STATIC_NMAX) + ".";
        return st;
    }
    if ((long long)nlat > STATIC_MAX_ROWS)
    {
        st.code = CHARM_EFUNCARG;
        st.msg = "charm_b200_sha_point_dev_static: the grid has " +
                 std::to_string(nlat) + " latitudes; the limit is " +
                 std::to_string(STATIC_MAX_ROWS) + ".";
        return st;
    }
    RfftArgs RF{};
    if (!rfft_shape((long long)nlon, &RF) || RF.C > 1 || RF.odd)
    {
        st.code = CHARM_EFUNCARG;
        st.msg = "charm_b200_sha_point_dev_static: no shared-memory row "
                 "transform for rows of " +
                 std::to_string(nlon) + " longitudes.";
        return st;
    }
    if (reinterpret_cast<uintptr_t>(d_f) % 16 != 0)
    {
        st.code = CHARM_EFUNCARG;
        st.msg = "charm_b200_sha_point_dev_static: the grid values must "
                 "start on a 16-byte boundary.";
        return st;
    }

    // latitude pairs of a quadrature grid (the rules of grid_pairs for
    // GL / DH grids, src/shs/shs_point_grd.c:113-197)
    const bool dh = is_dh(pnt->type);
    const size_t pnt_nlat = dh ? nlat + 1 : nlat;
    const bool even = (pnt_nlat % 2) == 0;
    const bool symm = pnt_nlat != 1;
    const unsigned long nmax_grd = pnt->type == CHARM_CRD_POINT_GRID_GL
                                       ? nlat - 1
                                       : (nlat - 2) / 2;
    size_t equator = (size_t)-1;
    if (!(pnt->type == CHARM_CRD_POINT_GRID_GL && (nmax_grd % 2)))
        equator = nlat / 2;
    const int np =
        (int)(symm ? (pnt_nlat + 1 - (even ? 1 : 0)) / 2 : nlat);
    double cq = (pnt->type == CHARM_CRD_POINT_GRID_DH2)
                    ? PI / (double)(2 * nmax_grd + 2)
                    : PI / (double)(nmax_grd + 1);
    const double r0 = pnt->r[0];
    cq *= 1.0 / (4.0 * PI) * (r0 / mu);
    StaticHost &hs = g_static_host;
    for (int p = 0; p < np; p++)
    {
        int s = !symm ? 0 : ((dh && p == 0) ? 0 : ((size_t)p < equator));
        int rs = s ? (int)(pnt_nlat - p - 1) : -1;
        // sincos, as sha_grid computes the same geometry, so that both
        // paths see identical latitude terms
        sincos(pnt->lat[p], &hs.geo_d[p], &hs.geo_d[np + p]);
        hs.geo_d[2 * np + p] = cq * pnt->w[p];
        hs.geo_d[3 * np + p] = rs >= 0 ? cq * pnt->w[rs] : 0.0;
        hs.geo_i[p] = p;
        hs.geo_i[np + p] = rs;
    }

    // scratch layout: words, recurrence tables and transform tables first
    // (their offsets depend on nmax only, so they stay valid while nmax and
    // the row length repeat), then the per-call arrays
    const long long T = (N + 1) * (N + 2) / 2;
    const int ldmul = (int)((N + 1 + 63) / 64);
    const int K = choose_k_sha(np);
    const int ntiles = (np + 32 * K - 1) / (32 * K);
    Carve cv;
    const size_t o_words = cv.take(256);
    const size_t o_tb = cv.take((size_t)T * 16);
    const size_t o_tc = cv.take((size_t)T * 8);
    const size_t o_tmul = cv.take((size_t)(N + 1) * ldmul * 8);
    const size_t o_sg = cv.take((size_t)(2 * (N + 1)) * 8);
    const size_t o_r = cv.take((size_t)(2 * N + 4) * 8);
    const size_t o_ri = cv.take((size_t)(2 * N + 4) * 8);
    const size_t o_smm = cv.take((size_t)(N + 1) * 8);
    const size_t o_tw = cv.take((size_t)RF.M * 16);
    const size_t o_w = RF.direct ? 0 : cv.take((size_t)RF.H * 16);
    const size_t o_bh = RF.direct ? 0 : cv.take((size_t)RF.M * 16);
    const size_t o_ht = cv.take((size_t)(RF.H + 1) * 16);
    const size_t o_geod = cv.take((size_t)np * 32);
    const size_t o_geoi = cv.take((size_t)np * 8);
    const size_t o_res = cv.take((size_t)(N + 1) * 8);
    const size_t o_F = cv.take(nlat * (size_t)(N + 1) * 16);
    const size_t part_from = cv.off;
    // the groups of sha_grid, fewer when the partial sums would not fit
    long long slots = (long long)c.num_sms * 8 * 4;
    long long G = std::max<long long>(1, (2 * slots + N) / (N + 1));
    G = std::min<long long>(G, ntiles);
    int tpg = (int)((ntiles + G - 1) / G);
    G = (ntiles + tpg - 1) / tpg;
    while (part_from + (size_t)G * T * 16 > STATIC_SCRATCH_BYTES && G > 1)
    {
        tpg++;
        G = (ntiles + tpg - 1) / tpg;
    }
    const size_t need = part_from + (size_t)G * T * 16;
    if (need > STATIC_SCRATCH_BYTES)
    {
        st.code = CHARM_EFUNCARG;
        st.msg = "charm_b200_sha_point_dev_static: this grid and nmax need " +
                 std::to_string(need) + " bytes of static scratch; it has " +
                 std::to_string(STATIC_SCRATCH_BYTES) + ".";
        return st;
    }
    unsigned char *b = sd.base;
    unsigned *d_status = reinterpret_cast<unsigned *>(b + o_words);
    unsigned long long *d_counter =
        reinterpret_cast<unsigned long long *>(b + o_words + 64);
    double2 *tb = reinterpret_cast<double2 *>(b + o_tb);
    double *tc = reinterpret_cast<double *>(b + o_tc);
    double *tmul = reinterpret_cast<double *>(b + o_tmul);
    double *sg = reinterpret_cast<double *>(b + o_sg);

    // recurrence tables (kept while nmax repeats)
    if (sd.tab_nmax != N)
    {
        // the tables below overwrite the scratch: nothing cached stays
        // valid if a copy or launch fails before they are complete
        sd.tab_nmax = -1;
        sd.fft_L = -1;
        sd.fft_nmax = -1;
        for (long long k = 0; k <= 2 * N + 3; k++)
        {
            double w = std::sqrt((double)k);
            hs.r[k] = w;
            hs.ri[k] = k ? 1.0 / w : 0.0;
        }
        host_smm(N, hs.smm);
        double *dr = reinterpret_cast<double *>(b + o_r);
        double *dri = reinterpret_cast<double *>(b + o_ri);
        double *dsm = reinterpret_cast<double *>(b + o_smm);
        CB_CUDA(cudaMemcpyAsync(dr, hs.r, (size_t)(2 * N + 4) * 8,
                                cudaMemcpyHostToDevice, c.stream), st);
        CB_CUDA(cudaMemcpyAsync(dri, hs.ri, (size_t)(2 * N + 4) * 8,
                                cudaMemcpyHostToDevice, c.stream), st);
        CB_CUDA(cudaMemcpyAsync(dsm, hs.smm, (size_t)(N + 1) * 8,
                                cudaMemcpyHostToDevice, c.stream), st);
        CB_CUDA(launch_tables(N, dr, dri, dsm, tb, tc, tmul, ldmul, sg,
                              c.stream), st);
        c.launches++;
        sd.tab_nmax = N;
        sd.fft_L = -1;
    }
    // transform tables (kept while the row length and nmax repeat)
    RF.tw = reinterpret_cast<double2 *>(b + o_tw);
    RF.w = RF.direct ? nullptr : reinterpret_cast<double2 *>(b + o_w);
    RF.bh = RF.direct ? nullptr : reinterpret_cast<double2 *>(b + o_bh);
    RF.ht = reinterpret_cast<double2 *>(b + o_ht);
    if (sd.fft_L != (long long)nlon || sd.fft_nmax != N)
    {
        sd.fft_L = -1;
        sd.fft_nmax = -1;
        RfftArgs tmp = RF;
        CB_CUDA(launch_rfft_tables(tmp, const_cast<double2 *>(RF.tw),
                                   const_cast<double2 *>(RF.w),
                                   const_cast<double2 *>(RF.ht),
                                   const_cast<double2 *>(RF.bh), c.stream),
                st);
        c.launches += RF.direct ? 1 : 2;
        sd.fft_L = (long long)nlon;
        sd.fft_nmax = N;
    }

    // geometry and rescaling factors (pageable copies from fixed arrays)
    double *dgd = reinterpret_cast<double *>(b + o_geod);
    int *dgi = reinterpret_cast<int *>(b + o_geoi);
    if (np > 0)
    {
        // the four double arrays are contiguous per quantity in geo_d
        CB_CUDA(cudaMemcpyAsync(dgd, hs.geo_d, (size_t)np * 32,
                                cudaMemcpyHostToDevice, c.stream), st);
        CB_CUDA(cudaMemcpyAsync(dgi, hs.geo_i, (size_t)np * 8,
                                cudaMemcpyHostToDevice, c.stream), st);
    }
    double *dres = nullptr;
    if (!nearly_equal(R, r0, charm_glob_threshold))
    {
        // src/sha/sha_point.c:1088-1108 with src/shc/shc_rescale.c; only
        // degrees <= nmax carry nonzero coefficients
        double r_ratio = r0 / R, tmp2 = (mu / mu) * r_ratio;
        hs.rescale[0] = mu / mu;
        for (long long n = 1; n <= N; n++)
        {
            hs.rescale[n] = tmp2;
            tmp2 *= r_ratio;
        }
        dres = reinterpret_cast<double *>(b + o_res);
        CB_CUDA(cudaMemcpyAsync(dres, hs.rescale, (size_t)(N + 1) * 8,
                                cudaMemcpyHostToDevice, c.stream), st);
    }

    // r2c of the rows into the scratch, orders 0..nmax
    double2 *F = reinterpret_cast<double2 *>(b + o_F);
    RF.nrows = (long long)nlat;
    RF.x = const_cast<double *>(d_f);
    RF.ldx = (long long)nlon;
    RF.X = F;
    RF.ldX = N + 1;
    RF.kmax = (int)N;
    CB_CUDA(launch_rfft(RF, false, c.stream), st);
    c.launches++;

    // Legendre contraction with the partial sums in the scratch
    CB_CUDA(cudaMemsetAsync(b + o_words, 0, 256, c.stream), st);
    double2 *part = reinterpret_cast<double2 *>(b + part_from);
    ShaGridArgs A{};
    A.nmax = N;
    A.npairs = np;
    A.ntiles = ntiles;
    A.ngroups = (int)G;
    A.tiles_per_group = tpg;
    A.nitems = (N + 1) * G;
    A.tb = tb;
    A.tmul = tmul;
    A.ldmul = ldmul;
    A.sg = sg;
    A.t = dgd;
    A.u = dgd + np;
    A.cw_n = dgd + 2 * np;
    A.cw_s = dgd + 3 * np;
    A.row_n = dgi;
    A.row_s = dgi + np;
    A.F = F;
    A.ldF = (int)(N + 1);
    A.part = part;
    A.polar_thr = polar_threshold(nmax);
    A.counter = d_counter;
    A.status = d_status;
    int grid = (int)std::min<long long>((A.nitems + 3) / 4,
                                        (long long)c.num_sms * 8);
    CB_CUDA(launch_sha_grid(A, K, std::max(grid, 1), c.stream), st);
    c.launches++;
    CB_CUDA(launch_sha_reduce(N, (long long)shc_nmax, (int)G, T, part, tc,
                              dres, 1.0, d_c, d_s, c.stream), st);
    c.launches++;
    return finish(c, d_status);
}

} // namespace

// ---------------------------------------------------------------------------
// Public engine entry points
// ---------------------------------------------------------------------------
// A coefficient triangle whose columns lie contiguously in pageable host
// memory (null otherwise).
const double *pageable_tri(double *const *cols, unsigned long nmax)
{
    const double *base = contiguous_tri(cols, nmax);
    return (base && is_pageable(base)) ? base : nullptr;
}

Status shs_point(const charm_point *pnt, const charm_shc *shcs,
                 unsigned long nmax, int kgrad, int dr, int dlat, int dlon,
                 double **f)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    Context &c = g_ctx;
    CB_TRY(init(c));
    CoefIn in;
    in.nmax = shcs->nmax;
    in.mu = shcs->mu;
    in.r = shcs->r;
    in.hc = shcs->c;
    in.hs = shcs->s;
    const bool sctr = pnt->type == CHARM_CRD_POINT_SCATTERED;
    // pageable host arrays: the coefficients uploaded and the output
    // downloaded through the ring, the transform on device arrays
    double mur;
    int dorder, npar;
    mur_dorder(in.mu, in.r, kgrad, dr, dlat, dlon, &mur, &dorder, &npar);
    const double *pc = pageable_tri(shcs->c, shcs->nmax);
    const double *ps = pageable_tri(shcs->s, shcs->nmax);
    bool pf = false;
    for (int q = 0; q < npar && pnt->npoint > 0; q++)
        pf = pf || is_pageable(f[q]);
    if (pc && ps)
    {
        const size_t Ts = (size_t)(shcs->nmax + 1) * (shcs->nmax + 2) / 2;
        double *raw = nullptr;
        CB_TRY(dbuf(c, "stage_shc", 2 * Ts, &raw));
        CB_TRY(stage_h2d(c, raw, pc, Ts * 8));
        CB_TRY(stage_h2d(c, raw + Ts, ps, Ts * 8));
        in.hc = in.hs = nullptr;
        in.dc = raw;
        in.ds = raw + Ts;
    }
    if (pf)
    {
        const size_t np = pnt->npoint;
        double *dout = nullptr;
        CB_TRY(dbuf(c, "stage_out", (size_t)npar * np, &dout));
        CB_TRY(sctr ? shs_sctr(c, pnt, in, nmax, kgrad, dr, dlat, dlon,
                               nullptr, dout)
                    : shs_grid(c, pnt, in, nmax, kgrad, dr, dlat, dlon,
                               nullptr, dout));
        for (int q = 0; q < npar; q++)
            CB_TRY(stage_d2h(c, f[q], dout + (size_t)q * np, np * 8));
        return Status{};
    }
    if (sctr)
        return shs_sctr(c, pnt, in, nmax, kgrad, dr, dlat, dlon, f, nullptr);
    return shs_grid(c, pnt, in, nmax, kgrad, dr, dlat, dlon, f, nullptr);
}

Status shs_point_dev(const charm_point *pnt, unsigned long shc_nmax,
                     double mu, double r, const double *d_c,
                     const double *d_s, unsigned long nmax, int kgrad, int dr,
                     int dlat, int dlon, double *d_f)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    CB_TRY(init(g_ctx));
    CoefIn in;
    in.nmax = shc_nmax;
    in.mu = mu;
    in.r = r;
    in.dc = d_c;
    in.ds = d_s;
    if (pnt->type == CHARM_CRD_POINT_SCATTERED)
        return shs_sctr(g_ctx, pnt, in, nmax, kgrad, dr, dlat, dlon, nullptr,
                        d_f);
    return shs_grid(g_ctx, pnt, in, nmax, kgrad, dr, dlat, dlon, nullptr, d_f);
}

Status sha_point(const charm_point *pnt, const double *f, unsigned long nmax,
                 charm_shc *shcs)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    Context &c = g_ctx;
    CB_TRY(init(c));
    // pageable host arrays: the grid uploaded and the coefficients
    // downloaded through the ring, the analysis on device arrays
    const bool pf = pnt->npoint > 0 && is_pageable(f);
    const double *pc = pageable_tri(shcs->c, shcs->nmax);
    const double *ps = pageable_tri(shcs->s, shcs->nmax);
    const double *din = nullptr;
    if (pf)
    {
        double *d = nullptr;
        CB_TRY(dbuf(c, "stage_in", pnt->npoint, &d));
        CB_TRY(stage_h2d(c, d, f, pnt->npoint * 8));
        din = d;
    }
    if (pc && ps)
    {
        const size_t Ts = (size_t)(shcs->nmax + 1) * (shcs->nmax + 2) / 2;
        double *dout = nullptr;
        CB_TRY(dbuf(c, "stage_shc", 2 * Ts, &dout));
        CB_TRY(sha_grid(c, pnt, din ? nullptr : f, din, nmax, shcs->mu,
                        shcs->r, shcs->nmax, nullptr, nullptr, dout,
                        dout + Ts));
        CB_TRY(stage_d2h(c, const_cast<double *>(pc), dout, Ts * 8));
        CB_TRY(stage_d2h(c, const_cast<double *>(ps), dout + Ts, Ts * 8));
        return Status{};
    }
    return sha_grid(c, pnt, din ? nullptr : f, din, nmax, shcs->mu, shcs->r,
                    shcs->nmax, shcs->c, shcs->s, nullptr, nullptr);
}

Status sha_point_dev(const charm_point *pnt, const double *d_f,
                     unsigned long nmax, double mu, double r,
                     unsigned long shc_nmax, double *d_c, double *d_s)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    CB_TRY(init(g_ctx));
    return sha_grid(g_ctx, pnt, nullptr, d_f, nmax, mu, r, shc_nmax, nullptr,
                    nullptr, d_c, d_s);
}

Status shs_cell(const charm_cell *cell, const charm_shc *shcs,
                unsigned long nmax, double *f)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    Context &c = g_ctx;
    CB_TRY(init(c));
    CoefIn in;
    in.nmax = shcs->nmax;
    in.mu = shcs->mu;
    in.r = shcs->r;
    in.hc = shcs->c;
    in.hs = shcs->s;
    const bool sctr = cell->type == CHARM_CRD_CELL_SCATTERED;
    // pageable host arrays through the ring, as shs_point
    const double *pc = pageable_tri(shcs->c, shcs->nmax);
    const double *ps = pageable_tri(shcs->s, shcs->nmax);
    if (pc && ps)
    {
        const size_t Ts = (size_t)(shcs->nmax + 1) * (shcs->nmax + 2) / 2;
        double *raw = nullptr;
        CB_TRY(dbuf(c, "stage_shc", 2 * Ts, &raw));
        CB_TRY(stage_h2d(c, raw, pc, Ts * 8));
        CB_TRY(stage_h2d(c, raw + Ts, ps, Ts * 8));
        in.hc = in.hs = nullptr;
        in.dc = raw;
        in.ds = raw + Ts;
    }
    if (cell->ncell > 0 && is_pageable(f))
    {
        double *dout = nullptr;
        CB_TRY(dbuf(c, "stage_out", cell->ncell, &dout));
        CB_TRY(sctr ? shs_cell_sctr(c, cell, in, nmax, nullptr, dout)
                    : shs_cell_grid(c, cell, in, nmax, nullptr, dout));
        return stage_d2h(c, f, dout, cell->ncell * 8);
    }
    if (sctr)
        return shs_cell_sctr(c, cell, in, nmax, f, nullptr);
    return shs_cell_grid(c, cell, in, nmax, f, nullptr);
}

Status shs_cell_dev(const charm_cell *cell, unsigned long shc_nmax,
                    double mu, double r, const double *d_c, const double *d_s,
                    unsigned long nmax, double *d_f)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    CB_TRY(init(g_ctx));
    CoefIn in;
    in.nmax = shc_nmax;
    in.mu = mu;
    in.r = r;
    in.dc = d_c;
    in.ds = d_s;
    if (cell->type == CHARM_CRD_CELL_SCATTERED)
        return shs_cell_sctr(g_ctx, cell, in, nmax, nullptr, d_f);
    return shs_cell_grid(g_ctx, cell, in, nmax, nullptr, d_f);
}

Status sha_cell(const charm_cell *cell, const double *f, unsigned long nmax,
                charm_shc *shcs)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    Context &c = g_ctx;
    CB_TRY(init(c));
    // pageable host arrays through the ring, as sha_point
    const double *din = nullptr;
    if (cell->ncell > 0 && is_pageable(f))
    {
        double *d = nullptr;
        CB_TRY(dbuf(c, "stage_in", cell->ncell, &d));
        CB_TRY(stage_h2d(c, d, f, cell->ncell * 8));
        din = d;
    }
    const double *pc = pageable_tri(shcs->c, shcs->nmax);
    const double *ps = pageable_tri(shcs->s, shcs->nmax);
    if (pc && ps)
    {
        const size_t Ts = (size_t)(shcs->nmax + 1) * (shcs->nmax + 2) / 2;
        double *dout = nullptr;
        CB_TRY(dbuf(c, "stage_shc", 2 * Ts, &dout));
        CB_TRY(sha_cell_grid(c, cell, din ? nullptr : f, din, nmax, shcs->mu,
                             shcs->r, shcs->nmax, nullptr, nullptr, dout,
                             dout + Ts));
        CB_TRY(stage_d2h(c, const_cast<double *>(pc), dout, Ts * 8));
        return stage_d2h(c, const_cast<double *>(ps), dout + Ts, Ts * 8);
    }
    return sha_cell_grid(c, cell, din ? nullptr : f, din, nmax, shcs->mu,
                         shcs->r, shcs->nmax, shcs->c, shcs->s, nullptr,
                         nullptr);
}

Status sha_cell_dev(const charm_cell *cell, const double *d_f,
                    unsigned long nmax, double mu, double r,
                    unsigned long shc_nmax, double *d_c, double *d_s)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    CB_TRY(init(g_ctx));
    return sha_cell_grid(g_ctx, cell, nullptr, d_f, nmax, mu, r, shc_nmax,
                         nullptr, nullptr, d_c, d_s);
}

Status shc_read_bin_dev(const char *path, unsigned long nmax,
                        unsigned long shc_nmax, double *d_c, double *d_s,
                        double *mu, double *r, unsigned long *nmax_file)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    CB_TRY(init(g_ctx));
    return shc_read_bin_dev_impl(g_ctx, path, nmax, shc_nmax, d_c, d_s, mu, r,
                                 nmax_file);
}

Status gfm_global(const GfmArgs &g)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    CB_TRY(init(g_ctx));
    return gfm_global_impl(g_ctx, g);
}

Status sha_point_dev_band(const charm_point *pnt, const double *d_f,
                          unsigned long nmax, double mu, double r,
                          unsigned long shc_nmax, int pair0, int pair1,
                          double *d_c, double *d_s)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    CB_TRY(init(g_ctx));
    return sha_grid(g_ctx, pnt, nullptr, d_f, nmax, mu, r, shc_nmax, nullptr,
                    nullptr, d_c, d_s, pair0, pair1 < pair0 ? pair0 : pair1);
}

int grid_pair_rows(const charm_point *pnt, int *row_n, int *row_s, int cap)
{
    Pairs P;
    grid_pairs(pnt, charm_glob_threshold2, true, P);
    const int np = (int)P.row_n.size();
    for (int p = 0; p < np && p < cap; p++)
    {
        if (row_n)
            row_n[p] = P.row_n[p];
        if (row_s)
            row_s[p] = P.row_s[p] < (int)pnt->nlat ? P.row_s[p] : -1;
    }
    return np;
}

Status shs_point_batch_dev(const charm_point *pnt, size_t nsets,
                           const unsigned long *nmax,
                           const unsigned long *shc_nmax, const double *mu,
                           double r, const double *const *d_c,
                           const double *const *d_s, int kgrad,
                           double *const *d_f)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    CB_TRY(init(g_ctx));
    return shs_batch(g_ctx, pnt, nsets, nmax, shc_nmax, mu, r, d_c, d_s,
                     kgrad, d_f);
}

// ---------------------------------------------------------------------------
// Batched synthesis captured into a CUDA graph
// ---------------------------------------------------------------------------
struct BatchGraph
{
    cudaGraphExec_t exec = nullptr;
    std::vector<void *> pins;
    unsigned long long epoch = 0;  // the context's epoch at capture
};

Status batch_graph_create(const charm_point *pnt, size_t nsets,
                          const unsigned long *nmax,
                          const unsigned long *shc_nmax, const double *mu,
                          double r, const double *const *d_c,
                          const double *const *d_s, int kgrad,
                          double *const *d_f, int split, void **out)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    Context &c = g_ctx;
    Status st;
    *out = nullptr;
    CB_TRY(init(c));
    auto run = [&]() {
        return split ? shs_batch_tc(c, pnt, nsets, nmax, shc_nmax, mu, r, d_c,
                                    d_s, d_f, kgrad)
                     : shs_batch(c, pnt, nsets, nmax, shc_nmax, mu, r, d_c,
                                 d_s, kgrad, d_f);
    };
    // a plain call first: checks the arguments, builds every table, plan,
    // buffer and tuned choice the captured call then finds in place
    CB_TRY(run());
    const bool timing = c.timing;
    c.timing = false;
    c.capturing = true;
    c.capture_pins.clear();
    cudaGraph_t g = nullptr;
    Status s2;
    cudaError_t e = cudaStreamBeginCapture(c.stream,
                                           cudaStreamCaptureModeRelaxed);
    if (e == cudaSuccess)
    {
        s2 = run();
        e = cudaStreamEndCapture(c.stream, &g);
    }
    c.capturing = false;
    c.timing = timing;
    std::vector<void *> pins;
    pins.swap(c.capture_pins);
    auto drop = [&]() {
        for (void *p : pins)
            cudaFreeHost(p);
        if (g)
            cudaGraphDestroy(g);
    };
    if (!s2.ok())
    {
        drop();
        return s2;
    }
    if (e != cudaSuccess)
    {
        drop();
        st.code = CHARM_EFUNCARG;
        st.msg = std::string("stream capture failed: ") + cudaGetErrorString(e);
        return st;
    }
    BatchGraph *G = new BatchGraph;
    e = cudaGraphInstantiate(&G->exec, g, 0);
    cudaGraphDestroy(g);
    g = nullptr;
    if (e != cudaSuccess)
    {
        drop();
        delete G;
        st.code = CHARM_EFUNCARG;
        st.msg = std::string("graph instantiation failed: ") +
                 cudaGetErrorString(e);
        return st;
    }
    G->pins.swap(pins);
    G->epoch = c.epoch;
    *out = G;
    return st;
}

Status batch_graph_launch(void *h)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    Context &c = g_ctx;
    Status st;
    BatchGraph *G = static_cast<BatchGraph *>(h);
    if (G->epoch != c.epoch)
    {
        // a call since the capture reallocated or rewrote buffers or
        // tables the graph reads: replaying it would touch freed or other
        // memory
        st.code = CHARM_EFUNCARG;
        st.msg = "the library's cached buffers or tables changed since this "
                 "graph was captured (a call with other sizes ran in "
                 "between); capture the graph again";
        return st;
    }
    CB_CUDA(cudaGraphLaunch(G->exec, c.stream), st);
    c.launches++;
    void *p = nullptr;
    CB_TRY(buf(c, "status", 256, &p));
    return finish(c, static_cast<unsigned *>(p));
}

void batch_graph_free(void *h)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    BatchGraph *G = static_cast<BatchGraph *>(h);
    if (!G)
        return;
    cudaStreamSynchronize(g_ctx.stream);
    if (G->exec)
        cudaGraphExecDestroy(G->exec);
    for (void *p : G->pins)
        cudaFreeHost(p);
    delete G;
}

// The autotuner's choices so far, one line per problem shape.
std::string autotune_report()
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    std::string out;
    for (const auto &kv : g_ctx.tuned)
    {
        const auto &k = kv.first;
        out += "k_shs_grid kgrad=" + std::to_string(std::get<0>(k)) +
               " dr=" + std::to_string(std::get<1>(k)) +
               " dlat=" + std::to_string(std::get<2>(k)) +
               " rr=" + std::to_string(std::get<3>(k)) +
               " nmax=" + std::to_string(std::get<4>(k)) +
               " pairs=" + std::to_string(std::get<5>(k)) +
               " K=" + std::to_string(kv.second.first) + " ms:";
        for (const auto &m : kv.second.second)
        {
            char b[64];
            snprintf(b, sizeof b, " %d:%.4f", m.first, (double)m.second);
            out += b;
        }
        out += "\n";
    }
    return out;
}

Status shs_point_batch_i8_dev(const charm_point *pnt, size_t nsets,
                              const unsigned long *nmax,
                              const unsigned long *shc_nmax, const double *mu,
                              double r, const double *const *d_c,
                              const double *const *d_s, int kgrad,
                              double *const *d_f)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    CB_TRY(init(g_ctx));
    return shs_batch_tc(g_ctx, pnt, nsets, nmax, shc_nmax, mu, r, d_c, d_s,
                        d_f, kgrad);
}

Status shs_point_dev_f32(const charm_point *pnt, unsigned long shc_nmax,
                         double mu, double r, const float *d_c,
                         const float *d_s, unsigned long nmax, float *d_f)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    CB_TRY(init(g_ctx));
    return shs_grid_f32(g_ctx, pnt, shc_nmax, mu, r, d_c, d_s, nmax, d_f);
}

Status sha_point_dev_f32(const charm_point *pnt, const float *d_f,
                         unsigned long nmax, double mu, double r,
                         unsigned long shc_nmax, float *d_c, float *d_s)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    CB_TRY(init(g_ctx));
    return sha_grid_f32(g_ctx, pnt, d_f, nmax, mu, r, shc_nmax, d_c, d_s);
}

bool f32_serves(const charm_point *pnt, unsigned long nmax, double R)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    if (!init(g_ctx).ok())
        return false;
    if (pnt->type == CHARM_CRD_POINT_SCATTERED || pnt->npoint == 0)
        return false;
    const RfftArgs *rf = nullptr;
    Status st = f32_grid_checks(g_ctx, pnt, nmax, R, &rf);
    return st.ok();
}

Status shs_point_f32_host(const charm_point *pnt, unsigned long shc_nmax,
                          double mu, double r, const float *c, const float *s,
                          unsigned long nmax, float *f)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    Context &cx = g_ctx;
    CB_TRY(init(cx));
    Status st;
    const size_t T = (size_t)(shc_nmax + 1) * (shc_nmax + 2) / 2;
    const size_t npt = pnt->nlat * pnt->nlon;
    float *dc = nullptr, *ds = nullptr, *df = nullptr;
    CB_TRY(dbuf(cx, "f32h_c", T, &dc));
    CB_TRY(dbuf(cx, "f32h_s", T, &ds));
    CB_TRY(dbuf(cx, "f32h_f", npt, &df));
    CB_TRY(stage_h2d(cx, dc, c, T * 4));
    CB_TRY(stage_h2d(cx, ds, s, T * 4));
    CB_TRY(shs_grid_f32(cx, pnt, shc_nmax, mu, r, dc, ds, nmax, df));
    CB_TRY(stage_d2h(cx, f, df, npt * 4));
    return st;
}

Status sha_point_f32_host(const charm_point *pnt, const float *f,
                          unsigned long nmax, double mu, double r,
                          unsigned long shc_nmax, float *c, float *s)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    Context &cx = g_ctx;
    CB_TRY(init(cx));
    Status st;
    const size_t T = (size_t)(shc_nmax + 1) * (shc_nmax + 2) / 2;
    const size_t npt = pnt->nlat * pnt->nlon;
    float *dc = nullptr, *ds = nullptr, *df = nullptr;
    CB_TRY(dbuf(cx, "f32h_c", T, &dc));
    CB_TRY(dbuf(cx, "f32h_s", T, &ds));
    CB_TRY(dbuf(cx, "f32h_f", npt, &df));
    CB_TRY(stage_h2d(cx, df, f, npt * 4));
    CB_TRY(sha_grid_f32(cx, pnt, df, nmax, mu, r, shc_nmax, dc, ds));
    CB_TRY(stage_d2h(cx, c, dc, T * 4));
    CB_TRY(stage_d2h(cx, s, ds, T * 4));
    return st;
}

Status shs_point_sctr_adjoint(const charm_point *pnt, const double *g,
                              unsigned long nmax, charm_shc *shcs)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    CB_TRY(init(g_ctx));
    return sctr_adjoint(g_ctx, pnt, g, nullptr, nmax, shcs->mu, shcs->r,
                        shcs->nmax, shcs->c, shcs->s, nullptr, nullptr);
}

Status shs_point_sctr_adjoint_dev(const charm_point *pnt, const double *d_g,
                                  unsigned long nmax, double mu, double r,
                                  unsigned long shc_nmax, double *d_c,
                                  double *d_s)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    CB_TRY(init(g_ctx));
    return sctr_adjoint(g_ctx, pnt, nullptr, d_g, nmax, mu, r, shc_nmax,
                        nullptr, nullptr, d_c, d_s);
}

Status sha_point_dev_static(const charm_point *pnt, const double *d_f,
                            unsigned long nmax, double mu, double r,
                            unsigned long shc_nmax, double *d_c, double *d_s)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    CB_TRY(init(g_ctx));
    return sha_point_dev_static_impl(g_ctx, pnt, d_f, nmax, mu, r, shc_nmax,
                                     d_c, d_s);
}

Status quad_nodes(int type, unsigned long nmax, double *lat, double *w)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    Context &c = g_ctx;
    CB_TRY(init(c));
    Status st;
    size_t nlat = type == CHARM_CRD_POINT_GRID_GL ? nmax + 1 : 2 * (nmax + 1);
    const auto key = std::make_pair(type, nmax);
    auto hit = c.nodes.find(key);
    if (hit != c.nodes.end())
    {
        std::memcpy(lat, hit->second.data(), nlat * 8);
        std::memcpy(w, hit->second.data() + nlat, nlat * 8);
        return st;
    }
    double *d = nullptr;
    CB_TRY(dbuf(c, "crd", 2 * nlat, &d));
    CB_CUDA(cudaMemsetAsync(d, 0, 2 * nlat * 8, c.stream), st);
    unsigned *d_status;
    unsigned long long *d_counter;
    CB_TRY(status_words(c, &d_status, &d_counter));
    {
        Scope sc(c, TIMER_PREP);
        if (type == CHARM_CRD_POINT_GRID_GL)
            CB_CUDA(launch_gl_nodes(nmax, d, d + nlat, d_status, c.stream), st);
        else
            CB_CUDA(launch_dh_nodes(nmax, d, d + nlat, c.stream), st);
    }
    CB_CUDA(cudaMemcpyAsync(lat, d, nlat * 8, cudaMemcpyDeviceToHost, c.stream),
            st);
    CB_CUDA(cudaMemcpyAsync(w, d + nlat, nlat * 8, cudaMemcpyDeviceToHost,
                            c.stream), st);
    st = finish(c, d_status);
    if (!st.ok() && type == CHARM_CRD_POINT_GRID_GL)
        st.msg = "Error in computing latitudes of the Gauss--Legendre grid.  "
                 "Either the maximum number of iterations was exceeded or at "
                 "least one latitude was detected to be not a real number.";
    if (st.ok())
    {
        // keep the eight most recent grids
        if (c.nodes_order.size() >= 8)
        {
            c.nodes.erase(c.nodes_order.front());
            c.nodes_order.erase(c.nodes_order.begin());
        }
        std::vector<double> v(2 * nlat);
        std::memcpy(v.data(), lat, nlat * 8);
        std::memcpy(v.data() + nlat, w, nlat * 8);
        c.nodes.emplace(key, std::move(v));
        c.nodes_order.push_back(key);
    }
    return st;
}

Status fp64_peak(double *tflops)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    Context &c = g_ctx;
    CB_TRY(init(c));
    Status st;
    double *sink = nullptr;
    CB_TRY(dbuf(c, "probe", 1024, &sink));
    const int threads = 256, blocks = c.num_sms * 8;
    const long long iters = 1 << 16;
    cudaEvent_t a = ev_get(c), b = ev_get(c);
    CB_CUDA(launch_fp64_probe(iters / 8, blocks, threads, sink, c.stream), st);
    CB_CUDA(cudaEventRecord(a, c.stream), st);
    CB_CUDA(launch_fp64_probe(iters, blocks, threads, sink, c.stream), st);
    CB_CUDA(cudaEventRecord(b, c.stream), st);
    CB_CUDA(cudaStreamSynchronize(c.stream), st);
    float ms = 0.f;
    CB_CUDA(cudaEventElapsedTime(&ms, a, b), st);
    c.ev_pool.push_back(a);
    c.ev_pool.push_back(b);
    double flops = 2.0 * 8.0 * (double)iters * threads * (double)blocks;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return st;
}

void *stream_handle()
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    if (!init(g_ctx).ok())
        return nullptr;
    return (void *)g_ctx.stream;
}

void set_timing(bool on)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    g_ctx.timing = on;
    for (int i = 0; i < TIMER_COUNT; i++)
    {
        g_ctx.timer_ms[i] = 0.0;
        g_ctx.timer_n[i] = 0;
    }
    g_ctx.launches = 0;
    g_ctx.fft_execs = 0;
}

void read_timing(double *ms, unsigned long long *n, unsigned long long *kern,
                 unsigned long long *ffts)
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    for (int i = 0; i < TIMER_COUNT; i++)
    {
        if (ms)
            ms[i] = g_ctx.timer_ms[i];
        if (n)
            n[i] = g_ctx.timer_n[i];
    }
    if (kern)
        *kern = g_ctx.launches;
    if (ffts)
        *ffts = g_ctx.fft_execs;
}

void shutdown()
{
    std::lock_guard<std::recursive_mutex> lock(g_ctx.mtx);
    Context &c = g_ctx;
    if (!c.ready)
        return;
    cudaStreamSynchronize(c.stream);
    for (auto &kv : c.rfft_mem)
        cudaFree(kv.second);
    c.rfft_mem.clear();
    c.rffts.clear();
    for (auto &kv : c.bufs)
        if (kv.second.p)
            cudaFree(kv.second.p);
    c.bufs.clear();
    if (c.pinned)
        cudaFreeHost(c.pinned);
    c.pinned = nullptr;
    c.pinned_bytes = 0;
    if (c.h_status)
        cudaFreeHost(c.h_status);
    c.h_status = nullptr;
    for (int b = 0; b < RING_N; b++)
    {
        if (c.ring[b])
            cudaFreeHost(c.ring[b]);
        c.ring[b] = nullptr;
        if (c.ring_ev[b])
            cudaEventDestroy(c.ring_ev[b]);
        c.ring_ev[b] = nullptr;
    }
    for (int k = 0; k < TAB_SLOTS; k++)
        c.tab_nmax[k] = -1;
    c.nodes.clear();
    c.nodes_order.clear();
    c.ready = false;
}

} // namespace cb
