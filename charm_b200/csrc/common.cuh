// Device-side building blocks shared by the sm_100a kernels of charm_b200:
// triangle indexing, 1-D bulk (TMA) copies into shared memory completed on
// an mbarrier with a bounded wait, and the warp "transpose-reduce" used by
// the analysis kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.h"

namespace cb
{


// Index of C_nm in an order-major triangle of maximum degree nmax:
// column m starts at m (2 nmax + 3 - m) / 2 (CHarm's layout,
// src/shc/shc_init_chunk.c:126-145).
__host__ __device__ __forceinline__ long long tri_col0(long long nmax,
                                                       long long m)
{
    return (m * (2 * nmax + 3 - m)) / 2;
}

__host__ __device__ __forceinline__ long long tri_size(long long nmax)
{
    return (nmax + 1) * (nmax + 2) / 2;
}

// ---------------------------------------------------------------------------
// 1-D bulk copies global -> shared completed on an mbarrier (sm_90+ TMA,
// non-tensor form).  Addresses and sizes must be multiples of 16 bytes.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (bulk copy) accesses.
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar,
                                                      unsigned bytes)
{
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
            smem_u32(bar)),
        "r"(bytes)
        : "memory");
}

__device__ __forceinline__ void bulk_g2s(void *dst_smem, const void *src_gmem,
                                         unsigned bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1], %2, [%3];" ::"r"(smem_u32(dst_smem)),
        "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase with the given parity to complete.  Gives up after
// "limit" polls (each poll may itself suspend briefly), records the failure
// in *status and returns false; the caller then stops its work.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar,
                                                  unsigned parity,
                                                  unsigned *status)
{
    const unsigned limit = 1u << 22;
    for (unsigned it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity))
            return true;
    atomicOr(status, DEV_ERR_WAIT_TIMEOUT);
    return false;
}

// ---------------------------------------------------------------------------
// Exact scaling by powers of two and binary exponents (normal numbers)
// ---------------------------------------------------------------------------
__device__ __forceinline__ int expo_of(double x)
{
    // floor(log2 |x|) for normal x; callers never pass zero
    int hi = __double2hiint(x);
    return ((hi >> 20) & 0x7ff) - 1023;
}

// ---------------------------------------------------------------------------
// Warp transpose-reduce: 32 consecutive per-lane values v_j (j = 0..31) are
// summed over the warp so that lane l ends with the total of v_l, using 31
// shuffles per 32 values.  Level k combines pairs of partial results with
// lanes l ^ 2^k.  "keep" is the value this lane retains (lower index if
// bit k of the lane is clear), the other one is sent to the partner.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double tr_combine(double lo, double hi, int off,
                                             unsigned lane)
{
    const bool upper = (lane & off) != 0;
    double keep = upper ? hi : lo;
    double send = upper ? lo : hi;
    return keep + __shfl_xor_sync(0xffffffffu, send, off);
}

} // namespace cb
