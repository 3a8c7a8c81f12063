// Fixed device scratch of the allocation-free analysis entry point
// charm_b200_sha_point_dev_static (engine.cpp, sha_point_dev_static).
//
// Its callers cannot allocate device memory during the call: their device
// memory is owned by another allocator (a framework's caching pool that
// holds the free memory), or they run the analysis inside a loop that must
// not synchronise the device, which cudaMalloc and cudaFree do.  Every
// temporary of that path - recurrence tables, transform tables, latitude
// geometry, row spectra, the per-group partial sums of k_sha_grid and the
// status / work-counter words - is carved from this one array.
//
// The array is a module global: it is zero when the module loads and is
// never freed.  Only the status word and the work counter must be zero at
// the start of each analysis kernel; the driver clears them before every
// launch.  Calls whose kernels overlap on the GPU race on this memory: the
// driver serialises its calls on the library stream and returns only after
// that stream is idle.
#include "kernels.h"

namespace cb
{

static __device__ __align__(256) unsigned char g_sha_static_scratch
    [STATIC_SCRATCH_BYTES];

cudaError_t static_scratch_address(void **ptr)
{
    return cudaGetSymbolAddress(ptr, g_sha_static_scratch);
}

} // namespace cb
