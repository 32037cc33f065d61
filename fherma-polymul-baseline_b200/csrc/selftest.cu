// Diagnostic: exercises the bounded mbarrier wait every device-side wait of the
// library uses (TMA and bulk-copy completions, MMA commits, the producer and
// worker hand-offs), on a barrier nothing ever arrives at.  The kernel must give
// up after the requested limit, report it, and leave the context usable.
#include <cuda_runtime.h>

#include "../../include/polymul.h"
#include "pm_internal.h"
#include "tc_ptx.cuh"

namespace pm {
namespace {

// out[0] = 1 if the wait gave up, out[1..2] = nanoseconds waited (lo, hi)
__global__ void selftest_wait_kernel(uint64_t limit_ns, uint32_t* out) {
    __shared__ uint64_t bar;
    if (threadIdx.x != 0) return;
    tc::mbar_init(&bar, 1);  // expects one arrival that never comes
    tc::fence_smem_async();
    const uint64_t t0 = tc::global_ns();
    const bool done = tc::mbar_wait(&bar, 0, limit_ns);
    const uint64_t waited = tc::global_ns() - t0;
    out[0] = done ? 0u : 1u;
    out[1] = uint32_t(waited);
    out[2] = uint32_t(waited >> 32);
}

}  // namespace
}  // namespace pm

extern "C" int pm_selftest_bounded_wait(uint32_t limit_us, uint32_t* timed_out, uint64_t* waited_ns) {
    if (!timed_out || !waited_ns) return pm::fail(PM_ERR_INVALID, "NULL argument");
    if (limit_us == 0 || limit_us > 2000000) return pm::fail(PM_ERR_INVALID, "limit_us must be in [1, 2000000]");
    uint32_t* d = nullptr;
    uint32_t h[3] = {0, 0, 0};
    cudaError_t e = cudaMalloc(&d, sizeof h);
    if (e != cudaSuccess) return pm::fail(PM_ERR_CUDA, std::string("selftest buffer: ") + cudaGetErrorString(e));
    pm::selftest_wait_kernel<<<1, 32>>>(uint64_t(limit_us) * 1000u, d);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof h, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return pm::fail(PM_ERR_CUDA, std::string("selftest: ") + cudaGetErrorString(e));
    pm::count_launches(1);
    *timed_out = h[0];
    *waited_ns = (uint64_t(h[2]) << 32) | h[1];
    return PM_OK;
}
