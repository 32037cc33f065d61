// pm_multiply_noalloc: one product whose scratch memory is a fixed array
// compiled into the library, so the call itself allocates nothing.
//
// Who needs it: code that may not call cudaMalloc (or any allocator) at the
// moment it multiplies -- for example a host callback or a real-time loop
// that must not block on the driver's allocator, or a process whose device
// memory is owned by another framework's fixed pool.  pm_multiply needs a
// workspace of pm_plan_info.workspace_bytes that the caller (or the plan)
// must have allocated; this entry point uses the built-in array instead.
//
// Limits and sharing:
//  - the array holds kNoAllocScratchBytes (4 MiB); a plan whose residue
//    planes need more (n > 8192 for an 868-bit q) is refused;
//  - every call on a device uses the same array, so calls whose kernels
//    overlap on that device (different streams, or host threads without
//    ordering) race and corrupt each other's results -- serialize them;
//  - the array keeps the previous call's contents; nothing in it has to start
//    at zero (every residue plane is written in full before it is read);
//  - each GPU that loads the library holds the array until the process exits.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/polymul.h"
#include "pm_internal.h"

namespace pm {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(4) << 20;

static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocScratchBytes / sizeof(uint32_t)];

std::mutex g_scratch_mutex;
void* g_scratch_address[256] = {};

// Device address of the array on the current device.  The host-side symbol
// g_noalloc_scratch is only a handle for the runtime; a kernel given its host
// address would fault or touch the wrong memory.  Looked up once per device
// (the first call on each device does it).
void* scratch_address(int device) {
    if (device < 0 || device >= 256) throw Failure(PM_ERR_INVALID, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_address[device]) {
        void* p = nullptr;
        cuda_check(cudaGetSymbolAddress(&p, g_noalloc_scratch), "look up the built-in scratch array");
        g_scratch_address[device] = p;
    }
    return g_scratch_address[device];
}

}  // namespace
}  // namespace pm

extern "C" int pm_multiply_noalloc(const pm_plan* plan, const uint64_t* a, const uint64_t* b, uint64_t* c,
                                   pm_stream stream) {
    if (!plan || !a || !b || !c) return pm::fail(PM_ERR_INVALID, "NULL argument");
    try {
        const pm::PlanCore& s = plan->core;
        if (s.workspace_bytes > pm::kNoAllocScratchBytes)
            return pm::fail(PM_ERR_UNSUPPORTED,
                            "pm_multiply_noalloc: this plan needs " + std::to_string(s.workspace_bytes) +
                                " bytes of scratch, above the built-in 4 MiB (n <= 8192 for an 868-bit q); "
                                "use pm_multiply with a workspace instead");
        int device = -1;
        pm::cuda_check(cudaGetDevice(&device), "cudaGetDevice");
        if (device != s.device) return pm::fail(PM_ERR_INVALID, "the plan belongs to another device");
        pm::check_device_pointers(s, a, b, c, nullptr);
        pm::launch_product(s, a, b, c, pm::scratch_address(device), reinterpret_cast<cudaStream_t>(stream));
        return PM_OK;
    } catch (const pm::Failure& f) {
        return pm::fail(f.status, f.what());
    } catch (const std::exception& e) {
        return pm::fail(PM_ERR_INVALID, e.what());
    }
}
