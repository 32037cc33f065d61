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
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/polymul.h"
#include "pm_internal.h"

namespace pm {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(4) << 20;

static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocScratchBytes / sizeof(uint32_t)];

std::mutex g_scratch_mutex;
struct ScratchAddress {
    unsigned long long context = 0;  // id of the CUDA context the address belongs to
    void* address = nullptr;
};
ScratchAddress g_scratch_address[256];

using CtxGetCurrent = CUresult (*)(CUcontext*);
using CtxGetId = CUresult (*)(CUcontext, unsigned long long*);

// Id of the current CUDA context (unique for the life of the process), or 0 if
// there is none yet or the driver cannot say.
unsigned long long current_context_id() {
    static CtxGetCurrent get_current = nullptr;
    static CtxGetId get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<CtxGetCurrent>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetId>(p);
        looked_up = true;
    }
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

// Device address of the array in the current context of `device` (the current
// device).  The host-side symbol g_noalloc_scratch is only a handle for the
// runtime; a kernel given its host address would fault or touch the wrong
// memory.  The address is looked up on the first call in each context and
// kept for that context: after cudaDeviceReset the runtime makes a new
// context, whose module (and array) has a new address, so the lookup runs
// again instead of handing out the old one.
void* scratch_address(int device) {
    if (device < 0 || device >= 256) throw Failure(PM_ERR_INVALID, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    ScratchAddress& slot = g_scratch_address[device];
    const unsigned long long context = current_context_id();
    if (slot.address && context != 0 && context == slot.context) return slot.address;
    void* p = nullptr;
    cuda_check(cudaGetSymbolAddress(&p, g_noalloc_scratch), "look up the built-in scratch array");
    // the lookup made sure a context exists: key the address by it
    slot.context = current_context_id();
    slot.address = slot.context ? p : nullptr;  // no context id: look it up again on every call
    return p;
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
        pm::require_plan_device(s);
        pm::check_device_pointers(s, a, b, c, nullptr);
        pm::launch_product(s, a, b, c, pm::scratch_address(s.device), reinterpret_cast<cudaStream_t>(stream));
        return PM_OK;
    } catch (const pm::Failure& f) {
        return pm::fail(f.status, f.what());
    } catch (const std::exception& e) {
        return pm::fail(PM_ERR_INVALID, e.what());
    }
}
