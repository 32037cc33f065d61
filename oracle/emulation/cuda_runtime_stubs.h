// Test infrastructure only: host-side CUDA runtime names that the reference's
// rns backend uses and its CPU emulation header (tests/cuda_emulation.h) does
// not define.  On the CPU there is one synchronous "device": streams and
// events are empty handles, asynchronous copies are plain memcpy.
#pragma once

#include <cstring>

struct CUevent_stub;
struct CUgraph_stub;
struct CUgraphExec_stub;
using cudaEvent_t = CUevent_stub*;
using cudaGraph_t = CUgraph_stub*;
using cudaGraphExec_t = CUgraphExec_stub*;
inline int cudaStreamSynchronize(cudaStream_t) { return 0; }
inline int cudaStreamDestroy(cudaStream_t) { return 0; }
inline int cudaEventDestroy(cudaEvent_t) { return 0; }
inline int cudaEventSynchronize(cudaEvent_t) { return 0; }
inline int cudaGraphExecDestroy(cudaGraphExec_t) { return 0; }
inline int cudaMemcpyAsync(void* dst, const void* src, size_t n, int, cudaStream_t = nullptr) {
    std::memcpy(dst, src, n);
    return 0;
}
// no GPU to pin the host threads near: the reference's pin_near_gpu() returns
inline int cudaDeviceGetPCIBusId(char*, int, int) { return 1; }
