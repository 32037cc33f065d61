// The quartic factorization of the reference's best backend (quartic/host_setup.h,
// quartic/solve.cu), for q = B^4 - delta.
#include <cuda_runtime.h>

#include "../../include/polymul.h"
#include "pm_internal.h"

namespace pm {

QuarticTables::~QuarticTables() {
    cudaFree(d_pc);
    cudaFree(d_tw_fwd);
    cudaFree(d_tw_inv);
    cudaFree(d_conv);
    cudaFree(d_crt);
    cudaFree(d_mix);
    cudaFree(d_ktab);
}

}  // namespace pm
