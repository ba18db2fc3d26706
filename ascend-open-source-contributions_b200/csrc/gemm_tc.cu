// gemm_tc.cu -- tensor-core (tcgen05) forms of the three real products.
#include "cg3m_internal.h"

namespace cg3m {

cudaError_t launch_gemm_tc(cudaStream_t, const Problem&, const Plan&, void*, int*)
{
    return cudaErrorNotSupported;
}

}  // namespace cg3m
