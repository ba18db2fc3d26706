// rounding.cu -- rounding-correction pass.
#include "cg3m_internal.h"

namespace cg3m {

cudaError_t launch_rounding(cudaStream_t, const Problem&, const Plan&, void*, int*, int*)
{
    return cudaErrorNotSupported;
}

}  // namespace cg3m
