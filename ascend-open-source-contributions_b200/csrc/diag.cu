// diag.cu -- the bounded-wait probe behind cg3mDiagBoundedWait.
//
// Every pipeline wait in this library gives up after a wall-time limit, sets
// kStatusTimeout in the call's status word and lets its kernel return, so a
// stalled copy or MMA can never hold the GPU.  The production kernels only
// reach that branch when something is already wrong, so this probe exercises
// it on purpose without any fault: one thread initialises an mbarrier that
// nothing ever arrives on, waits on it through the same mbar_wait the kernels
// use, with a short caller-given limit, and records whether the wait gave up.
#include "cg3m_internal.h"
#include "ptx.cuh"

namespace cg3m {
namespace {

__global__ void wait_probe_kernel(int* status, unsigned long long limit_ns, int* gave_up)
{
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // Phase 0 of a fresh barrier with no arrivals never completes.
        const bool completed = mbar_wait(&bar, 0, status, limit_ns);
        *gave_up = completed ? 0 : 1;
    }
}

}  // namespace

cudaError_t launch_wait_probe(cudaStream_t s, int* status, unsigned long long limit_ns, int* gave_up)
{
    wait_probe_kernel<<<1, 32, 0, s>>>(status, limit_ns, gave_up);
    return cudaGetLastError();
}

}  // namespace cg3m
