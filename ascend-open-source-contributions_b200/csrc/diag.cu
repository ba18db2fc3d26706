// diag.cu -- the bounded-wait probe behind cg3mDiagBoundedWait.
//
// Every pipeline wait in this library gives up after a wall-time limit, sets
// kStatusTimeout in the call's status word and lets its kernel return, so a
// stalled copy or MMA can never hold the GPU.  The production kernels only
// reach that branch when something is already wrong, so this probe exercises
// it on purpose without any fault: one thread initialises an mbarrier that
// nothing ever arrives on, waits on it through the same mbar_wait the kernels
// use, with a short caller-given limit, and records whether the wait gave up.
#include <cstdlib>

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

// Set when a check finds a damaged guard band; read and cleared by
// cg3mDiagGuardStatus.
__device__ unsigned int g_guard_damage;

struct GuardList {
    unsigned long long off[Plan::kMaxGuards];
};

// One block per band: every 32-bit word of it must still hold the pattern.
__global__ void guard_check_kernel(const unsigned char* ws, GuardList list)
{
    const uint32_t* band = reinterpret_cast<const uint32_t*>(ws + list.off[blockIdx.x]);
    const uint32_t want = 0x01010101u * kGuardByte;
    bool bad = false;
    for (size_t i = threadIdx.x; i < kGuardBytes / 4; i += blockDim.x) {
        bad |= band[i] != want;
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) {
        atomicOr(&g_guard_damage, 1u);
    }
}

}  // namespace

bool guard_bands_on()
{
    static const bool on = std::getenv("CG3M_GUARD_BANDS") != nullptr;
    return on;
}

cudaError_t fill_guards(cudaStream_t s, void* ws, const size_t* offs, int count)
{
    for (int i = 0; i < count; ++i) {
        const cudaError_t e = cudaMemsetAsync(static_cast<unsigned char*>(ws) + offs[i], kGuardByte, kGuardBytes, s);
        if (e != cudaSuccess) {
            return e;
        }
    }
    return cudaSuccess;
}

cudaError_t check_guards(cudaStream_t s, const void* ws, const size_t* offs, int count)
{
    if (count <= 0) {
        return cudaSuccess;
    }
    GuardList list{};
    for (int i = 0; i < count && i < Plan::kMaxGuards; ++i) {
        list.off[i] = offs[i];
    }
    guard_check_kernel<<<count, 256, 0, s>>>(static_cast<const unsigned char*>(ws), list);
    return cudaGetLastError();
}

cudaError_t read_guard_damage(int* damaged)
{
    unsigned int v = 0;
    const unsigned int zero = 0;
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) {
        e = cudaMemcpyFromSymbol(&v, g_guard_damage, sizeof(v));
    }
    if (e == cudaSuccess) {
        e = cudaMemcpyToSymbol(g_guard_damage, &zero, sizeof(zero));
    }
    *damaged = (int)v;
    return e;
}

cudaError_t launch_wait_probe(cudaStream_t s, int* status, unsigned long long limit_ns, int* gave_up)
{
    wait_probe_kernel<<<1, 32, 0, s>>>(status, limit_ns, gave_up);
    return cudaGetLastError();
}

}  // namespace cg3m
