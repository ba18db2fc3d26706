// noalloc.cu -- cg3mCgemm3mNoAlloc: the FP32 drop-in product with its scratch
// held in a fixed device array instead of an allocated workspace.
//
// Who needs this: code that is not allowed to call cudaMalloc / cudaFree at
// the point where it multiplies -- for example a framework whose caching
// allocator owns (and has already reserved) the device heap, or a latency-
// critical loop where an allocation would synchronize the device.  The normal
// entry points allocate a status word and grow a workspace on first use; this
// one never allocates.  Its scratch is the file-scope array below: a fixed
// 32 MiB (the size of the default workspace the reference creates per handle)
// that every GPU loading this library keeps for the life of the process.
//
// The array's host-side name is only a stand-in for the symbol, not a device
// address, so the device address is looked up once per device with
// cudaGetSymbolAddress (with that device current) and cached.  That lookup
// happens inside the first call made on each device.
//
// The first 256 bytes of the array hold the status word the kernels set when
// a bounded wait gives up.  The word is sticky: calls only add bits to it, and
// cg3mGetDeviceStatus(NULL, ...) reads and clears it (the call itself returns
// before its kernels run, so it cannot report them).
#include <cstdio>
#include <cstdlib>
#include <mutex>

#include "cg3m_internal.h"

namespace {

constexpr size_t kScratchBytes = size_t(32) << 20;
constexpr size_t kStatusBytes = 256;  // bounded-wait status word (sticky) and a probe slot
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {};
int g_sm_count[kMaxDevices] = {};

// Once per device, with that device current: resolve the array's device
// address and the SM count the planner needs.
cg3mStatus_t setup_device(int dev, void** addr, int* sms)
{
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (g_scratch_addr[dev] == nullptr) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || p == nullptr) {
            return CG3M_STATUS_INTERNAL_ERROR;
        }
        int count = 0;
        if (cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || count <= 0) {
            return CG3M_STATUS_INTERNAL_ERROR;
        }
        g_sm_count[dev] = count;
        g_scratch_addr[dev] = p;
    }
    *addr = g_scratch_addr[dev];
    *sms = g_sm_count[dev];
    return CG3M_STATUS_SUCCESS;
}

}  // namespace

extern "C" cg3mStatus_t cg3mCgemm3mNoAlloc(void* stream, cg3mOperation_t transa, cg3mOperation_t transb, int m,
                                           int n, int k, const cg3mComplex* alpha, const cg3mComplex* A, int lda,
                                           const cg3mComplex* B, int ldb, const cg3mComplex* beta, cg3mComplex* C,
                                           int ldc)
{
    using namespace cg3m;
    int action = 0;
    const cg3mStatus_t st = validate(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, false, &action);
    if (st != CG3M_STATUS_SUCCESS || action == 0) {
        return st;
    }
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        return CG3M_STATUS_INTERNAL_ERROR;
    }
    // The scratch address is per device: a stream of another device would get
    // this device's array, so such a stream is refused.
    int stream_dev = dev;
    if (cudaStreamGetDevice(s, &stream_dev) != cudaSuccess) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    if (stream_dev != dev) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    void* base = nullptr;
    int sms = 0;
    const cg3mStatus_t su = setup_device(dev, &base, &sms);
    if (su != CG3M_STATUS_SUCCESS) {
        return su;
    }
    if (action == 1) {
        return launch_beta_scale(s, m, n, beta->real, beta->imag, C, ldc) == cudaSuccess
                   ? CG3M_STATUS_SUCCESS
                   : CG3M_STATUS_EXECUTION_FAILED;
    }
    Problem p{transa, transb, m, n, k, alpha->real, alpha->imag, beta->real, beta->imag, A, lda, B, ldb, C, ldc};
    Plan plan;
    const cg3mOptions opts{};
    if (!make_plan(p, opts, sms, &plan)) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    if (plan.total > kScratchBytes - kStatusBytes) {
        if (std::getenv("CG3M_LOG") != nullptr) {
            std::fprintf(stderr, "cg3mCgemm3mNoAlloc: needs %zu scratch bytes, the fixed array holds %zu\n",
                         plan.total, kScratchBytes - kStatusBytes);
        }
        return CG3M_STATUS_INVALID_VALUE;
    }
    // Kernels only OR bits into the status word (zero when the library is
    // loaded, cleared when it is read); the planes and partials are fully
    // rewritten before they are read, so nothing else needs clearing.
    int* status = static_cast<int*>(base);
    void* ws = static_cast<unsigned char*>(base) + kStatusBytes;
    const cudaError_t err = enqueue(s, p, plan, ws, status, nullptr);
    return err == cudaSuccess ? CG3M_STATUS_SUCCESS : CG3M_STATUS_EXECUTION_FAILED;
}

namespace cg3m {

// The status word of the allocation-free entry point on the current device
// (its address resolved if no call has done so yet).
cg3mStatus_t noalloc_status_word(int** word)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        return CG3M_STATUS_INTERNAL_ERROR;
    }
    void* base = nullptr;
    int sms = 0;
    const cg3mStatus_t st = setup_device(dev, &base, &sms);
    if (st == CG3M_STATUS_SUCCESS) {
        *word = static_cast<int*>(base);
    }
    return st;
}

}  // namespace cg3m
