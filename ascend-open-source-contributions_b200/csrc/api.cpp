// api.cpp -- the C ABI (include/cg3m.h, include/cg3m_aclblas.h).
//
// Reference: aclblasCgemm3m (blas/gemm/arch35/cgemm3m_host.cpp:17-23) ->
// LaunchComplexGemm (cgemm_host.cpp:701-730) -> LaunchCgemmKernel (:553-587)
// -> HandleCgemmAlphaZero (:636-663) or LaunchGeneralCgemm (:503-551); handle
// API cann_ops_blas.h:31-110.  Every launch goes to the handle's stream and
// nothing here synchronizes except Destroy, GetDeviceStatus and the
// host-buffer entry point (which returns with C on the host).
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/cg3m_aclblas.h"
#include "cg3m_internal.h"

using namespace cg3m;

namespace {

constexpr int kVersion = 10000;  // 1.0.0

bool log_enabled()
{
    static const bool on = std::getenv("CG3M_LOG") != nullptr;
    return on;
}

void log_call(const char* what, const Plan& plan, const Problem& p)
{
    if (!log_enabled()) {
        return;
    }
    std::fprintf(stderr,
                 "{\"cg3m\":\"%s\",\"m\":%d,\"n\":%d,\"k\":%d,\"transa\":%d,\"transb\":%d,\"form\":%d,"
                 "\"tile\":[%d,%d],\"parts\":%d,\"span\":%d,\"rounding\":%d,\"workspace\":%zu}\n",
                 what, p.m, p.n, p.k, p.transa, p.transb, plan.form, plan.tile_m, plan.tile_n, plan.parts, plan.span,
                 plan.rounding ? 1 : 0, plan.total);
}

// Allocations still to fail on purpose (cg3mDiagFailAllocations).
std::atomic<int> g_fail_allocs{0};

cg3mStatus_t bind_device(cg3mContext* h)
{
    if (h->device >= 0) {
        return CG3M_STATUS_SUCCESS;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        return CG3M_STATUS_INTERNAL_ERROR;
    }
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) {
        return CG3M_STATUS_INTERNAL_ERROR;
    }
    int* status = nullptr;
    if (device_malloc(reinterpret_cast<void**>(&status), 64) != cudaSuccess) {
        return CG3M_STATUS_ALLOC_FAILED;
    }
    if (cudaMemset(status, 0, 64) != cudaSuccess) {
        cudaFree(status);
        return CG3M_STATUS_INTERNAL_ERROR;
    }
    void* ws = nullptr;
    if (device_malloc(&ws, kDefaultWorkspaceBytes) != cudaSuccess) {
        cudaFree(status);
        return CG3M_STATUS_ALLOC_FAILED;
    }
    h->device = dev;
    h->sm_count = sms;
    h->status = status;
    h->default_ws = ws;
    h->default_ws_bytes = kDefaultWorkspaceBytes;
    return CG3M_STATUS_SUCCESS;
}

// Effective workspace of at least `bytes` (EnsureDefaultWorkspace /
// GetEffectiveWorkspace in the reference): the borrowed one when large enough,
// else the library's own, grown on demand.
cg3mStatus_t workspace(cg3mContext* h, size_t bytes, void** out)
{
    if (h->user_ws != nullptr && h->user_ws_bytes >= bytes) {
        *out = h->user_ws;
        return CG3M_STATUS_SUCCESS;
    }
    if (h->default_ws_bytes < bytes) {
        // Work already queued may still read the old buffer; cudaFree waits for it.
        if (h->default_ws != nullptr) {
            cudaFree(h->default_ws);
            h->default_ws = nullptr;
            h->default_ws_bytes = 0;
        }
        const size_t grow = align_up(bytes, size_t(2) << 20);
        if (device_malloc(&h->default_ws, grow) != cudaSuccess) {
            h->default_ws = nullptr;
            return CG3M_STATUS_ALLOC_FAILED;
        }
        h->default_ws_bytes = grow;
    }
    *out = h->default_ws;
    return CG3M_STATUS_SUCCESS;
}

// Options of cg3mCgemm's three-product case: the FP32 drop-in arithmetic, no
// rounding pass.
cg3mOptions cgemm_unit_options()
{
    cg3mOptions o{};
    o.form = CG3M_FORM_FP32;
    o.rounding = CG3M_ROUNDING_OFF;
    return o;
}

cg3mStatus_t to_status(cudaError_t e)
{
    if (e == cudaSuccess) {
        return CG3M_STATUS_SUCCESS;
    }
    if (log_enabled()) {
        std::fprintf(stderr, "{\"cg3m\":\"cuda error\",\"code\":%d,\"what\":\"%s\"}\n", (int)e,
                     cudaGetErrorString(e));
    }
    if (e == cudaErrorMemoryAllocation) {
        return CG3M_STATUS_ALLOC_FAILED;
    }
    return CG3M_STATUS_EXECUTION_FAILED;
}

cg3mStatus_t run_one(cg3mContext* h, int transa, int transb, int m, int n, int k, const cg3mComplex* alpha,
                     const cg3mComplex* A, int lda, const cg3mComplex* B, int ldb, const cg3mComplex* beta,
                     cg3mComplex* C, int ldc, const cg3mOptions& opts, bool allow_conj_only, cg3mCallInfo* info)
{
    int action = 0;
    const cg3mStatus_t st =
        validate(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, allow_conj_only, &action);
    if (info != nullptr) {
        std::memset(info, 0, sizeof(*info));
        info->form = opts.form;
    }
    if (st != CG3M_STATUS_SUCCESS || action == 0) {
        return st;
    }
    if (opts.form < CG3M_FORM_FP32 || opts.form > CG3M_FORM_BF16X9 || opts.rounding < CG3M_ROUNDING_AUTO ||
        opts.rounding > CG3M_ROUNDING_OFF || opts.k_partitions < 0) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    const cg3mStatus_t bs = bind_device(h);
    if (bs != CG3M_STATUS_SUCCESS) {
        return bs;
    }
    if (action == 1) {
        if (info != nullptr) {
            info->path = 1;
            info->kernels = 1;
        }
        return to_status(launch_beta_scale(h->stream, m, n, beta->real, beta->imag, C, ldc));
    }
    Problem p{transa, transb, m, n, k, alpha->real, alpha->imag, beta->real, beta->imag, A, lda, B, ldb, C, ldc};
    Plan plan;
    if (!make_plan(p, opts, h->sm_count, &plan)) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    void* ws = nullptr;
    const cg3mStatus_t wst = workspace(h, plan.total, &ws);
    if (wst != CG3M_STATUS_SUCCESS) {
        return wst;
    }
    log_call("cgemm3m", plan, p);
    int kernels = 0;
    const cudaError_t err = enqueue(h->stream, p, plan, ws, h->status, &kernels, h->stage_events,
                                    h->stage_event_count);
    h->round_stats = plan.rounding ? rounding_stats_ptr(plan, ws, p.n) : nullptr;
    if (info != nullptr) {
        info->path = plan.engine == 2 ? 4 : plan.parts > 1 ? 3 : 2;
        info->form = plan.form;
        info->tile_m = plan.tile_m;
        info->tile_n = plan.tile_n;
        info->k_partitions = plan.parts;
        info->k_span = plan.span;
        info->rounding = plan.rounding ? 1 : 0;
        info->kernels = kernels;
        info->workspace_bytes = plan.total;
    }
    return to_status(err);
}

}  // namespace

namespace cg3m {

cudaError_t device_malloc(void** p, size_t bytes)
{
    int pending = g_fail_allocs.load();
    while (pending > 0) {
        if (g_fail_allocs.compare_exchange_weak(pending, pending - 1)) {
            *p = nullptr;
            return cudaErrorMemoryAllocation;
        }
    }
    return cudaMalloc(p, bytes);
}

cudaError_t enqueue(cudaStream_t s, const Problem& p, const Plan& plan, void* ws, int* status, int* kernels,
                    const cudaEvent_t* events, int nevents)
{
    auto record = [&](int idx, cudaStream_t st) {
        if (events != nullptr && idx >= 0 && idx < nevents && events[idx] != nullptr) {
            cudaEventRecord(events[idx], st);
        }
    };
    // Marks for a run of `len` kernels with call indices first, first + 1, ...
    // on stream st: the first one's begin now, and after the i-th (1-based)
    // its end and the next one's begin.
    auto run_marks = [&](int first, int len, cudaStream_t st) {
        record(2 * first, st);
        return [&record, first, len, st](int i) {
            record(2 * (first + i - 1) + 1, st);
            if (i < len) {
                record(2 * (first + i), st);
            }
        };
    };
    if (plan.guards > 0) {
        const cudaError_t e = fill_guards(s, ws, plan.guard_off, plan.guards);
        if (e != cudaSuccess) {
            return e;
        }
    }
    if (plan.engine == 2) {
        auto mark = run_marks(0, 1, s);
        const cudaError_t e = launch_single(s, p, 0, 0, plan.onchip_tile, plan.parts);
        mark(1);
        if (kernels != nullptr) {
            *kernels = 1;
        }
        return e;
    }
    // tensor-core forms in the rounding pass: packed rows with the leading
    // planes and the energies precede the risk-plane GEMM, which selects
    const bool tc_round = plan.rounding && plan.form != CG3M_FORM_FP32;
    const int main_len = 2 + (tc_round ? 1 : 0) + (plan.parts > 1 && !plan.cluster_merge ? 1 : 0);
    const int prep_len = plan.rounding ? rounding_prep_kernels(plan.form) : 0;
    cudaError_t err = cudaSuccess;
    int prep_launched = 0;
    int count = 0;
    {
        auto mark = run_marks(0, main_len, s);
        if (tc_round) {
            // the rest of the planes is packed after the selection
            err = launch_rounding_pack(s, p, plan, ws, [&]() { mark(++count); });
        } else {
            err = launch_pack(s, p, plan, ws);
            mark(++count);
        }
        if (err == cudaSuccess) {
            if (plan.rounding) {
                err = launch_gemm_with_path(s, p, plan, ws, status);
            } else {
                err = plan.form == CG3M_FORM_FP32 ? launch_gemm_fp32(s, p, plan, ws, status)
                                                  : launch_gemm_tc(s, p, plan, ws, status);
            }
            mark(++count);
        }
        if (err == cudaSuccess && plan.parts > 1 && !plan.cluster_merge) {
            err = launch_merge(s, p, plan, ws);
            mark(++count);
        }
    }
    if (err == cudaSuccess && plan.rounding) {
        err = launch_rounding_prep(s, p, plan, ws, &prep_launched, run_marks(count, prep_len, s));
        count += prep_launched;
        if (err == cudaSuccess) {
            int launched = 0;
            err = launch_rounding_finish(s, p, plan, ws, status, &launched, run_marks(count, 64, s));
            count += launched;
        }
    }
    if (err == cudaSuccess && plan.guards > 0) {
        err = check_guards(s, ws, plan.guard_off, plan.guards);
    }
    if (kernels != nullptr) {
        *kernels = count;
    }
    return err;
}

}  // namespace cg3m

extern "C" {

cg3mStatus_t cg3mCreate(cg3mHandle_t* handle)
{
    if (handle == nullptr) {
        return CG3M_STATUS_HANDLE_IS_NULLPTR;
    }
    if (*handle != nullptr) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    cg3mContext* h = new (std::nothrow) cg3mContext();
    if (h == nullptr) {
        return CG3M_STATUS_ALLOC_FAILED;
    }
    *handle = h;
    return CG3M_STATUS_SUCCESS;
}

cg3mStatus_t cg3mDestroy(cg3mHandle_t h)
{
    if (h == nullptr) {
        return CG3M_STATUS_HANDLE_IS_NULLPTR;
    }
    cg3mStatus_t st = CG3M_STATUS_SUCCESS;
    if (h->device >= 0) {
        if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
            st = CG3M_STATUS_EXECUTION_FAILED;
        }
        cudaFree(h->default_ws);
        cudaFree(h->status);
        cudaFree(h->host_arena);
        if (h->h2d != nullptr) {
            cudaStreamDestroy(h->h2d);
        }
        if (h->d2h != nullptr) {
            cudaStreamDestroy(h->d2h);
        }
    }
    delete h;
    return st;
}

cg3mStatus_t cg3mSetStream(cg3mHandle_t h, void* stream)
{
    if (h == nullptr) {
        return CG3M_STATUS_HANDLE_IS_NULLPTR;
    }
    h->stream = static_cast<cudaStream_t>(stream);
    h->user_ws = nullptr;  // back to the default workspace (cann_ops_blas.h:63-71)
    h->user_ws_bytes = 0;
    return CG3M_STATUS_SUCCESS;
}

cg3mStatus_t cg3mGetStream(cg3mHandle_t h, void** stream)
{
    if (h == nullptr) {
        return CG3M_STATUS_HANDLE_IS_NULLPTR;
    }
    if (stream == nullptr) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    *stream = h->stream;
    return CG3M_STATUS_SUCCESS;
}

cg3mStatus_t cg3mSetWorkspace(cg3mHandle_t h, void* ws, size_t bytes)
{
    if (h == nullptr) {
        return CG3M_STATUS_HANDLE_IS_NULLPTR;
    }
    if (ws == nullptr || bytes == 0) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    if (bytes > h->user_ws_bytes) {  // grow-only (cann_ops_blas.h:86-98)
        h->user_ws = ws;
        h->user_ws_bytes = bytes;
    }
    return CG3M_STATUS_SUCCESS;
}

cg3mStatus_t cg3mGetVersion(cg3mHandle_t, int* version)
{
    if (version == nullptr) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    *version = kVersion;
    return CG3M_STATUS_SUCCESS;
}

cg3mStatus_t cg3mCgemm3m(cg3mHandle_t h, cg3mOperation_t transa, cg3mOperation_t transb, int m, int n, int k,
                         const cg3mComplex* alpha, const cg3mComplex* A, int lda, const cg3mComplex* B, int ldb,
                         const cg3mComplex* beta, cg3mComplex* C, int ldc)
{
    if (h == nullptr) {
        return CG3M_STATUS_HANDLE_IS_NULLPTR;
    }
    const cg3mOptions opts{};
    return run_one(h, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, opts, false, nullptr);
}

cg3mStatus_t cg3mCgemm3mEx(cg3mHandle_t h, cg3mOperation_t transa, cg3mOperation_t transb, int m, int n, int k,
                           const cg3mComplex* alpha, const cg3mComplex* A, int lda, const cg3mComplex* B, int ldb,
                           const cg3mComplex* beta, cg3mComplex* C, int ldc, const cg3mOptions* opts,
                           cg3mCallInfo* info)
{
    if (h == nullptr) {
        return CG3M_STATUS_HANDLE_IS_NULLPTR;
    }
    const cg3mOptions o = opts != nullptr ? *opts : cg3mOptions{};
    return run_one(h, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, o, true, info);
}

cg3mStatus_t cg3mCgemm3mStridedBatched(cg3mHandle_t h, cg3mOperation_t transa, cg3mOperation_t transb, int m,
                                       int n, int k, const cg3mComplex* alpha, const cg3mComplex* A, int lda,
                                       int64_t strideA, const cg3mComplex* B, int ldb, int64_t strideB,
                                       const cg3mComplex* beta, cg3mComplex* C, int ldc, int64_t strideC,
                                       int batch_count)
{
    // Statuses of the strided API (blas/gemm/README.md:850-858): enum errors stay INVALID_ENUM.
    if (h == nullptr) {
        return CG3M_STATUS_HANDLE_IS_NULLPTR;
    }
    auto op_ok = [](int op) { return op == CG3M_OP_N || op == CG3M_OP_T || op == CG3M_OP_C; };
    if (!op_ok(transa) || !op_ok(transb)) {
        return CG3M_STATUS_INVALID_ENUM;
    }
    if (batch_count < 0) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    int action = 0;
    // Shape / ld / scalar checks as the single call; an empty batch needs no
    // matrices at all (blas/gemm/README.md:850-851).
    const void* any = reinterpret_cast<const void*>(1);
    const bool empty = batch_count == 0;
    const cg3mStatus_t st = validate(transa, transb, m, n, k, alpha, empty ? any : A, lda, empty ? any : B, ldb, beta,
                                     empty ? any : C, ldc, false, &action);
    if (st != CG3M_STATUS_SUCCESS || action == 0 || batch_count == 0) {
        return st;
    }
    const cg3mStatus_t bs = bind_device(h);
    if (bs != CG3M_STATUS_SUCCESS) {
        return bs;
    }
    if (action == 1) {  // k == 0 or alpha == 0: beta scaling of every batch, in batch order
        for (int i = 0; i < batch_count; ++i) {
            const cudaError_t e = launch_beta_scale(h->stream, m, n, beta->real, beta->imag, C + i * strideC, ldc);
            if (e != cudaSuccess) {
                return to_status(e);
            }
        }
        return CG3M_STATUS_SUCCESS;
    }
    // The reference runs strided 3M batches on its on-chip kernel with the
    // non-finite repair (cgemm_host.cpp:749-782, cgemm_compute_kernel.cpp:672-706):
    // here one persistent launch of the on-chip product family (3M, repair on).
    // Output batches that overlap (strideC == 0 included) are updated in batch
    // order, one launch each (blas/gemm/README.md:850-858).
    const long long span_c = (long long)(n - 1) * ldc + m;
    const bool overlap = batch_count > 1 && (strideC < 0 ? -strideC : strideC) < span_c;
    const int per_launch = overlap ? 1 : batch_count;
    Problem p{transa, transb, m, n, k, alpha->real, alpha->imag, beta->real, beta->imag, A, lda, B, ldb, C, ldc};
    StridedPlan plan;
    if (!make_strided_plan(p, 0, per_launch, h->sm_count, &plan)) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    // One problem per launch (a batch of one, or overlapping outputs): the
    // one-launch kernel, no workspace.
    int tile = 0, parts = 1;
    void* ws = nullptr;
    if (per_launch == 1) {
        plan_single(m, n, k, 0, h->sm_count, -1, 0, &tile, &parts);
    } else {
        const cg3mStatus_t wst = workspace(h, plan.bytes, &ws);
        if (wst != CG3M_STATUS_SUCCESS) {
            return wst;
        }
    }
    for (int i = 0; i < batch_count; i += per_launch) {
        Problem pi = p;
        pi.A = A + i * strideA;
        pi.B = B + i * strideB;
        pi.C = C + i * strideC;
        const cudaError_t e = per_launch == 1 ? launch_single(h->stream, pi, 0, 1, tile, parts)
                                              : launch_strided(h->stream, pi, 0, 1, strideA, strideB, strideC,
                                                               per_launch, plan, ws, h->sm_count);
        if (e != cudaSuccess) {
            return to_status(e);
        }
    }
    return CG3M_STATUS_SUCCESS;
}

cg3mStatus_t cg3mCgemm(cg3mHandle_t h, cg3mOperation_t transa, cg3mOperation_t transb, int m, int n, int k,
                       const cg3mComplex* alpha, const cg3mComplex* A, int lda, const cg3mComplex* B, int ldb,
                       const cg3mComplex* beta, cg3mComplex* C, int ldc)
{
    // aclblasCgemm (cgemm_host.cpp:701-738 with forceThreeProducts = false):
    // enum errors stay INVALID_ENUM, and A, B must be non-null whenever k > 0
    // for a non-empty output, alpha == 0 included.
    if (h == nullptr) {
        return CG3M_STATUS_HANDLE_IS_NULLPTR;
    }
    auto op_ok = [](int op) { return op == CG3M_OP_N || op == CG3M_OP_T || op == CG3M_OP_C; };
    if (!op_ok(transa) || !op_ok(transb)) {
        return CG3M_STATUS_INVALID_ENUM;
    }
    int action = 0;
    const cg3mStatus_t st = validate(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, false, &action);
    if (st != CG3M_STATUS_SUCCESS) {
        return st;
    }
    if (m == 0 || n == 0) {
        return CG3M_STATUS_SUCCESS;
    }
    if (k > 0 && (A == nullptr || B == nullptr)) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    if (action == 0) {
        return CG3M_STATUS_SUCCESS;
    }
    const cg3mStatus_t bs = bind_device(h);
    if (bs != CG3M_STATUS_SUCCESS) {
        return bs;
    }
    if (action == 1) {
        return to_status(launch_beta_scale(h->stream, m, n, beta->real, beta->imag, C, ldc));
    }
    // Unit outputs (alpha = 1, beta = 0) take three products with the
    // non-finite repair, as the reference's cgemm does (cgemm_host.cpp:239-241,
    // 444-453); general alpha/beta take four real products.
    const bool unit = alpha->real == 1.0f && alpha->imag == 0.0f && beta->real == 0.0f && beta->imag == 0.0f;
    const int mode = unit ? 0 : 1;
    Problem p{transa, transb, m, n, k, alpha->real, alpha->imag, beta->real, beta->imag, A, lda, B, ldb, C, ldc};
    if (unit) {
        // Three products with the repair: the FP32 planner's engine.  The packed
        // engine's products equal the on-chip family's bit for bit for the same
        // K split, and its epilogues (GEMM, cluster merge or merge kernel)
        // recompute a non-finite output with the four-product sum before
        // storing it, as the on-chip kernels do.
        Plan plan;
        if (!make_plan(p, cgemm_unit_options(), h->sm_count, &plan)) {
            return CG3M_STATUS_INVALID_VALUE;
        }
        plan.repair = true;
        if (plan.engine == 2) {
            return to_status(launch_single(h->stream, p, 0, 1, plan.onchip_tile, plan.parts));
        }
        void* ws = nullptr;
        const cg3mStatus_t wst = workspace(h, plan.total, &ws);
        if (wst != CG3M_STATUS_SUCCESS) {
            return wst;
        }
        return to_status(enqueue(h->stream, p, plan, ws, h->status, nullptr));
    }
    // Four products: the one-launch kernel of the on-chip family (K
    // partitions merged in a cluster; no workspace).
    int tile = 0, parts = 1;
    plan_single(m, n, k, mode, h->sm_count, -1, 0, &tile, &parts);
    return to_status(launch_single(h->stream, p, mode, 0, tile, parts));
}

cg3mStatus_t cg3mCgemm3mHost(cg3mHandle_t h, cg3mOperation_t transa, cg3mOperation_t transb, int m, int n, int k,
                             const cg3mComplex* alpha, const cg3mComplex* A, int lda, const cg3mComplex* B, int ldb,
                             const cg3mComplex* beta, cg3mComplex* C, int ldc, const cg3mOptions* opts, int panels,
                             cg3mCallInfo* info)
{
    if (h == nullptr) {
        return CG3M_STATUS_HANDLE_IS_NULLPTR;
    }
    int action = 0;
    const cg3mStatus_t st = validate(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, true, &action);
    if (info != nullptr) {
        std::memset(info, 0, sizeof(*info));
    }
    if (st != CG3M_STATUS_SUCCESS || action == 0) {
        return st;
    }
    cg3mOptions o = opts != nullptr ? *opts : cg3mOptions{};
    const cg3mStatus_t bs = bind_device(h);
    if (bs != CG3M_STATUS_SUCCESS) {
        return bs;
    }
    const bool a_normal = transa == CG3M_OP_N || transa == CG3M_OP_R;
    const bool b_normal = transb == CG3M_OP_N || transb == CG3M_OP_R;
    const bool beta_zero = beta->real == 0.0f && beta->imag == 0.0f;
    const bool product = action == 2;
    // Stored shapes: A is (a_rows x a_cols, lda), B (b_rows x b_cols, ldb).
    const int a_rows = a_normal ? m : k, a_cols = a_normal ? k : m;
    const int b_rows = b_normal ? k : n, b_cols = b_normal ? n : k;

    // Panel width: whole output tiles of the whole problem's plan, with the
    // whole problem's K split for every panel (same bits as one call).
    int tile_n = 64;
    if (product) {
        Problem whole{transa, transb, m, n, k, alpha->real, alpha->imag, beta->real, beta->imag, A, lda, B, ldb, C,
                      ldc};
        Plan plan;
        if (!make_plan(whole, o, h->sm_count, &plan)) {
            return CG3M_STATUS_INVALID_VALUE;
        }
        if (o.k_partitions <= 0) {
            o.k_partitions = plan.parts;
        }
        o.form = static_cast<cg3mForm_t>(plan.form);  // a small tensor-core call may run as plain FP32
        tile_n = plan.tile_n;
        if (plan.rounding) {
            panels = 1;
        }
    }
    if (panels <= 0) {
        const int per = std::max(tile_n, ceil_div(ceil_div(n, 8), tile_n) * tile_n);
        panels = ceil_div(n, per);
    }
    panels = std::max(1, std::min(panels, n));
    const int nb = ceil_div(n, panels);
    panels = ceil_div(n, nb);

    // Device copies with the caller's leading dimensions.
    const size_t a_elems = product ? (size_t)lda * a_cols : 0;
    const size_t b_elems = product ? (size_t)ldb * b_cols : 0;
    const size_t c_elems = (size_t)ldc * n;
    const size_t a_off = 0, b_off = align_up(a_elems * 8, 256), c_off = b_off + align_up(b_elems * 8, 256);
    const size_t bytes = c_off + c_elems * 8;
    if (h->host_arena_bytes < bytes) {
        cudaFree(h->host_arena);  // synchronizes with work that may still use it
        h->host_arena = nullptr;
        h->host_arena_bytes = 0;
        if (device_malloc(&h->host_arena, bytes) != cudaSuccess) {
            h->host_arena = nullptr;
            return CG3M_STATUS_ALLOC_FAILED;
        }
        h->host_arena_bytes = bytes;
    }
    if ((h->h2d == nullptr && cudaStreamCreateWithFlags(&h->h2d, cudaStreamNonBlocking) != cudaSuccess) ||
        (h->d2h == nullptr && cudaStreamCreateWithFlags(&h->d2h, cudaStreamNonBlocking) != cudaSuccess)) {
        return CG3M_STATUS_INTERNAL_ERROR;
    }
    char* arena = static_cast<char*>(h->host_arena);
    cg3mComplex* dA = reinterpret_cast<cg3mComplex*>(arena + a_off);
    cg3mComplex* dB = reinterpret_cast<cg3mComplex*>(arena + b_off);
    cg3mComplex* dC = reinterpret_cast<cg3mComplex*>(arena + c_off);

    std::vector<cudaEvent_t> ev(2 * (size_t)panels + 2, nullptr);
    cudaError_t err = cudaSuccess;
    for (auto& e : ev) {
        if (err == cudaSuccess) {
            err = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
        }
    }
    cudaEvent_t ev_start = ev[0], ev_a = ev[1];
    // Copies start after the handle stream's earlier work (which may read the arena).
    if (err == cudaSuccess) err = cudaEventRecord(ev_start, h->stream);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(h->h2d, ev_start, 0);
    if (err == cudaSuccess && product) {
        err = cudaMemcpy2DAsync(dA, (size_t)lda * 8, A, (size_t)lda * 8, (size_t)a_rows * 8, a_cols,
                                cudaMemcpyHostToDevice, h->h2d);
    }
    if (err == cudaSuccess) err = cudaEventRecord(ev_a, h->h2d);
    // Uploads of op(B) and C panels, in panel order on the copy-in stream.
    for (int j = 0; j < panels && err == cudaSuccess; ++j) {
        const int j0 = j * nb, w = std::min(nb, n - j0);
        if (product) {
            if (b_normal) {  // columns j0.. of the stored k x n
                err = cudaMemcpy2DAsync(dB + (size_t)j0 * ldb, (size_t)ldb * 8, B + (size_t)j0 * ldb, (size_t)ldb * 8,
                                        (size_t)b_rows * 8, w, cudaMemcpyHostToDevice, h->h2d);
            } else {  // rows j0.. of the stored n x k
                err = cudaMemcpy2DAsync(dB + j0, (size_t)ldb * 8, B + j0, (size_t)ldb * 8, (size_t)w * 8, b_cols,
                                        cudaMemcpyHostToDevice, h->h2d);
            }
        }
        if (err == cudaSuccess && !beta_zero) {
            err = cudaMemcpy2DAsync(dC + (size_t)j0 * ldc, (size_t)ldc * 8, C + (size_t)j0 * ldc, (size_t)ldc * 8,
                                    (size_t)m * 8, w, cudaMemcpyHostToDevice, h->h2d);
        }
        if (err == cudaSuccess) err = cudaEventRecord(ev[2 + 2 * j], h->h2d);
    }
    cg3mStatus_t result = to_status(err);
    int kernels = 0;
    for (int j = 0; j < panels && result == CG3M_STATUS_SUCCESS; ++j) {
        const int j0 = j * nb, w = std::min(nb, n - j0);
        err = cudaStreamWaitEvent(h->stream, ev_a, 0);
        if (err == cudaSuccess) err = cudaStreamWaitEvent(h->stream, ev[2 + 2 * j], 0);
        if (err != cudaSuccess) {
            result = to_status(err);
            break;
        }
        cg3mCallInfo pi{};
        const cg3mComplex* bj = product ? (b_normal ? dB + (size_t)j0 * ldb : dB + j0) : nullptr;
        result = run_one(h, transa, transb, m, w, k, alpha, product ? dA : nullptr, lda, bj, ldb, beta,
                         dC + (size_t)j0 * ldc, ldc, o, true, &pi);
        if (result != CG3M_STATUS_SUCCESS) {
            break;
        }
        kernels += pi.kernels;
        if (j == 0 && info != nullptr) {
            *info = pi;
        }
        err = cudaEventRecord(ev[3 + 2 * j], h->stream);
        if (err == cudaSuccess) err = cudaStreamWaitEvent(h->d2h, ev[3 + 2 * j], 0);
        if (err == cudaSuccess) {
            err = cudaMemcpy2DAsync(C + (size_t)j0 * ldc, (size_t)ldc * 8, dC + (size_t)j0 * ldc, (size_t)ldc * 8,
                                    (size_t)m * 8, w, cudaMemcpyDeviceToHost, h->d2h);
        }
        result = to_status(err);
    }
    // Drain all three streams before returning (also on errors).
    const cudaError_t s1 = cudaStreamSynchronize(h->h2d);
    const cudaError_t s2 = cudaStreamSynchronize(h->stream);
    const cudaError_t s3 = cudaStreamSynchronize(h->d2h);
    for (auto& e : ev) {
        if (e != nullptr) {
            cudaEventDestroy(e);
        }
    }
    if (result == CG3M_STATUS_SUCCESS) {
        result = to_status(s1 != cudaSuccess ? s1 : s2 != cudaSuccess ? s2 : s3);
    }
    if (info != nullptr && result == CG3M_STATUS_SUCCESS) {
        info->kernels = kernels;  // over all panels
    }
    return result;
}

cg3mStatus_t cg3mSetStageEvents(cg3mHandle_t h, void* const* events, int count)
{
    if (h == nullptr) {
        return CG3M_STATUS_HANDLE_IS_NULLPTR;
    }
    if (count < 0 || count > 32 || (count > 0 && events == nullptr)) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    for (int i = 0; i < 32; ++i) {
        h->stage_events[i] = i < count ? static_cast<cudaEvent_t>(events[i]) : nullptr;
    }
    h->stage_event_count = count;
    return CG3M_STATUS_SUCCESS;
}

cg3mStatus_t cg3mGetDeviceStatus(cg3mHandle_t h, int* flags)
{
    if (flags == nullptr) {
        return h == nullptr ? CG3M_STATUS_HANDLE_IS_NULLPTR : CG3M_STATUS_INVALID_VALUE;
    }
    *flags = 0;
    if (h == nullptr) {
        // The allocation-free entry point's word on the current device: its
        // calls may be on any stream of the device, so the device is drained.
        int* word = nullptr;
        const cg3mStatus_t st = noalloc_status_word(&word);
        if (st != CG3M_STATUS_SUCCESS) {
            return st;
        }
        int v = 0;
        if (cudaDeviceSynchronize() != cudaSuccess ||
            cudaMemcpy(&v, word, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemset(word, 0, sizeof(int)) != cudaSuccess) {
            return CG3M_STATUS_EXECUTION_FAILED;
        }
        *flags = v;
        return CG3M_STATUS_SUCCESS;
    }
    if (h->device < 0) {
        return CG3M_STATUS_SUCCESS;
    }
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
        return CG3M_STATUS_EXECUTION_FAILED;
    }
    int v = 0;
    if (cudaMemcpy(&v, h->status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemset(h->status, 0, sizeof(int)) != cudaSuccess) {
        return CG3M_STATUS_EXECUTION_FAILED;
    }
    *flags = v;
    return CG3M_STATUS_SUCCESS;
}

cg3mStatus_t cg3mGetRoundingStats(cg3mHandle_t h, long long* stats, int count)
{
    if (h == nullptr) {
        return CG3M_STATUS_HANDLE_IS_NULLPTR;
    }
    if (stats == nullptr || count < 0) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    for (int i = 0; i < count; ++i) {
        stats[i] = -1;
    }
    if (h->round_stats == nullptr) {
        return CG3M_STATUS_SUCCESS;
    }
    uint32_t v[8] = {};
    if (cudaStreamSynchronize(h->stream) != cudaSuccess ||
        cudaMemcpy(v, h->round_stats, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess) {
        return CG3M_STATUS_EXECUTION_FAILED;
    }
    for (int i = 0; i < count && i < 8; ++i) {
        stats[i] = (long long)v[i];
    }
    return CG3M_STATUS_SUCCESS;
}

cg3mStatus_t cg3mDiagGuardStatus(int* enabled, int* damaged)
{
    if (enabled == nullptr || damaged == nullptr) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    *enabled = guard_bands_on() ? 1 : 0;
    *damaged = 0;
    if (!guard_bands_on()) {
        return CG3M_STATUS_SUCCESS;
    }
    return read_guard_damage(damaged) == cudaSuccess ? CG3M_STATUS_SUCCESS : CG3M_STATUS_EXECUTION_FAILED;
}

cg3mStatus_t cg3mDiagFailAllocations(int count)
{
    if (count < 0) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    g_fail_allocs.store(count);
    return CG3M_STATUS_SUCCESS;
}

cg3mStatus_t cg3mDiagBoundedWait(cg3mHandle_t h, long long limit_ns, int* gave_up)
{
    if (gave_up == nullptr || limit_ns <= 0 || limit_ns > 10000000000ll) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    *gave_up = 0;
    int* word = nullptr;
    cudaStream_t s = nullptr;
    if (h == nullptr) {
        const cg3mStatus_t st = noalloc_status_word(&word);
        if (st != CG3M_STATUS_SUCCESS) {
            return st;
        }
    } else {
        const cg3mStatus_t bs = bind_device(h);
        if (bs != CG3M_STATUS_SUCCESS) {
            return bs;
        }
        word = h->status;
        s = h->stream;
    }
    // word[1] is spare in both status blocks (64 and 256 bytes): the probe's
    // result slot.
    int v = 0;
    if (cudaMemsetAsync(word + 1, 0, sizeof(int), s) != cudaSuccess ||
        launch_wait_probe(s, word, (unsigned long long)limit_ns, word + 1) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess ||
        cudaMemcpy(&v, word + 1, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
        return CG3M_STATUS_EXECUTION_FAILED;
    }
    *gave_up = v;
    return CG3M_STATUS_SUCCESS;
}

cg3mStatus_t cg3mValidate(cg3mOperation_t transa, cg3mOperation_t transb, int m, int n, int k,
                          const cg3mComplex* alpha, const void* A, int lda, const void* B, int ldb,
                          const cg3mComplex* beta, const void* C, int ldc, int allow_conj_only, int* action)
{
    int a = 0;
    const cg3mStatus_t st =
        validate(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, allow_conj_only != 0, &a);
    if (action != nullptr) {
        *action = a;
    }
    return st;
}

cg3mStatus_t cg3mPlan(cg3mOperation_t transa, cg3mOperation_t transb, int m, int n, int k, const cg3mComplex* alpha,
                      int lda, int ldb, const cg3mComplex* beta, int ldc, const cg3mOptions* opts, int sm_count,
                      cg3mCallInfo* info)
{
    if (info == nullptr || alpha == nullptr || beta == nullptr || m <= 0 || n <= 0 || k <= 0) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    const cg3mOptions o = opts != nullptr ? *opts : cg3mOptions{};
    Problem p{transa, transb, m, n, k, alpha->real, alpha->imag, beta->real, beta->imag,
              nullptr, lda, nullptr, ldb, nullptr, ldc};
    Plan plan;
    if (!make_plan(p, o, sm_count, &plan)) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    std::memset(info, 0, sizeof(*info));
    info->path = plan.engine == 2 ? 4 : plan.parts > 1 ? 3 : 2;
    info->form = plan.form;
    info->tile_m = plan.tile_m;
    info->tile_n = plan.tile_n;
    info->k_partitions = plan.parts;
    info->k_span = plan.span;
    info->rounding = plan.rounding ? 1 : 0;
    info->kernels =
        plan.engine == 2 ? 1 : 2 + (plan.parts > 1 && !plan.cluster_merge ? 1 : 0) + (plan.rounding ? (plan.form == CG3M_FORM_FP32 ? 7 : 11) : 0);
    info->workspace_bytes = plan.total;
    return CG3M_STATUS_SUCCESS;
}

cg3mStatus_t cg3mPlanOnchip(int m, int n, int k, int mode, int batch, int sm_count, cg3mCallInfo* info)
{
    if (info == nullptr) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    if (mode == 2) {  // cg3mCgemm with alpha = 1, beta = 0: the FP32 planner's engine, repair in its epilogue
        if (batch != 1 || m <= 0 || n <= 0 || k <= 0) {
            return CG3M_STATUS_INVALID_VALUE;
        }
        Problem p{CG3M_OP_N, CG3M_OP_N, m, n, k, 1.0f, 0.0f, 0.0f, 0.0f, nullptr, m, nullptr, k, nullptr, m};
        Plan plan;
        if (!make_plan(p, cgemm_unit_options(), sm_count > 0 ? sm_count : 148, &plan)) {
            return CG3M_STATUS_INVALID_VALUE;
        }
        std::memset(info, 0, sizeof(*info));
        info->path = plan.engine == 2 ? 4 : plan.parts > 1 ? 3 : 2;
        info->tile_m = plan.tile_m;
        info->tile_n = plan.tile_n;
        info->k_partitions = plan.parts;
        info->k_span = plan.span;
        info->kernels = plan.engine == 2 ? 1 : 2 + (plan.parts > 1 && !plan.cluster_merge ? 1 : 0);
        info->workspace_bytes = plan.total;
        return CG3M_STATUS_SUCCESS;
    }
    Problem p{CG3M_OP_N, CG3M_OP_N, m, n, k, 1.0f, 0.0f, 0.0f, 0.0f, nullptr, m, nullptr, k, nullptr, m};
    StridedPlan plan;
    if (!make_strided_plan(p, mode, batch, sm_count > 0 ? sm_count : 148, &plan)) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    std::memset(info, 0, sizeof(*info));
    if (batch == 1) {  // one problem: the one-launch kernel
        int tile = 0, parts = 1;
        plan_single(m, n, k, mode, sm_count > 0 ? sm_count : 148, -1, 0, &tile, &parts);
        info->path = 4;
        info->tile_m = single_tile_bm(tile);
        info->tile_n = single_tile_bn(tile);
        info->k_partitions = parts;
        info->k_span = parts > 1 ? ceil_div(ceil_div(k, 16), parts) * 16 : k;
        info->kernels = 1;
        return CG3M_STATUS_SUCCESS;
    }
    info->path = plan.parts > 1 ? 3 : 2;
    info->tile_m = plan.tile_m;
    info->tile_n = plan.tile_n;
    info->k_partitions = plan.parts;
    info->k_span = plan.span;
    info->kernels = 1;
    info->workspace_bytes = plan.bytes;
    return CG3M_STATUS_SUCCESS;
}

cg3mStatus_t cg3mZgemmReference(cg3mHandle_t h, cg3mOperation_t transa, cg3mOperation_t transb, int m, int n, int k,
                                const cg3mComplex* alpha, const cg3mComplex* A, int lda, const cg3mComplex* B,
                                int ldb, const cg3mComplex* beta, const cg3mComplex* C, int ldc, void* out64)
{
    if (h == nullptr) {
        return CG3M_STATUS_HANDLE_IS_NULLPTR;
    }
    int action = 0;
    const cg3mStatus_t st = validate(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, true, &action);
    if (st != CG3M_STATUS_SUCCESS || m == 0 || n == 0) {
        return st;
    }
    if (out64 == nullptr) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    const cg3mStatus_t bs = bind_device(h);
    if (bs != CG3M_STATUS_SUCCESS) {
        return bs;
    }
    Problem p{transa, transb, m, n, k, alpha->real, alpha->imag, beta->real, beta->imag, A, lda, B, ldb,
              const_cast<cg3mComplex*>(C), ldc};
    return to_status(launch_zgemm_ref(h->stream, p, C, out64));
}

cg3mStatus_t cg3mErrorReport(cg3mHandle_t h, int m, int n, const cg3mComplex* C, int ldc, const void* out64,
                             double* report)
{
    if (h == nullptr) {
        return CG3M_STATUS_HANDLE_IS_NULLPTR;
    }
    if (m <= 0 || n <= 0 || ldc < m || C == nullptr || out64 == nullptr || report == nullptr) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    const cg3mStatus_t bs = bind_device(h);
    if (bs != CG3M_STATUS_SUCCESS) {
        return bs;
    }
    double* dev = nullptr;
    if (cudaMalloc(&dev, 8 * sizeof(double)) != cudaSuccess) {
        return CG3M_STATUS_ALLOC_FAILED;
    }
    cudaError_t err = launch_error_report(h->stream, m, n, C, ldc, out64, dev);
    double host[8] = {0};
    if (err == cudaSuccess) {
        err = cudaMemcpyAsync(host, dev, sizeof(host), cudaMemcpyDeviceToHost, h->stream);
    }
    if (err == cudaSuccess) {
        err = cudaStreamSynchronize(h->stream);
    }
    cudaFree(dev);
    if (err != cudaSuccess) {
        return CG3M_STATUS_EXECUTION_FAILED;
    }
    // host: [0] sum |d|^2, [1] sum |x|^2, [2] max rel re, [3] max rel im, [4] max abs re, [5] max abs im
    report[0] = host[1] > 0 ? __builtin_sqrt(host[0] / host[1]) : __builtin_sqrt(host[0]);
    report[1] = host[2];
    report[2] = host[3];
    report[3] = host[4];
    report[4] = host[5];
    return CG3M_STATUS_SUCCESS;
}

// ---- aclblas-named entry points (drop-in link compatibility) -----------------

aclblasStatus_t aclblasCreate(aclblasHandle_t* handle) { return cg3mCreate(handle); }
aclblasStatus_t aclblasDestroy(aclblasHandle_t handle) { return cg3mDestroy(handle); }
aclblasStatus_t aclblasSetStream(aclblasHandle_t handle, aclrtStream stream) { return cg3mSetStream(handle, stream); }
aclblasStatus_t aclblasGetStream(aclblasHandle_t handle, aclrtStream* stream) { return cg3mGetStream(handle, stream); }
aclblasStatus_t aclblasSetWorkspace(aclblasHandle_t handle, void* workspace, size_t bytes)
{
    return cg3mSetWorkspace(handle, workspace, bytes);
}
aclblasStatus_t aclblasGetVersion(aclblasHandle_t handle, int* version) { return cg3mGetVersion(handle, version); }

aclblasStatus_t aclblasCgemm(aclblasHandle_t handle, aclblasOperation_t transa, aclblasOperation_t transb, int m,
                             int n, int k, const aclblasComplex* alpha, const aclblasComplex* A, int lda,
                             const aclblasComplex* B, int ldb, const aclblasComplex* beta, aclblasComplex* C, int ldc)
{
    return cg3mCgemm(handle, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

aclblasStatus_t aclblasCgemm3m(aclblasHandle_t handle, aclblasOperation_t transa, aclblasOperation_t transb, int m,
                               int n, int k, const aclblasComplex* alpha, const aclblasComplex* A, int lda,
                               const aclblasComplex* B, int ldb, const aclblasComplex* beta, aclblasComplex* C,
                               int ldc)
{
    return cg3mCgemm3m(handle, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

aclblasStatus_t aclblasCgemm3mStridedBatched(aclblasHandle_t handle, aclblasOperation_t transa,
                                             aclblasOperation_t transb, int m, int n, int k,
                                             const aclblasComplex* alpha, const aclblasComplex* A, int lda,
                                             int64_t strideA, const aclblasComplex* B, int ldb, int64_t strideB,
                                             const aclblasComplex* beta, aclblasComplex* C, int ldc, int64_t strideC,
                                             int batchCount)
{
    return cg3mCgemm3mStridedBatched(handle, transa, transb, m, n, k, alpha, A, lda, strideA, B, ldb, strideB, beta,
                                     C, ldc, strideC, batchCount);
}

}  // extern "C"
