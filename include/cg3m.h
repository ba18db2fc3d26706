/*
 * cg3m.h -- C ABI of the B200-native cgemm3m (complex64 GEMM with three real
 * matrix products), a drop-in for the reference's aclblasCgemm3m surface.
 *
 * All entry points are extern "C", take plain pointers and sizes, and return a
 * cg3mStatus_t.  Citations name the reference interface each entry replaces
 * (paths inside the reference's ops-blas/ tree).
 *
 * Conventions shared with the reference:
 *   - A, B, C are column-major complex64 arrays in device memory owned by the
 *     caller; alpha and beta are host pointers read during the call.
 *   - Work is enqueued asynchronously on the handle's stream; no entry point
 *     synchronizes except cg3mDestroy, cg3mGetDeviceStatus, the batch-plan
 *     calls and the host-buffer cg3mCgemm3mHost.
 *   - One handle must not be used by several host threads at once (its
 *     workspace is shared by every call made through it).
 *   - C must not alias A or B.  Padding rows [m, ldc) of C are never written.
 */
#ifndef CG3M_H_
#define CG3M_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference names are kept (cann_ops_blas.h:40-57 uses
 * ACLBLAS_STATUS_*); their numeric values are not shipped with the reference,
 * so these values are this library's own. */
typedef enum {
    CG3M_STATUS_SUCCESS = 0,
    CG3M_STATUS_HANDLE_IS_NULLPTR = 1,
    CG3M_STATUS_INVALID_VALUE = 2,
    CG3M_STATUS_INVALID_ENUM = 3,
    CG3M_STATUS_ALLOC_FAILED = 4,
    CG3M_STATUS_INTERNAL_ERROR = 5,
    CG3M_STATUS_EXECUTION_FAILED = 6,
    CG3M_STATUS_NOT_SUPPORTED = 7
} cg3mStatus_t;

/* op() codes: N, T, C as in the reference (numeric values follow cuBLAS).
 * CG3M_OP_R (conjugate without transpose) is accepted only by the extended
 * entry points; the drop-in cg3mCgemm3m rejects it like any other bad enum. */
typedef enum { CG3M_OP_N = 0, CG3M_OP_T = 1, CG3M_OP_C = 2, CG3M_OP_R = 3 } cg3mOperation_t;

/* Arithmetic form of the three real products.
 *   FP32     -- strict FP32 FFMA on the CUDA cores; the drop-in form;
 *               bitwise deterministic run to run.
 *   TF32X3   -- tensor-core 3xTF32: each operand split x = hi + lo (both TF32),
 *               products hi*hi + hi*lo + lo*hi accumulated in FP32 (TMEM).
 *   BF16X6   -- tensor-core split-BF16: x = b0 + b1 + b2, the six products
 *               with b_i*b_j, i+j <= 2, accumulated in FP32 (TMEM).
 *   BF16X9   -- as BF16X6 with all nine products.
 * In every form the sums Ar+Ai, Br+Bi are formed in FP32 before splitting and
 * the epilogue (Re = P0-P1, Im = P2-P0-P1, alpha, beta) runs in FP32. */
typedef enum { CG3M_FORM_FP32 = 0, CG3M_FORM_TF32X3 = 1, CG3M_FORM_BF16X6 = 2, CG3M_FORM_BF16X9 = 3 } cg3mForm_t;

/* Rounding-correction pass (reference: gemm_cgemm3m_rounding_do,
 * blas/gemm/arch35/cgemm3m_rounding_kernel.cpp:474-497, gated at
 * cgemm_host.cpp:234-238).
 *   AUTO -- as the reference: only for m==n==k in [2048,4096], lda==ldb==ldc==m,
 *           alpha==1, beta==0.  FP32 form: flagged outputs are recomputed in
 *           FP32 fixed order (the reference's replay bit for bit).  Tensor-core
 *           forms: the risk plane comes from one tensor pass (four real
 *           products) over the leading split planes of the real and imaginary
 *           parts, and the call runs unsplit over K whatever k_partitions asks;
 *           every output of a 256 x 256 tile holding a 16 x 16
 *           tile with more than 64 flagged outputs is computed to within one
 *           FP32 rounding of the exact product (exact int8 products by residues
 *           on the tensor cores, FP64 where their bound does not certify it);
 *           the other tiles get the form's own products, their flagged outputs
 *           recomputed to within one FP32 rounding in FP64.
 *   OFF  -- never. */
typedef enum { CG3M_ROUNDING_AUTO = 0, CG3M_ROUNDING_OFF = 1 } cg3mRounding_t;

typedef struct {
    float real;
    float imag;
} cg3mComplex; /* layout of aclblasComplex {float real; float imag;} (cgemm_host.cpp:719) */

typedef struct cg3mContext* cg3mHandle_t;

/* Options of the extended entry points (zero-initialised = drop-in behaviour). */
typedef struct {
    cg3mForm_t form;
    cg3mRounding_t rounding;
    int k_partitions; /* 0 = planner's choice; else force this many K partitions (1..64; the
                         tensor-core forms' rounding pass runs unsplit) */
    int tc_segment;   /* tensor-core forms: K terms accumulated in TMEM before each round-to-nearest
                         FP32 merge (0 = planner: 128 for k >= 2048, 64 for k > 1024, else 32;
                         rounded up to the kernel's K-block of 32 or 64) */
    int engine;       /* FP32 form: 0 = planner's choice; 1 = packed planes (pack kernel, TMA-fed FFMA
                         GEMM, split-K merge kernel); 2 = one launch that reads the caller's matrices and
                         merges its K partitions (<= 8) inside a thread-block cluster.  For a given K
                         split both give the same bits.  2 is refused (INVALID_VALUE) for the
                         tensor-core forms, with the rounding pass, or with k_partitions > 8.
                         Tensor-core forms: 0 may run a small problem as the plain FP32 product (the
                         FP32 planner's plan) when that is clearly faster (the call info then reports
                         form FP32; its error is the plain form's); 1 always uses the tensor cores. */
    int onchip_tile;  /* engine 2: 0 = planner, 1..6 = 128x64, 64x64, 128x32, 32x128, 64x32, 32x32 */
    int reserved[2];
} cg3mOptions;

/* What one call did (filled when a non-null pointer is passed). */
typedef struct {
    int path;            /* 0 quick return, 1 beta-scale only, 2 fused GEMM, 3 split-K GEMM + merge,
                            4 one launch with the K partitions merged in a cluster (engine 2) */
    int form;            /* cg3mForm_t actually used */
    int tile_m, tile_n;  /* output tile of the GEMM kernel */
    int k_partitions;    /* K partitions (1 = none) */
    int k_span;          /* K terms per partition */
    int rounding;        /* 1 if the rounding-correction pass was enqueued */
    int kernels;         /* kernels launched by this call */
    size_t workspace_bytes;
} cg3mCallInfo;

/* ---- handle / stream / workspace (cann_ops_blas.h:31-98) ------------------ */

/* aclblasCreate (cann_ops_blas.h:46).  *handle must be NULL on entry
 * (non-null -> INVALID_VALUE).  Device resources (the 32 MiB default workspace
 * and a status word) are bound to the current device on the first call that
 * launches work, so a handle can be created and validated without a GPU. */
cg3mStatus_t cg3mCreate(cg3mHandle_t* handle);

/* aclblasDestroy (cann_ops_blas.h:59): synchronizes the handle's stream, frees
 * the default workspace; a user workspace is forgotten, never freed. */
cg3mStatus_t cg3mDestroy(cg3mHandle_t handle);

/* aclblasSetStream (cann_ops_blas.h:71): NULL selects the legacy default
 * stream; switching streams returns the handle to its default workspace. */
cg3mStatus_t cg3mSetStream(cg3mHandle_t handle, void* stream);

/* aclblasGetStream (cann_ops_blas.h:81). */
cg3mStatus_t cg3mGetStream(cg3mHandle_t handle, void** stream);

/* aclblasSetWorkspace (cann_ops_blas.h:98): borrows device memory (grow-only:
 * kept only when larger than the current user workspace). */
cg3mStatus_t cg3mSetWorkspace(cg3mHandle_t handle, void* workspace, size_t workspace_bytes);

/* aclblasGetVersion (cann_ops_blas.h:108): MAJOR*10000 + MINOR*100 + PATCH. */
cg3mStatus_t cg3mGetVersion(cg3mHandle_t handle, int* version);

/* ---- the drop-in (cann_ops_blas.h:497-500; cgemm3m_host.cpp:17-23) ------- */

/* C <- alpha*op(A)*op(B) + beta*C with three real products, strict FP32.
 * Validation order and statuses follow LaunchComplexGemm/ValidateCgemmParams
 * (cgemm_host.cpp:589-634,687-730): null handle -> HANDLE_IS_NULLPTR; bad
 * transa/transb, negative m/n/k, lda/ldb/ldc too small, null alpha/beta ->
 * INVALID_VALUE; then m==0||n==0 -> SUCCESS with nothing touched; then C must
 * be non-null and, unless alpha==0, A and B must be non-null when k>0.
 * k==0 or alpha==0 scales C by beta only (beta==1: nothing; beta==0: C=0
 * without reading C).  beta==0 never reads C. */
cg3mStatus_t cg3mCgemm3m(cg3mHandle_t handle, cg3mOperation_t transa, cg3mOperation_t transb, int m, int n, int k,
                         const cg3mComplex* alpha, const cg3mComplex* A, int lda, const cg3mComplex* B, int ldb,
                         const cg3mComplex* beta, cg3mComplex* C, int ldc);

/* ---- extensions (no single reference counterpart) ------------------------ */

/* The drop-in with a form / rounding / K-split choice and an optional report of
 * what ran.  Also accepts CG3M_OP_R.  opts == NULL means the drop-in. */
cg3mStatus_t cg3mCgemm3mEx(cg3mHandle_t handle, cg3mOperation_t transa, cg3mOperation_t transb, int m, int n, int k,
                           const cg3mComplex* alpha, const cg3mComplex* A, int lda, const cg3mComplex* B, int ldb,
                           const cg3mComplex* beta, cg3mComplex* C, int ldc, const cg3mOptions* opts,
                           cg3mCallInfo* info);

/* aclblasCgemm3mStridedBatched (cann_ops_blas.h:652; semantics
 * blas/gemm/README.md:809-907): C_i = alpha*op(A_i)*op(B_i) + beta*C_i with
 * X_i = X + i*strideX (complex elements, zero or negative allowed); when
 * output batches overlap (strideC==0 included) they are updated in batch
 * order.  Statuses as the reference's strided API: bad enum -> INVALID_ENUM.
 * Runs as one persistent launch of 3M products read straight from A and B,
 * with products that came out non-finite recomputed by explicit FP32
 * four-product terms (the reference's RepairNonFiniteOutput,
 * cgemm_compute_kernel.cpp:672-706); bitwise repeatable. */
/* aclblasCgemm (cann_ops_blas.h:492; cgemm_host.cpp:701-738): the same
 * product with the reference cgemm's statuses (bad enum -> INVALID_ENUM; A and
 * B required whenever k > 0, alpha == 0 included).  alpha = 1, beta = 0 runs
 * three products with the non-finite repair; other scalars run four real
 * products (Re = Ar.Br - Ai.Bi, Im = Ar.Bi + Ai.Br) with one FFMA per term. */
cg3mStatus_t cg3mCgemm(cg3mHandle_t handle, cg3mOperation_t transa, cg3mOperation_t transb, int m, int n, int k,
                       const cg3mComplex* alpha, const cg3mComplex* A, int lda, const cg3mComplex* B, int ldb,
                       const cg3mComplex* beta, cg3mComplex* C, int ldc);

cg3mStatus_t cg3mCgemm3mStridedBatched(cg3mHandle_t handle, cg3mOperation_t transa, cg3mOperation_t transb, int m,
                                       int n, int k, const cg3mComplex* alpha, const cg3mComplex* A, int lda,
                                       int64_t strideA, const cg3mComplex* B, int ldb, int64_t strideB,
                                       const cg3mComplex* beta, cg3mComplex* C, int ldc, int64_t strideC,
                                       int batch_count);

/* One problem of a heterogeneous batch (device pointers, host scalars). */
typedef struct {
    int transa, transb;
    int m, n, k;
    cg3mComplex alpha, beta;
    const cg3mComplex* A;
    int lda;
    const cg3mComplex* B;
    int ldb;
    cg3mComplex* C;
    int ldc;
} cg3mProblem;

/* Opaque plan of a heterogeneous batch: tile/K-split tables chosen by the
 * autotuner, a device-side task list, and (optionally) a captured CUDA graph
 * holding the one persistent launch. */
typedef struct cg3mBatchPlan* cg3mBatchPlan_t;

/* Plans `count` problems (validated individually like cg3mCgemm3m, op code R
 * also accepted; the first invalid one returns its status and its index in
 * *bad_index).  `tune` != 0 times the candidate tile/split tables on the
 * device before choosing (the problems' A and B are read, C is not written;
 * the choice is cached per device and batch shape).  Each output is
 * bit-identical to cg3mCgemm3mEx (FP32 form) with the K split the plan chose.
 * A plan is executed on one stream at a time; its buffers must stay valid. */
cg3mStatus_t cg3mBatchPlanCreate(cg3mHandle_t handle, const cg3mProblem* problems, int count, int tune,
                                 cg3mBatchPlan_t* plan, int* bad_index);
/* Enqueues the whole batch on the handle's stream as one persistent launch
 * (replaying the captured graph when use_graph != 0). */
cg3mStatus_t cg3mBatchPlanExecute(cg3mHandle_t handle, cg3mBatchPlan_t plan, int use_graph);
cg3mStatus_t cg3mBatchPlanDestroy(cg3mBatchPlan_t plan);
/* Tile shape / K split the plan chose per problem (arrays of `count`). */
cg3mStatus_t cg3mBatchPlanDescribe(cg3mBatchPlan_t plan, int* tile_m, int* tile_n, int* k_partitions);

/* Instrumentation: when count > 0 (at most 32), every later call made through
 * the handle brackets its j-th kernel (0-based, in the order the call info's
 * kernel count enumerates them) by events[2j] and events[2j + 1], both
 * recorded on the stream that kernel runs on, for the entries below count; no
 * work is skipped or reordered.  The events are
 * cudaEvent_t values owned by the caller.  count == 0 turns it off. */
cg3mStatus_t cg3mSetStageEvents(cg3mHandle_t handle, void* const* events, int count);

/* Device status word of the handle: synchronizes the stream, returns and
 * clears the error bits kernels set when a bounded wait gave up
 * (1: pipeline wait timed out).  0 means no device-side error.
 * handle == NULL reads (and clears) the word of cg3mCgemm3mNoAlloc on the
 * current device instead, after synchronizing the whole device. */
cg3mStatus_t cg3mGetDeviceStatus(cg3mHandle_t handle, int* flags);

/* Counters of the rounding-correction pass of the last call made through the
 * handle (synchronizes its stream): stats[0] = outputs flagged, stats[1] =
 * flagged outputs recomputed by the tile kernels (16 x 16 tiles holding more
 * than 64 flagged outputs; tensor-core forms: every 256 x 256 tile holding
 * one), stats[2] = flagged outputs recomputed one by one (the other tiles),
 * stats[3] = tensor-core forms: outputs of those tiles the exact int8
 * products could not certify, recomputed in FP64, stats[4] = 256 x 256 tiles
 * run on the exact int8 products, stats[5] = the output positions inside the
 * matrix those tiles cover; entries past 5 are reserved.  All -1 when that call ran no rounding pass.  Valid until the
 * next call through the handle (the counters live in its workspace). */
cg3mStatus_t cg3mGetRoundingStats(cg3mHandle_t handle, long long* stats, int count);

/* ---- diagnostics for failure handling (test use) -------------------------- */

/* The next `count` device allocations the handle API attempts (status word,
 * default workspace, workspace growth, host-buffer copies) fail as if the
 * device were out of memory; the call that needed one returns
 * CG3M_STATUS_ALLOC_FAILED without touching C.  0 turns it off. */
cg3mStatus_t cg3mDiagFailAllocations(int count);

/* Guard bands around the workspace regions of cg3mCgemm3m / cg3mCgemm3mEx /
 * cg3mCgemm3mNoAlloc calls, enabled only when CG3M_GUARD_BANDS is set in the
 * environment before the library loads (a test-build switch: it adds 4 KB
 * after every region of the planned workspace).  Each call then fills the
 * bands with a byte pattern before its first kernel and checks them after
 * its last.  *enabled = 1 when bands are on; *damaged = 1 when any call since
 * the last query found a band overwritten (synchronizes the device, clears). */
cg3mStatus_t cg3mDiagGuardStatus(int* enabled, int* damaged);

/* Runs one bounded wait that cannot complete (an mbarrier nothing arrives on)
 * through the wait every pipeline kernel uses, with a limit of limit_ns
 * (0 < limit_ns <= 10 s), on the handle's stream, and synchronizes.  The
 * wait gives up, sets bit 1 of the handle's status word (handle == NULL: the
 * cg3mCgemm3mNoAlloc word of the current device) and the kernel returns;
 * *gave_up is 1 when it did.  No fault, no hang: the context stays usable. */
cg3mStatus_t cg3mDiagBoundedWait(cg3mHandle_t handle, long long limit_ns, int* gave_up);

/* ---- allocation-free variant (no counterpart in the reference) ----------- */

/* The drop-in FP32 product (same arguments, validation, statuses and result
 * bits as cg3mCgemm3m) for callers that must not call cudaMalloc/cudaFree at
 * this point -- e.g. under a caching allocator that owns the device heap, or
 * in a loop where an allocation would synchronize the device.  It allocates
 * nothing: its scratch is one fixed 32 MiB device array inside the library
 * (held by every GPU that loads it, until exit).  It takes a CUDA stream
 * instead of a handle.  The first call on each device resolves the array's
 * device address (cudaGetSymbolAddress), so make that first call before any
 * stream capture.  Problems whose scratch would exceed the array return
 * CG3M_STATUS_INVALID_VALUE with C untouched, and so is a stream that does
 * not belong to the current device (the array's address is per device).
 * Every call shares the one array, so calls whose work overlaps on the GPU
 * (other streams, other host threads) race on it; serialise them.  The call
 * returns before its kernels run, so a kernel whose bounded wait gave up
 * (C then incomplete) cannot change its status: kernels set bit 1 of a status
 * word that stays set until cg3mGetDeviceStatus(NULL, &flags) reads it. */
cg3mStatus_t cg3mCgemm3mNoAlloc(void* stream, cg3mOperation_t transa, cg3mOperation_t transb, int m, int n, int k,
                                const cg3mComplex* alpha, const cg3mComplex* A, int lda, const cg3mComplex* B,
                                int ldb, const cg3mComplex* beta, cg3mComplex* C, int ldc);

/* Host-buffer form (extension): A, B and C live in HOST memory (page-locked
 * for the copies to overlap).  The call uploads A, streams op(B) and C in
 * column panels -- panel j+1 uploads while panel j computes on the handle's
 * stream and panel j-1 downloads -- and returns once all of C is back on the
 * host.  Every panel is the cg3mCgemm3mEx call on device copies that keep the
 * caller's leading dimensions, with the K split of the whole problem, so C
 * holds the bits the device call on the whole problem would give.  When the
 * rounding-correction pass applies to the whole problem it runs as one panel.
 * `panels` <= 0 picks the count (about 8 panels of whole tiles); the device
 * copies are kept in the handle for later calls.  op code R is accepted.
 * C rows past m (padding) are neither read nor written. */
cg3mStatus_t cg3mCgemm3mHost(cg3mHandle_t handle, cg3mOperation_t transa, cg3mOperation_t transb, int m, int n, int k,
                             const cg3mComplex* alpha, const cg3mComplex* A, int lda, const cg3mComplex* B, int ldb,
                             const cg3mComplex* beta, cg3mComplex* C, int ldc, const cg3mOptions* opts, int panels,
                             cg3mCallInfo* info);

/* ---- host-only helpers (no device access; usable without a GPU) ---------- */

/* Runs exactly the validation of cg3mCgemm3m (including the quick-return
 * classification) without touching the device: returns the status the call
 * would return, and in *action 0 = nothing to do, 1 = beta scale only,
 * 2 = product path. */
cg3mStatus_t cg3mValidate(cg3mOperation_t transa, cg3mOperation_t transb, int m, int n, int k,
                          const cg3mComplex* alpha, const void* A, int lda, const void* B, int ldb,
                          const cg3mComplex* beta, const void* C, int ldc, int allow_conj_only, int* action);

/* The planner's decision for a problem on a device with `sm_count` SMs
 * (fills info; no device access). */
cg3mStatus_t cg3mPlan(cg3mOperation_t transa, cg3mOperation_t transb, int m, int n, int k, const cg3mComplex* alpha,
                      int lda, int ldb, const cg3mComplex* beta, int ldc, const cg3mOptions* opts, int sm_count,
                      cg3mCallInfo* info);

/* The on-chip family's decision (cg3mCgemm, cg3mCgemm3mStridedBatched) for
 * one problem shape: mode 0 = three products, 1 = four; `batch` problems per
 * launch.  Fills tile_m, tile_n, k_partitions, k_span and workspace_bytes.
 * batch == 1 (cg3mCgemm, a strided batch of one, or overlapping outputs run
 * one per launch) reports the one-launch kernel: path 4, no workspace.
 * mode 2 (batch 1 only) = cg3mCgemm with alpha = 1, beta = 0: three products
 * with the non-finite repair on the FP32 planner's engine (the one-launch
 * kernel, or the packed engine, whose epilogue repairs each non-finite
 * output before storing it). */
cg3mStatus_t cg3mPlanOnchip(int m, int n, int k, int mode, int batch, int sm_count, cg3mCallInfo* info);

/* ---- diagnostics (not a compute path of cgemm3m) ------------------------- */

/* FP64 reference product on the device, for error reports only:
 * out64[j*m+i] = alpha*op(A)*op(B) (+ beta*C) in complex128, m x n packed. */
cg3mStatus_t cg3mZgemmReference(cg3mHandle_t handle, cg3mOperation_t transa, cg3mOperation_t transb, int m, int n,
                                int k, const cg3mComplex* alpha, const cg3mComplex* A, int lda, const cg3mComplex* B,
                                int ldb, const cg3mComplex* beta, const cg3mComplex* C, int ldc, void* out64);

/* Normwise and componentwise errors of C (ldc) against out64 (m x n packed),
 * computed on the device.  report[0] = ||C-C64||_F/||C64||_F,
 * report[1] = max |dRe|/|Re64|, report[2] = max |dIm|/|Im64|,
 * report[3] = max |dRe|, report[4] = max |dIm| (host array of 5 doubles). */
cg3mStatus_t cg3mErrorReport(cg3mHandle_t handle, int m, int n, const cg3mComplex* C, int ldc, const void* out64,
                             double* report);

#ifdef __cplusplus
}
#endif

#endif /* CG3M_H_ */
