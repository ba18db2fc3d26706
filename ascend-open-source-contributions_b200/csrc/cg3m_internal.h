// cg3m_internal.h -- host-side types shared by the C ABI, the planner and the
// kernel launchers.  No torch types anywhere: plain CUDA runtime only.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <functional>
#include <vector>

#include "../../include/cg3m.h"

struct cg3mContext {
    cudaStream_t stream = nullptr;
    int device = -1;             // bound on first launch
    int sm_count = 0;
    void* default_ws = nullptr;  // library-owned workspace (grown on demand)
    size_t default_ws_bytes = 0;
    void* user_ws = nullptr;     // borrowed (cg3mSetWorkspace), never freed here
    size_t user_ws_bytes = 0;
    int* status = nullptr;       // device status word (bounded-wait failures)
    uint32_t* round_stats = nullptr;  // counters of the last call's rounding pass (null if it had none)
    cudaEvent_t stage_events[32] = {};
    int stage_event_count = 0;
    // host-buffer entry point: device copies of A, B, C and its copy streams
    void* host_arena = nullptr;
    size_t host_arena_bytes = 0;
    cudaStream_t h2d = nullptr;
    cudaStream_t d2h = nullptr;
};

namespace cg3m {

constexpr size_t kDefaultWorkspaceBytes = size_t(32) << 20;  // cann_ops_blas.h:33-35
constexpr size_t kRegionAlign = 512;                          // cgemm_host.cpp:33 (16 x 32 B)

// Which plane layout a GEMM kernel consumes.
enum class Layout { MnMajor, KMajor };

// One planned cgemm3m call.
struct Plan {
    int action = 0;   // 0 nothing, 1 beta-scale only, 2 product path
    int form = CG3M_FORM_FP32;
    int tile_m = 128, tile_n = 64;
    int parts = 1;
    int span = 0;
    bool unit = false;       // alpha == 1, beta == 0
    bool beta_zero = false;
    bool rounding = false;
    int tc_segment = 0;      // K terms per TMEM accumulation segment (tensor-core forms)
    int engine = 1;          // 1 packed planes (pack + GEMM [+ merge]), 2 one cluster-merged launch
    int onchip_tile = 0;     // engine 2: tile index of the on-chip family (0 128x64 .. 5 32x32)
    bool cluster_merge = false;  // FP32 packed engine: the K partitions (2..8) merge inside their cluster
    bool repair = false;         // cg3mCgemm, alpha = 1, beta = 0: non-finite outputs repaired in the epilogue
    double est_us = 0.0;         // FP32 plans: the planner's time estimate (microseconds)
    // workspace layout (byte offsets from the workspace base)
    size_t planes_a_off = 0, planes_b_off = 0, partial_off = 0, round_off = 0, total = 0;
    int pitch_a = 0, pitch_b = 0;  // elements per plane row
    int planes = 3;                // planes per operand
    size_t plane_a_elems = 0, plane_b_elems = 0;
    size_t partial_plane_elems = 0;
    int partial_pitch = 0;
    // guard-band offsets from the workspace base (guard bands on only)
    static constexpr int kMaxGuards = 24;
    size_t guard_off[kMaxGuards] = {};
    int guards = 0;
};

struct Problem {
    int transa, transb, m, n, k;
    float ar, ai, br, bi;
    const void* A;
    int lda;
    const void* B;
    int ldb;
    void* C;
    int ldc;
};

cg3mStatus_t validate(int transa, int transb, int m, int n, int k, const cg3mComplex* alpha, const void* A, int lda,
                      const void* B, int ldb, const cg3mComplex* beta, const void* C, int ldc, bool allow_conj_only,
                      int* action);

bool make_plan(const Problem& p, const cg3mOptions& opts, int sm_count, Plan* plan);

// Tensor-map encoding through the driver entry point (no -lcuda needed).
bool encode_tensor_map(CUtensorMap* map, CUtensorMapDataType type, int rank, const uint64_t* dims,
                       const uint64_t* strides_bytes, const uint32_t* box, CUtensorMapSwizzle swizzle,
                       const void* base);

// ---- kernel launchers (return cudaSuccess or the launch error) -------------
cudaError_t launch_beta_scale(cudaStream_t s, int m, int n, float br, float bi, void* C, int ldc);
// band_a / band_b (tensor-core forms' rounding pass): pack only the planes the
// packed rows did not (all but the leading term of re and im), and only for the
// 256-row bands of op(A) rows / op(B) columns whose byte is nonzero.
cudaError_t launch_pack(cudaStream_t s, const Problem& p, const Plan& plan, void* ws, const uint8_t* band_a = nullptr,
                        const uint8_t* band_b = nullptr);
cudaError_t launch_gemm_fp32(cudaStream_t s, const Problem& p, const Plan& plan, void* ws, int* status);
cudaError_t launch_gemm_tc(cudaStream_t s, const Problem& p, const Plan& plan, void* ws, int* status);
cudaError_t launch_merge(cudaStream_t s, const Problem& p, const Plan& plan, void* ws);
// The rounding-correction pass.  Tensor-core forms start the call with the
// packed rows, which also write the leading split planes the risk-plane GEMM
// reads (launch_rounding_pack, instead of the full pack).  Then two halves:
// the preparation reads only op(A) and op(B) (packed rows for the FP32 form,
// energies and, for the tensor-core forms, the residues of the exact
// recompute); the finish needs the GEMM's C and risk plane (FP32: selection,
// then the recomputes; the tensor-core forms' risk-plane GEMM selected in its
// epilogue, and they pack the rest of their planes in the finish, for the
// bands whose tiles the exact recompute leaves to the form).  mark(i) is
// called after the i-th kernel of each half (1-based) is enqueued.
cudaError_t launch_rounding_pack(cudaStream_t s, const Problem& p, const Plan& plan, void* ws,
                                 const std::function<void()>& mark);
// The tensor-core forms' risk-plane GEMM applies the selection in its
// epilogue: these are the selection's inputs and outputs.
struct LeadSelect {
    const float* energy;  // [n] op(A) rows, then [n] op(B) columns
    float bridge, conf2;
    uint32_t* flag_bits;
    uint32_t* tile_count;
    uint32_t* stats;
};
int rounding_prep_kernels(int form);
cudaError_t launch_rounding_prep(cudaStream_t s, const Problem& p, const Plan& plan, void* ws, int* launched,
                                 const std::function<void(int)>& mark);
cudaError_t launch_rounding_finish(cudaStream_t s, const Problem& p, const Plan& plan, void* ws, int* status,
                                   int* launched, const std::function<void(int)>& mark);
// GEMM that also writes the risk plane used by the rounding-correction pass
// (the tensor-core forms: one pass over the leading split planes, whose C the
// pass then replaces everywhere).
cudaError_t launch_gemm_with_path(cudaStream_t s, const Problem& p, const Plan& plan, void* ws, int* status);
// Tensor-core forms in the rounding pass: the form's own products on every
// 256 x 128 pair tile outside the tiles the exact recompute takes (tile_count:
// the pass's per-16 x 16 flagged counts).
cudaError_t launch_gemm_tc_tiles(cudaStream_t s, const Problem& p, const Plan& plan, void* ws, int* status,
                                 const uint32_t* tile_count);
// Rounding pass: a 16 x 16 tile with more flagged outputs than this is
// recomputed as part of a tile; sparser tiles have each flagged output
// recomputed on its own.  Counters it leaves beside the flags:
constexpr uint32_t kSparseMax = 64;
enum : int {
    kStatFlagged = 0,
    kStatDenseOutputs = 1,
    kStatSparseOutputs = 2,
    kStatFallback = 3,
    kStatExactTiles = 4,
    kStatExactOutputs = 5,
    kStatWords = 8
};

// Output rows of the exact recompute's tile; its width is ozaki_tile_n(n).
// It runs on every tile holding a 16 x 16 tile with more than kSparseMax
// flagged outputs.
constexpr int kOzakiTile = 256;
int ozaki_tile_n(int n);

// Exponents, rounding counts, residue planes and product residues of the
// tensor-core forms' exact recompute (ozaki.cu), carved from the rounding
// region.
struct OzLayout {
    int* E = nullptr;            // op(A) row exponents
    int* F = nullptr;            // op(B) column exponents
    int* CA = nullptr;           // rounded parts per op(A) row
    int* CB = nullptr;           // rounded parts per op(B) column
    uint8_t* tile_ran = nullptr; // per exact tile: 1 when it ran
    int8_t* planes_a = nullptr;  // operand residues, [modulus][part][row][kpitch]
    int8_t* planes_b = nullptr;
    uint8_t* residues = nullptr; // product residues, [modulus][part][col / 16][y_pad][16]
    int kpitch = 0;
    size_t plane_bytes = 0;
    int y_pad = 0;               // order rounded up to whole exact tiles
    size_t y_plane = 0;
    size_t bytes = 0;
};
OzLayout oz_layout(int n, uint8_t* base, std::vector<size_t>* guards = nullptr);
// Residues of op(A) rows and op(B) columns (needs only the packed rows).
cudaError_t launch_ozaki_split(cudaStream_t s, int n, int pitch, const float2* rows_a, const float2* rows_b,
                               const OzLayout& L);
// The exact products of every tile holding a dense 16 x 16 tile and their
// reconstruction into every output of those tiles; outputs it cannot certify
// are marked in fallback_bits.  Two launches; mark(i) after the i-th (1-based).
cudaError_t launch_ozaki_tiles(cudaStream_t s, int n, const OzLayout& L, const uint32_t* tile_count, uint32_t* stats, uint32_t* fallback_bits, float2* C,
                               int* status, int* launched, const std::function<void(int)>& mark);
// Bytes of the rounding-correction region for a square problem of order n.
size_t rounding_bytes(int n, int form, std::vector<size_t>* guards = nullptr);
// Device address of the pass's counters (flagged, recomputed as tiles, one by
// one) inside a planned call's workspace.
uint32_t* rounding_stats_ptr(const Plan& plan, void* ws, int n);
cudaError_t launch_zgemm_ref(cudaStream_t s, const Problem& p, const void* Cin, void* out64);
// Diagnostics: one thread waits on an mbarrier nothing arrives on, with the
// given limit; *gave_up (device) becomes 1 when the wait gave up.
cudaError_t launch_wait_probe(cudaStream_t s, int* status, unsigned long long limit_ns, int* gave_up);
// The allocation-free entry point's status word on the current device.
cg3mStatus_t noalloc_status_word(int** word);
// Every device allocation the handle API makes goes through this: it fails
// like cudaMalloc out of memory while a diagnostics failure count is pending.
cudaError_t device_malloc(void** p, size_t bytes);
cudaError_t launch_error_report(cudaStream_t s, int m, int n, const void* C, int ldc, const void* out64,
                                double* dev_report);

// On-chip product family (batched.cu): op() applied while staging the
// caller's interleaved matrices, no pack pass.  mode 0 = standard 3M, 1 = four
// real products; `repair` recomputes non-finite products with explicit FP32
// four-product terms.  One launch covers `batch` problems at element strides
// sA, sB, sC (a single problem is batch 1).
struct StridedPlan {
    int tile = 0, tile_m = 0, tile_n = 0, parts = 1, span = 0, tiles = 0, ppitch = 0;
    size_t partial_stride = 0;  // floats of partials per batch
    size_t counters = 0;        // task counter + tile counters (uint32)
    size_t partial_off = 0;     // byte offset of the partials in the workspace
    size_t bytes = 0;           // workspace bytes
};
bool make_strided_plan(const Problem& p, int mode, int batch, int sm_count, StridedPlan* out);
// One problem in one launch of the on-chip family: grid (tiles, parts), the
// `parts` K partitions of a tile merged through its thread-block cluster
// (parts <= 8, and (parts - 1) * span < k).  tile: 0 128x64, 1 64x64,
// 2 128x32, 3 32x128, 4 64x32, 5 32x32.  No workspace.
cudaError_t launch_single(cudaStream_t s, const Problem& p, int mode, int repair, int tile, int parts);
// The one-launch plan for an m x n x k problem in `mode`: tile and K
// partitions (each forced when >= 0), chosen to minimise the estimated time,
// which is returned in microseconds.
double plan_single(int m, int n, int k, int mode, int sm_count, int forced_tile, int forced_parts, int* tile,
                   int* parts);
int single_tile_bm(int tile);
int single_tile_bn(int tile);
cudaError_t launch_strided(cudaStream_t s, const Problem& p, int mode, int repair, long long sA, long long sB,
                           long long sC, int batch, const StridedPlan& plan, void* ws, int sm_count);

// Enqueue a fully planned call (pack + GEMM [+ merge] [+ rounding]); when
// `events` is non-null, kernel j (in the order the call info names them) is
// bracketed by events[2j] and events[2j + 1], recorded on the stream it runs
// on (entries past nevents are skipped).
cudaError_t enqueue(cudaStream_t s, const Problem& p, const Plan& plan, void* ws, int* status, int* kernels,
                    const cudaEvent_t* events = nullptr, int nevents = 0);

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Guard bands (diagnostics, the memory-safety check of the test suite): with
// CG3M_GUARD_BANDS set in the environment when the library loads, every
// workspace region is followed by kGuardBytes of a fixed byte pattern that
// each call fills before its first kernel and checks after its last
// (cg3mDiagGuardStatus reports a damaged band).  Off by default: no bands.
constexpr size_t kGuardBytes = 4096;
constexpr unsigned char kGuardByte = 0xA5;
bool guard_bands_on();
// End of a region of `bytes` bytes starting at `off`: aligned to kRegionAlign
// and, with guard bands on, followed by a band whose offset goes to *guards.
inline size_t next_region(size_t off, size_t bytes, std::vector<size_t>* guards)
{
    size_t end = align_up(off + bytes, kRegionAlign);
    if (bytes != 0 && guard_bands_on()) {
        if (guards != nullptr) {
            guards->push_back(end);
        }
        end += kGuardBytes;
    }
    return end;
}
// Fills (before) and checks (after) a call's guard bands on stream s.
cudaError_t fill_guards(cudaStream_t s, void* ws, const size_t* offs, int count);
cudaError_t check_guards(cudaStream_t s, const void* ws, const size_t* offs, int count);
// Synchronizes the device, returns and clears the damaged-band flag.
cudaError_t read_guard_damage(int* damaged);
inline int ceil_div(int a, int b) { return (a + b - 1) / b; }

}  // namespace cg3m
