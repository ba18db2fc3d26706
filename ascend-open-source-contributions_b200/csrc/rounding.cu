// rounding.cu -- the rounding-correction pass.
//
// Reference: gemm_cgemm3m_rounding_do, blas/gemm/arch35/cgemm3m_rounding_kernel.cpp
// :474-497, run after the path-tracking GEMM when the call is a contiguous
// square unit-output product of order 2048..4096 (cgemm_host.cpp:234-238):
//   1. pack (:148-190)      op(A) rows and op(B) columns as contiguous complex
//                           K vectors (conjugation applied);
//   2. permute (:406-472)   per-row energies sum |x|^2, accumulated per lane of
//                           a 64-lane segment layout (lane l holds k in
//                           [l*span, (l+1)*span), span = ceil(n/64) | 1) and
//                           reduced across lanes;
//   3. select (:43-130)     flag output (i,j) when max(|Re|,|Im|) or
//                           var = 2^-48 (path + E_i E_j bridge) is not finite,
//                           or 3.75^2 var >= 1e-4; the reference compacts
//                           flagged indices into per-core lists;
//   4. recompute (:192-404) each flagged output again, in a fixed order.
// B200 design: one CTA of 64 threads per row for the energies (the row is
// staged in shared memory; span is odd so the strided lane reads are
// conflict-free); a grid-stride select in which each warp writes one 32-bit
// word of the flag bitmap (its ballot) and adds its flags to a count per
// 16 x 16 output tile.  The recompute then splits by density, on the device,
// from those counts: a tile with more than kSparseMax flagged outputs is
// recomputed as a tile (operands staged once for all its outputs), every other
// flagged output on its own by a 64-thread block (recompute_sparse), so a
// handful of flags no longer costs a whole tile.  FP32 form: the reference's
// segmented replay, bit for bit -- over 16 x 16 tiles with 2 x 2 outputs per
// thread for 8 of the 64 lanes, or one lane per thread for a single output.
// Tensor-core forms: every output of a 256 x 256 tile holding a dense 16 x 16
// tile comes back within one FP32 rounding of the exact product -- exact int8
// products by residues on the tensor cores (ozaki.cu), FP64 for the few
// outputs their bound cannot certify -- and the other tiles get the form's
// own products, their flagged outputs recomputed in FP64 one by one.
#include <cstring>
#include <functional>

#include "cg3m_internal.h"
#include "ptx.cuh"

namespace cg3m {

cudaError_t launch_pack_rows(cudaStream_t stream, const Problem& p, void* rows_a, void* rows_b, int pitch,
                             const Plan* lead_plan = nullptr, void* ws = nullptr);
cudaError_t launch_gemm_fp32_path(cudaStream_t stream, const Problem& pr, const Plan& plan, void* ws, float* path,
                                  int* status);
cudaError_t launch_gemm_tc_path(cudaStream_t stream, const Problem& pr, const Plan& plan, void* ws,
                                const LeadSelect& sel, int* status);

namespace {

constexpr int kLanes = 64;
constexpr int kTile = 16;             // flag granule: 16 x 16 outputs
constexpr int kMaxSpan = 65;          // ceil(4096/64) | 1
constexpr float kConfidence = 3.75f;  // CGEMM_ROUNDING_CONFIDENCE, cgemm_host.cpp:37

// ---- 2. energies ----------------------------------------------------------------

__global__ void __launch_bounds__(kLanes) energy_kernel(const float2* __restrict__ rows_a,
                                                        const float2* __restrict__ rows_b, int n, int pitch,
                                                        int span, float* __restrict__ energy)
{
    __shared__ float lanes[kLanes];
    const int r = blockIdx.x;
    const float2* src = r < n ? rows_a + (size_t)r * pitch : rows_b + (size_t)(r - n) * pitch;
    // Each lane reads its own span of consecutive terms straight from global
    // memory (no staged row, so many rows are in flight per SM); the sector a
    // thread fetches serves its next terms from L1.
    const int l = threadIdx.x;
    float e = 0.0f;
    const int k0 = l * span, k1 = min(n, k0 + span);
    for (int k = k0; k < k1; ++k) {
        const float2 x = __ldg(src + k);
        e = __fmaf_rn(x.x, x.x, e);
        e = __fmaf_rn(x.y, x.y, e);
    }
    lanes[l] = e;
    __syncthreads();
    for (int stride = kLanes / 2; stride >= 1; stride /= 2) {
        if (l < stride) {
            lanes[l] = __fadd_rn(lanes[l], lanes[l + stride]);
        }
        __syncthreads();
    }
    if (l == 0) {
        energy[r] = lanes[0];
    }
}

// ---- 3. selection -----------------------------------------------------------------

// One warp handles 32 consecutive outputs (idx = j*n + i) per step, so each
// 32-bit word of the flag bitmap is the warp's ballot and is stored whole (no
// memset, no atomics); flagged outputs are counted per 16 x 16 tile (the
// warp's lanes of one tile add their count once) and in total.
__global__ void select_kernel(int n, const float2* __restrict__ C, const float* __restrict__ energy,
                              const float* __restrict__ path, float bridge, uint32_t* __restrict__ flag_bits,
                              uint32_t* __restrict__ tile_count, uint32_t* __restrict__ stats)
{
    // n <= 4096 (the gate), so output indices fit 32 bits.  Each warp takes
    // kGroups consecutive 32-output words per trip and issues all their loads
    // before any ballot, so several words' memory latency overlaps.
    constexpr int kGroups = 4;
    const uint32_t total = (uint32_t)n * (uint32_t)n;
    const uint32_t un = (uint32_t)n;
    const int tiles = (n + kTile - 1) / kTile;
    const float conf2 = __fmul_rn(kConfidence, kConfidence);
    const int lane = threadIdx.x & 31;
    uint32_t local = 0;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t base = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32 * kGroups; base < total;
         base += warps * 32 * kGroups) {
        float2 c[kGroups];
        float pth[kGroups], ei[kGroups], ej[kGroups];
        uint32_t ii[kGroups], jj[kGroups];
#pragma unroll
        for (int g = 0; g < kGroups; ++g) {
            const uint32_t idx = base + g * 32 + lane;
            if (idx < total) {
                jj[g] = idx / un;
                ii[g] = idx - jj[g] * un;
                c[g] = C[idx];
                pth[g] = path[idx];
                ei[g] = energy[ii[g]];
                ej[g] = energy[n + jj[g]];
            }
        }
#pragma unroll
        for (int g = 0; g < kGroups; ++g) {
            const uint32_t wbase = base + g * 32;
            if (wbase >= total) {
                break;  // warp-uniform
            }
            const uint32_t idx = wbase + lane;
            bool sel = false;
            int tile = -1;
            if (idx < total) {
                const float re = fabsf(c[g].x), im = fabsf(c[g].y);
                const float magnitude = re > im ? re : im;
                const float variance = __fmul_rn(0x1p-48f, __fadd_rn(pth[g], __fmul_rn(__fmul_rn(ei[g], ej[g]), bridge)));
                sel = !isfinite(magnitude) || !isfinite(variance) || __fmul_rn(conf2, variance) >= 0.0001f;
                tile = (int)(jj[g] / kTile) * tiles + (int)(ii[g] / kTile);
            }
            const uint32_t word = __ballot_sync(0xffffffffu, sel);
            if (lane == 0) {
                flag_bits[wbase >> 5] = word;
            }
            const uint32_t peers = __match_any_sync(0xffffffffu, sel ? tile : -1);
            if (sel && lane == __ffs(peers) - 1) {
                atomicAdd(&tile_count[tile], (uint32_t)__popc(peers));
            }
            local += sel ? 1u : 0u;
        }
    }
    local = __reduce_add_sync(0xffffffffu, local);
    if (lane == 0 && local != 0) {
        atomicAdd(&stats[kStatFlagged], local);
    }
}

// Per 256 x 256 tile (blockIdx.x: op(A) row band, blockIdx.y: op(B) column
// band): when none of its 16 x 16 count tiles holds more than kSparseMax
// flagged outputs (the exact recompute's and the pair kernel's own test), the
// form's products run there and read that row band of op(A) and column band
// of op(B), so both bands are marked for the rest of the pack.
static_assert(kOzakiTile / kTile == 16, "16 x 16 count tiles per exact tile");
__global__ void __launch_bounds__(256) band_need_kernel(int n, const uint32_t* __restrict__ tile_count,
                                                         uint8_t* __restrict__ band_a, uint8_t* __restrict__ band_b)
{
    const int g16 = (n + kTile - 1) / kTile;
    const int gi = blockIdx.x * 16 + threadIdx.x % 16;
    const int gj = blockIdx.y * 16 + threadIdx.x / 16;
    const bool dense = gi < g16 && gj < g16 && tile_count[(size_t)gj * g16 + gi] > kSparseMax;
    if (!__syncthreads_or(dense) && threadIdx.x == 0) {
        band_a[blockIdx.x] = 1;
        band_b[blockIdx.y] = 1;
    }
}

__device__ __forceinline__ bool flagged(const uint32_t* bits, size_t idx)
{
    return (bits[idx >> 5] >> (idx & 31)) & 1u;
}

// ---- 4a. FP32 segmented replay (FastSegmentDot) ---------------------------------------

// FP32 segmented replay of one 16 x 16 output tile with 512 threads.  Warps
// 2g and 2g + 1 hold the K lanes 8g .. 8g + 7 (lane l holds k in
// [l*span, (l+1)*span)); each of their threads owns the 2 x 2 outputs of one
// micro-tile (rows mr, mr + 8, columns 2*mc, 2*mc + 1).  So every op(A) and
// op(B) value a thread loads from shared memory feeds two outputs, and the
// operand sums of the fused identity (xr + xi, yi - yr, yr + yi) are formed
// once per load rather than once per output.  A lane is walked in kChunks
// chunks of ch = ceil(span / kChunks) terms.  One step stages chunk c of lane
// 8g + s for all eight groups: one thread issues two 2-D tensor copies per
// group (16 rows of op(A), 16 of op(B), w columns from the even K offset at or
// below the chunk's start), completing on the buffer's mbarrier, while the
// block sums the previous step.  The 64 lane sums of each output sit in shared
// memory (S[l][output]); one thread per output and part (real or imaginary)
// computes the direct reduction, the inclusive scan and the final selection
// with the 64 values in registers, and the groups replay their lanes seeded
// with the scanned prefixes -- all in the oracle's fixed orders, with each
// output's K terms of a lane added one at a time in increasing k.  Only
// flagged outputs are written.
constexpr int kGroups = 8;                                   // lane groups, two warps each
constexpr int kGroupLanes = kLanes / kGroups;                // 8 lanes per group
constexpr int kChunks = 4;                                   // chunks per lane
constexpr int kChunk = (kMaxSpan + kChunks - 1) / kChunks;   // 17: the longest chunk (n = 4096)
constexpr int kChunkMin = (((2048 + kLanes - 1) / kLanes | 1) + kChunks - 1) / kChunks;  // 9: n = 2048
constexpr int kSteps = kGroupLanes * kChunks;                // 32 staging steps per pass
constexpr int kBoxMax = 18;                                  // widest staged row (float2)
constexpr size_t kLaneSumBytes = (size_t)2 * kLanes * 256 * sizeof(float);
constexpr size_t kBoxElems = (size_t)kTile * kBoxMax;               // float2 per staged box
constexpr size_t kBufElems = (size_t)kGroups * 2 * kBoxElems;       // float2 per staging buffer
constexpr size_t kRecomputeSmem = 128 + kLaneSumBytes + 2 * kBufElems * sizeof(float2) + 2 * sizeof(uint64_t);
constexpr int kBand = 16;                                           // tile rows per band of the launch order
static_assert(kBoxElems * sizeof(float2) % 128 == 0, "staged boxes start on 128-byte boundaries");

// Staged row width for chunks of ch terms: at least ch + 1 (the copy starts at
// the even K offset at or below the chunk's start), even (16-byte rows) and
// 2 mod 4, so the 8 rows (or 4 columns) a warp reads at one K offset fall in
// distinct shared-memory bank pairs.
constexpr int box_width(int ch)
{
    int w = ch + 1;
    while (w % 4 != 2) {
        ++w;
    }
    return w;
}

// One term at K offset q for the 2 x 2 outputs: X0, X1 are the two op(A) rows,
// Y0, Y1 the two op(B) columns, all at the chunk's first term.  Output (a, b)
// is acc[a + 2b].  The term is the fused identity of ThreeProductTerms
// (:192-208): p = (xr + xi) yr, re = p - xi (yr + yi), im = p + xr (yi - yr).
__device__ __forceinline__ void replay_term(const float2* X0, const float2* X1, const float2* Y0, const float2* Y1,
                                            int q, float2* acc)
{
    const float2 x0 = X0[q], x1 = X1[q];
    const float2 y0 = Y0[q], y1 = Y1[q];
    const float sx[2] = {__fadd_rn(x0.x, x0.y), __fadd_rn(x1.x, x1.y)};
    const float dy[2] = {__fsub_rn(y0.y, y0.x), __fsub_rn(y1.y, y1.x)};
    const float ey[2] = {__fadd_rn(y0.x, y0.y), __fadd_rn(y1.x, y1.y)};
    const float xr[2] = {x0.x, x1.x}, xi[2] = {x0.y, x1.y}, yr[2] = {y0.x, y1.x};
#pragma unroll
    for (int b = 0; b < 2; ++b) {
#pragma unroll
        for (int a = 0; a < 2; ++a) {
            const float p = __fmul_rn(sx[a], yr[b]);
            const float qq = __fmul_rn(xr[a], dy[b]);
            const float rr = __fmul_rn(xi[a], ey[b]);
            // (re, im) of the term, added to the output's (re, im) by one
            // packed add: two independent round-to-nearest adds of sums, no
            // product feeds it.
            acc[a + 2 * b] = __fadd2_rn(acc[a + 2 * b], make_float2(__fsub_rn(p, rr), __fadd_rn(p, qq)));
        }
    }
}

// Terms [0, len) of one staged chunk, in increasing K: a full chunk (len = CH)
// as one straight-line block, a shorter one (the last chunk of a lane) as a
// loop.
template <int CH>
__device__ __forceinline__ void replay_chunk(const float2* X0, const float2* X1, const float2* Y0,
                                             const float2* Y1, int len, float2* acc)
{
    if (len == CH) {
#pragma unroll
        for (int q = 0; q < CH; ++q) {
            replay_term(X0, X1, Y0, Y1, q, acc);
        }
    } else {
#pragma unroll 4
        for (int q = 0; q < len; ++q) {
            replay_term(X0, X1, Y0, Y1, q, acc);
        }
    }
}

// One instance per chunk length CH = ceil(span / kChunks) (9 at n = 2048 .. 17
// at n = 4096), so the box width and the full-chunk loop are constants.
template <int CH>
__global__ void __launch_bounds__(512) recompute_fp32_tiled(const __grid_constant__ CUtensorMap tm_a,
                                                            const __grid_constant__ CUtensorMap tm_b, int n,
                                                            int span, const uint32_t* __restrict__ flag_bits,
                                                            const uint32_t* __restrict__ tile_count,
                                                            uint32_t* __restrict__ stats, float2* __restrict__ C,
                                                            int* status)
{
    constexpr int ch = CH;
    constexpr int w = box_width(CH);
    extern __shared__ uint8_t replay_smem[];
    uint8_t* base = align_shared<128>(replay_smem);
    // Lane sums, real then imaginary: S[l][o] for output o = ti + 16 tj of the tile.
    float* sr = reinterpret_cast<float*>(base);
    float* si = sr + kLanes * 256;
    float2* stage = reinterpret_cast<float2*>(base + kLaneSumBytes);
    uint64_t* full = reinterpret_cast<uint64_t*>(stage + 2 * kBufElems);
    // Tiles run in bands of kBand tile rows, rows fastest within a band: the
    // op(A) rows of a band stay in L2 while its columns go by, so op(A) is read
    // from DRAM about once and op(B) once per band.
    const int tiles = (n + kTile - 1) / kTile;
    const int band = blockIdx.x / (kBand * tiles), first = band * kBand;
    const int rows_in_band = min(kBand, tiles - first), in_band = blockIdx.x - band * kBand * tiles;
    const int ti_tile = first + in_band % rows_in_band, tj_tile = in_band / rows_in_band;
    const uint32_t tile_flagged = tile_count[(size_t)tj_tile * tiles + ti_tile];
    if (tile_flagged <= kSparseMax) {
        return;  // no flags, or few enough for the per-output kernel
    }
    const int i0 = ti_tile * kTile, j0 = tj_tile * kTile;
    const int tid = threadIdx.x;
    if (tid == 0) {
        atomicAdd(&stats[kStatDenseOutputs], tile_flagged);
    }
    auto lane_count = [&](int l) { return max(0, min(span, n - l * span)); };
    auto chunk_len = [&](int l, int c) { return max(0, min(ch, lane_count(l) - c * ch)); };

    // Compute role: group g = warp / 2; the warp's 32 micro-tiles cover all 16
    // rows (mr = lane % 8, rows mr and mr + 8) and 8 of the 16 columns, so one
    // operand load of a warp touches 8 distinct op(A) rows or 4 distinct op(B)
    // columns.
    const int warp = tid >> 5, wl = tid & 31;
    const int g = warp >> 1;
    const int mr = wl & 7, cb = 2 * (((warp & 1) << 2) | (wl >> 3));
    int out[4];  // o of output (a, b) at out[a + 2b]
#pragma unroll
    for (int b = 0; b < 2; ++b) {
#pragma unroll
        for (int a = 0; a < 2; ++a) {
            out[a + 2 * b] = (mr + 8 * a) + kTile * (cb + b);
        }
    }

    // Staging: thread 0 arms buffer T % 2 with the step's bytes and issues, per
    // group, the op(A) box (rows i0 .., x) and the op(B) box (rows j0 .., x),
    // x = the chunk's K start rounded down to even.  Boxes past the matrix or
    // past K read as zero.  T counts steps over both passes: buffer T % 2,
    // phase parity (T / 2) % 2.
    const uint32_t step_bytes = (uint32_t)(kGroups * 2 * kTile * w * sizeof(float2));
    if (tid == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        fence_mbar_init();
        tma_prefetch_desc(&tm_a);
        tma_prefetch_desc(&tm_b);
    }
    __syncthreads();
    auto issue = [&](int T) {
        if (tid == 0) {
            const int t = T % kSteps, b = T & 1;
            mbar_arrive_expect_tx(&full[b], step_bytes);
#pragma unroll 1
            for (int gg = 0; gg < kGroups; ++gg) {
                const int l = kGroupLanes * gg + t / kChunks;
                const int x = (l * span + (t % kChunks) * ch) & ~1;
                float2* dst = stage + (size_t)b * kBufElems + (size_t)(gg * 2) * kBoxElems;
                tma_load_2d(dst, &tm_a, &full[b], x, i0);
                tma_load_2d(dst + kBoxElems, &tm_b, &full[b], x, j0);
            }
        }
    };
    // Bounded waits: a thread whose wait gave up (status flagged) stops
    // waiting and runs on, so the block ends; the call's result is then
    // reported as failed.
    bool ok = true;
    auto wait_step = [&](int T) {
        if (ok) {
            ok = mbar_wait(&full[T & 1], (uint32_t)((T >> 1) & 1), status);
        }
    };
    // Operand pointers of this thread's rows and columns in buffer b for the
    // step's lane l and chunk c (the copy started at an even K offset).
    auto chunk_ptrs = [&](int T, int l, int c, const float2** xp) {
        const int off = (l * span + c * ch) & 1;
        const float2* a = stage + (size_t)(T & 1) * kBufElems + (size_t)(g * 2) * kBoxElems + off;
        const float2* bb = a + kBoxElems;
        xp[0] = a + mr * w;
        xp[1] = a + (mr + 8) * w;
        xp[2] = bb + cb * w;
        xp[3] = bb + (cb + 1) * w;
    };

    // pass 1: lane sums (the next step's boxes are copied while this one is summed)
    float2 acc[4];  // (re, im) of output (a, b) at acc[a + 2b]
    issue(0);
    for (int t = 0; t < kSteps; ++t) {
        __syncthreads();  // every thread is done with the previous step's buffer
        if (t + 1 < kSteps) {
            issue(t + 1);
        }
        wait_step(t);
        const int l = kGroupLanes * g + t / kChunks, c = t % kChunks;
        if (c == 0) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                acc[u] = make_float2(0.0f, 0.0f);
            }
        }
        const float2* xp[4];
        chunk_ptrs(t, l, c, xp);
        replay_chunk<CH>(xp[0], xp[1], xp[2], xp[3], chunk_len(l, c), acc);
        if (c == kChunks - 1) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                sr[l * 256 + out[u]] = acc[u].x;
                si[l * 256 + out[u]] = acc[u].y;
            }
        }
    }
    __syncthreads();  // all 64 lane sums of every output are in place
    // Lane reductions and the scan: thread t takes the real (t < 256) or the
    // imaginary part of output o = t % 256, with its 64 lane values in
    // registers.
    const int o = tid & 255;
    float* const part = tid < 256 ? sr : si;
    float direct, peak = 0.0f;
    {
        float v[kLanes];
#pragma unroll
        for (int l = 0; l < kLanes; ++l) {
            v[l] = part[l * 256 + o];
        }
        // direct reduction (pairwise, stride 32 .. 1)
#pragma unroll
        for (int stride = kLanes / 2; stride >= 1; stride /= 2) {
#pragma unroll
            for (int l = 0; l < stride; ++l) {
                v[l] = __fadd_rn(v[l], v[l + stride]);
            }
        }
        direct = v[0];
#pragma unroll
        for (int l = 0; l < kLanes; ++l) {
            v[l] = part[l * 256 + o];
        }
        // inclusive Hillis-Steele scan in place: new[l] = s[l] + s[l-d] for l >= d
#pragma unroll
        for (int d = 1; d < kLanes; d *= 2) {
#pragma unroll
            for (int l = kLanes - 1; l >= d; --l) {
                v[l] = __fadd_rn(v[l], v[l - d]);
            }
        }
#pragma unroll
        for (int l = 0; l < kLanes; ++l) {
            const float a = fabsf(v[l]);
            peak = a > peak ? a : peak;
            part[l * 256 + o] = v[l];
        }
    }
    __syncthreads();  // scanned prefixes in place; every thread is done with the last buffer
    // pass 2: replay each lane seeded with the previous lane's prefix.  Group g
    // starts from the prefix of lane 8g - 1, read here, before group g - 1
    // overwrites it at the last step; each lane's own prefix is read at the
    // lane's first chunk, before its replayed value replaces it.
    float prev_r[4], prev_i[4], init_r[4], init_i[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        prev_r[u] = g == 0 ? 0.0f : sr[(kGroupLanes * g - 1) * 256 + out[u]];
        prev_i[u] = g == 0 ? 0.0f : si[(kGroupLanes * g - 1) * 256 + out[u]];
        init_r[u] = 0.0f;
        init_i[u] = 0.0f;
    }
    issue(kSteps);
    for (int t = 0; t < kSteps; ++t) {
        const int T = kSteps + t;
        __syncthreads();
        if (t + 1 < kSteps) {
            issue(T + 1);
        }
        wait_step(T);
        const int l = kGroupLanes * g + t / kChunks, c = t % kChunks;
        if (c == 0) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                init_r[u] = prev_r[u];
                init_i[u] = prev_i[u];
                prev_r[u] = sr[l * 256 + out[u]];
                prev_i[u] = si[l * 256 + out[u]];
                acc[u] = make_float2(__fadd_rn(init_r[u], 0.0f), __fadd_rn(init_i[u], 0.0f));
            }
        }
        const float2* xp[4];
        chunk_ptrs(T, l, c, xp);
        replay_chunk<CH>(xp[0], xp[1], xp[2], xp[3], chunk_len(l, c), acc);
        if (c == kChunks - 1) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                sr[l * 256 + out[u]] = __fsub_rn(acc[u].x, init_r[u]);
                si[l * 256 + out[u]] = __fsub_rn(acc[u].y, init_i[u]);
            }
        }
    }
    __syncthreads();  // every replayed lane is in place
    {
        float v[kLanes];
#pragma unroll
        for (int l = 0; l < kLanes; ++l) {
            v[l] = part[l * 256 + o];
        }
#pragma unroll
        for (int stride = kLanes / 2; stride >= 1; stride /= 2) {
#pragma unroll
            for (int l = 0; l < stride; ++l) {
                v[l] = __fadd_rn(v[l], v[l + stride]);
            }
        }
        float bridged = v[0];
        if (peak >= __fmul_rn(fabsf(direct), 32.0f)) {
            bridged = direct;
        }
        const int i = i0 + (o & (kTile - 1)), j = j0 + o / kTile;
        if (i < n && j < n) {
            const size_t idx = (size_t)j * n + i;
            if (flagged(flag_bits, idx)) {
                reinterpret_cast<float*>(C)[2 * idx + (tid < 256 ? 0 : 1)] = bridged;
            }
        }
    }
    // A block in which a wait gave up drains its last copies (bounded) before
    // it exits, so no copy lands in shared memory after the block is gone.
    if (__syncthreads_or(!ok) && tid == 0) {
        mbar_wait(&full[0], (uint32_t)(((2 * kSteps - 2) >> 1) & 1), status);
        mbar_wait(&full[1], (uint32_t)(((2 * kSteps - 1) >> 1) & 1), status);
    }
}

// ---- 4b. lane-major copies for the per-output recompute ---------------------------

// Lane-major copies of the packed op(A) rows and op(B) columns, the layout of
// the reference's PermuteSegments (cgemm3m_rounding_kernel.cpp:406-435):
// element k = l * span + s of a row goes to s * 64 + l (zero past n), so the
// 64 lanes of one K step are 512 contiguous bytes.  One block per row: the
// row is staged with coalesced loads and written out coalesced (span is odd,
// so the strided shared-memory reads of a half-warp hit distinct banks).
__global__ void __launch_bounds__(256) lane_major_kernel(int n, int pitch, int span, const float2* __restrict__ rows_a,
                                                         const float2* __restrict__ rows_b,
                                                         float2* __restrict__ lanes_a, float2* __restrict__ lanes_b,
                                                         const uint8_t* __restrict__ need)
{
    extern __shared__ float2 row[];
    const int r = blockIdx.x;
    if (!need[r]) {
        return;  // no output the per-output kernels recompute lies in this row or column
    }
    const size_t width = (size_t)kLanes * span;
    const float2* src = r < n ? rows_a + (size_t)r * pitch : rows_b + (size_t)(r - n) * pitch;
    float2* dst = r < n ? lanes_a + (size_t)r * width : lanes_b + (size_t)(r - n) * width;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        row[k] = src[k];
    }
    __syncthreads();
    for (int f = threadIdx.x; f < (int)width; f += blockDim.x) {
        const int sidx = f / kLanes, l = f % kLanes;
        const int k = l * span + sidx;
        dst[f] = k < n ? row[k] : make_float2(0.0f, 0.0f);
    }
}

// The op(A) rows (need[i]) and op(B) columns (need[n + j]) of the outputs the
// per-output kernels recompute: flagged outputs of 16 x 16 tiles the tile
// kernels leave (FP32: tiles with at most kSparseMax flagged outputs;
// tensor-core forms: outside the 256 x 256 tiles the exact recompute took),
// and, for the tensor-core forms, the outputs it marked for the FP64 fallback.
// need[] starts zeroed; only those rows and columns get lane-major copies.
__global__ void __launch_bounds__(256) lanes_needed_kernel(int n, int tc, const uint32_t* __restrict__ flag_bits,
                                                           const uint32_t* __restrict__ fallback_bits,
                                                           const uint32_t* __restrict__ tile_count,
                                                           const uint8_t* __restrict__ tile_ran, int exact_tiles,
                                                           uint8_t* __restrict__ need)
{
    const size_t words = ((size_t)n * n + 31) / 32;
    const int tiles16 = (n + kTile - 1) / kTile;
    for (size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x; w < words; w += (size_t)gridDim.x * blockDim.x) {
        const uint32_t fb = tc ? fallback_bits[w] : 0u;
        uint32_t bits = flag_bits[w] | fb;
        // Fast path: a word inside one column and one tile row band whose tile
        // kernels take all its flags leaves only its fallback bits.
        const size_t first = w * 32, last = min(first + 31, (size_t)n * n - 1);
        const int j0 = (int)(first / n), j1 = (int)(last / n);
        if (bits != 0 && j0 == j1) {
            const int i0 = (int)(first - (size_t)j0 * n), i1 = (int)(last - (size_t)j1 * n);
            if (tc) {
                if (i0 / kOzakiTile == i1 / kOzakiTile &&
                    tile_ran[(size_t)(j0 / kOzakiTile) * exact_tiles + i0 / kOzakiTile]) {
                    bits = fb;
                }
            } else {
                const size_t t = (size_t)(j0 / kTile) * tiles16;
                if (tile_count[t + i0 / kTile] > kSparseMax && tile_count[t + i1 / kTile] > kSparseMax &&
                    i1 / kTile - i0 / kTile <= 1) {
                    bits = 0;
                }
            }
        }
        while (bits != 0) {
            const int b = __ffs(bits) - 1;
            bits &= bits - 1;
            const size_t idx = w * 32 + (size_t)b;
            if (idx >= (size_t)n * n) {
                break;  // bits past the last output are never set; bounds need[] all the same
            }
            const int j = (int)(idx / n), i = (int)(idx - (size_t)j * n);
            bool want = (fb >> b) & 1u;
            if (!want) {
                want = tc ? !tile_ran[(size_t)(j / kOzakiTile) * exact_tiles + i / kOzakiTile]
                          : tile_count[(size_t)(j / kTile) * tiles16 + i / kTile] <= kSparseMax;
            }
            if (want) {
                need[i] = 1;
                need[n + j] = 1;
            }
        }
    }
}

// ---- 4c. per-output recompute of sparse tiles ----------------------------------

// Whether the exact (int8 residue) recompute tile holding 16 x 16 tile (gi, gj)
// runs, i.e. holds a dense 16 x 16 tile (ozaki_pair_kernel's predicate).
__device__ __forceinline__ bool ozaki_tile_dense(const uint32_t* tile_count, int tiles16, int gi, int gj, int gn)
{
    constexpr int G = kOzakiTile / kTile;  // count tiles down the exact tile; gn across it
    const int bi = gi / G * G, bj = gj / gn * gn;
    bool dense = false;
    for (int q = 0; q < G * gn; ++q) {
        const int qi = bi + q % G, qj = bj + q / G;
        if (qi < tiles16 && qj < tiles16) {
            dense |= tile_count[qj * tiles16 + qi] > kSparseMax;
        }
    }
    return dense;
}

// Per-output recompute, one block of 64 threads per 16 x 16 output tile.
//   kSparseFp32 / kSparseFp64: tiles holding between 1 and kSparseMax
//     flagged outputs (FP64: outside every tile the exact recompute takes);
//   kFallbackFp64: the outputs the exact recompute marked in `bits` (a
//     non-finite operand, or a result it could not certify).
// The tile's outputs are recomputed one after another, each from the
// lane-major copies of its op(A) row and op(B) column:
//   FP32 (FastSegmentDot, cgemm3m_rounding_kernel.cpp:264-309): thread l is
//     K lane l (k in [l*span, (l+1)*span)); its direct sum, the pairwise lane
//     reduction, the inclusive Hillis-Steele scan, the replay seeded with the
//     previous lane's prefix and the 32x fallback follow the oracle's order
//     exactly (one rounding per operation, no contraction);
//   FP64: thread l sums the same lane's complex products in FP64, the lane
//     sums are reduced in FP64 and the result is rounded once to FP32.
enum { kSparseFp32 = 0, kSparseFp64 = 1, kFallbackFp64 = 2 };

template <int MODE>
__global__ void __launch_bounds__(kLanes) recompute_sparse(int n, int span,
                                                          const float2* __restrict__ lanes_a,
                                                          const float2* __restrict__ lanes_b,
                                                          const uint32_t* __restrict__ bits,
                                                          const uint32_t* __restrict__ tile_count,
                                                          uint32_t* __restrict__ stats, float2* __restrict__ C,
                                                          int exact_gn)
{
    constexpr bool FP64 = MODE != kSparseFp32;
    __shared__ float sr[kLanes], si[kLanes], tr[kLanes], ti[kLanes];
    __shared__ double dr[kLanes], di[kLanes];
    __shared__ int list[kTile * kTile];
    __shared__ int listed;
    __shared__ float peak_r[2], peak_i[2];
    // Tiles in bands of kSparseBand tile rows, rows fastest within a band: the
    // op(A) rows of a band (1024 rows, 32 MB at n = 4096) stay in L2 while the
    // band's columns go by, so each staged row comes from L2, not HBM.
    constexpr int kSparseBand = 64;
    const int tiles = (n + kTile - 1) / kTile;
    const int band = blockIdx.x / (kSparseBand * tiles), first = band * kSparseBand;
    const int rows_in_band = min(kSparseBand, tiles - first), in_band = blockIdx.x - band * kSparseBand * tiles;
    const int gi = first + in_band % rows_in_band, gj = in_band / rows_in_band;
    const uint32_t count = tile_count[(size_t)gj * tiles + gi];
    if (count == 0) {
        return;
    }
    if (MODE != kFallbackFp64 && count > kSparseMax) {
        return;
    }
    const int l = threadIdx.x;
    const int i0 = gi * kTile, j0 = gj * kTile;
    if (MODE == kFallbackFp64) {
        // Fallback bits are only ever set inside the exact recompute's tiles:
        // look at this tile's bits first (one or two words per column).
        bool any = false;
        if (l < kTile && j0 + l < n) {
            const size_t first = (size_t)(j0 + l) * n + i0, last = first + min(kTile, n - i0) - 1;
            for (size_t w = first >> 5; w <= (last >> 5); ++w) {
                any |= bits[w] != 0u;
            }
        }
        if (!__syncthreads_or(any)) {
            return;
        }
    }
    // The exact recompute writes (or marks) every flagged output of its tiles.
    if (MODE == kSparseFp64 && ozaki_tile_dense(tile_count, tiles, gi, gj, exact_gn)) {
        return;
    }
    if (l == 0) {
        listed = 0;
    }
    __syncthreads();
    for (int o = l; o < kTile * kTile; o += kLanes) {
        const int i = i0 + o % kTile, j = j0 + o / kTile;
        if (i < n && j < n && flagged(bits, (size_t)j * n + i)) {
            list[atomicAdd(&listed, 1)] = o;
        }
    }
    __syncthreads();
    const int outputs = listed;
    if (outputs == 0) {
        return;
    }
    if (l == 0 && MODE != kFallbackFp64) {
        atomicAdd(&stats[kStatSparseOutputs], (uint32_t)outputs);
    }
    // Lane l's terms, read from the lane-major copies (element s of lane l at
    // s * 64 + l): every warp load is 256 contiguous bytes, and no shared
    // memory is staged, so many blocks share an SM.
    const int kbeg = min(n, l * span), cnt = min(n, kbeg + span) - kbeg;
    for (int u = 0; u < outputs; ++u) {
        const int o = list[u];
        const int i = i0 + o % kTile, j = j0 + o / kTile;
        const float2* X = lanes_a + (size_t)i * (kLanes * span) + l;
        const float2* Y = lanes_b + (size_t)j * (kLanes * span) + l;
        // Lane l's own terms; the 64 lane values then meet in warp 0, which
        // holds lanes t and t + 32 in thread t and combines them with
        // shuffles in the oracle's fixed orders (no block barrier inside).
        const unsigned full = 0xffffffffu;
        if constexpr (FP64) {
            double ar = 0.0, ai = 0.0;
            for (int step = 0; step < cnt; ++step) {
                const float2 x = X[step * kLanes], y = Y[step * kLanes];
                ar = fma((double)x.x, (double)y.x, fma(-(double)x.y, (double)y.y, ar));
                ai = fma((double)x.x, (double)y.y, fma((double)x.y, (double)y.x, ai));
            }
            dr[l] = ar;
            di[l] = ai;
            __syncthreads();
            if (l < 32) {
                double vr = dr[l] + dr[l + 32], vi = di[l] + di[l + 32];
#pragma unroll
                for (int stride = 16; stride >= 1; stride /= 2) {
                    vr += __shfl_down_sync(full, vr, stride);
                    vi += __shfl_down_sync(full, vi, stride);
                }
                if (l == 0) {
                    C[(size_t)j * n + i] = make_float2((float)vr, (float)vi);
                }
            }
        } else {
            // pass 1: the lane's direct sum
            float r = 0.0f, im = 0.0f;
            for (int step = 0; step < cnt; ++step) {
                const float2 x = X[step * kLanes], y = Y[step * kLanes];
                const float p = __fmul_rn(__fadd_rn(x.x, x.y), y.x);
                const float q = __fmul_rn(x.x, __fsub_rn(y.y, y.x));
                const float rr = __fmul_rn(x.y, __fadd_rn(y.x, y.y));
                r = __fadd_rn(r, __fsub_rn(p, rr));
                im = __fadd_rn(im, __fadd_rn(p, q));
            }
            sr[l] = r;
            si[l] = im;
            __syncthreads();
            if (l < 32) {
                const float lo_r = sr[l], hi_r = sr[l + 32], lo_i = si[l], hi_i = si[l + 32];
                // direct: pairwise reduction, stride 32, 16, ..., 1 (lane_reduce)
                float wr = __fadd_rn(lo_r, hi_r), wi = __fadd_rn(lo_i, hi_i);
#pragma unroll
                for (int stride = 16; stride >= 1; stride /= 2) {
                    const float xr = __shfl_down_sync(full, wr, stride), xi = __shfl_down_sync(full, wi, stride);
                    if (l < stride) {
                        wr = __fadd_rn(wr, xr);
                        wi = __fadd_rn(wi, xi);
                    }
                }
                const float direct_r = __shfl_sync(full, wr, 0), direct_i = __shfl_sync(full, wi, 0);
                // inclusive Hillis-Steele scan, distances 1 .. 32, every step
                // reading the previous one: new[x] = v[x] + v[x - d] for x >= d
                float ar = lo_r, br = hi_r, ai = lo_i, bi = hi_i;  // lanes l and l + 32
#pragma unroll
                for (int d = 1; d < 32; d *= 2) {
                    const float up_ar = __shfl_up_sync(full, ar, d), up_ai = __shfl_up_sync(full, ai, d);
                    const float up_br = __shfl_up_sync(full, br, d), up_bi = __shfl_up_sync(full, bi, d);
                    const int src = l + 32 - d;  // for l < d: lane l + 32 - d of the low half
                    const float lo_wr = __shfl_sync(full, ar, src & 31), lo_wi = __shfl_sync(full, ai, src & 31);
                    const float nbr = __fadd_rn(br, l >= d ? up_br : lo_wr);
                    const float nbi = __fadd_rn(bi, l >= d ? up_bi : lo_wi);
                    if (l >= d) {
                        ar = __fadd_rn(ar, up_ar);
                        ai = __fadd_rn(ai, up_ai);
                    }
                    br = nbr;
                    bi = nbi;
                }
                br = __fadd_rn(br, ar);  // d = 32: lane l + 32 adds lane l
                bi = __fadd_rn(bi, ai);
                // largest |inclusive prefix| per part (max is order-free)
                float mr = fmaxf(fabsf(ar), fabsf(br)), mi = fmaxf(fabsf(ai), fabsf(bi));
#pragma unroll
                for (int off = 16; off >= 1; off /= 2) {
                    mr = fmaxf(mr, __shfl_xor_sync(full, mr, off));
                    mi = fmaxf(mi, __shfl_xor_sync(full, mi, off));
                }
                // seeds: lane x starts from the inclusive prefix of lane x - 1
                const float pa_r = __shfl_up_sync(full, ar, 1), pa_i = __shfl_up_sync(full, ai, 1);
                const float pb_r = __shfl_up_sync(full, br, 1), pb_i = __shfl_up_sync(full, bi, 1);
                const float last_r = __shfl_sync(full, ar, 31), last_i = __shfl_sync(full, ai, 31);
                tr[l] = l >= 1 ? pa_r : 0.0f;
                ti[l] = l >= 1 ? pa_i : 0.0f;
                tr[l + 32] = l >= 1 ? pb_r : last_r;
                ti[l + 32] = l >= 1 ? pb_i : last_i;
                if (l == 0) {
                    peak_r[0] = mr;
                    peak_i[0] = mi;
                    peak_r[1] = direct_r;
                    peak_i[1] = direct_i;
                }
            }
            __syncthreads();
            // pass 2: replay seeded with the previous lane's prefix
            const float init_r = tr[l], init_i = ti[l];
            r = __fadd_rn(init_r, 0.0f);
            im = __fadd_rn(init_i, 0.0f);
            for (int step = 0; step < cnt; ++step) {
                const float2 x = X[step * kLanes], y = Y[step * kLanes];
                const float p = __fmul_rn(__fadd_rn(x.x, x.y), y.x);
                const float q = __fmul_rn(x.x, __fsub_rn(y.y, y.x));
                const float rr = __fmul_rn(x.y, __fadd_rn(y.x, y.y));
                r = __fadd_rn(r, __fsub_rn(p, rr));
                im = __fadd_rn(im, __fadd_rn(p, q));
            }
            sr[l] = __fsub_rn(r, init_r);
            si[l] = __fsub_rn(im, init_i);
            __syncthreads();
            if (l < 32) {
                float wr = __fadd_rn(sr[l], sr[l + 32]), wi = __fadd_rn(si[l], si[l + 32]);
#pragma unroll
                for (int stride = 16; stride >= 1; stride /= 2) {
                    const float xr = __shfl_down_sync(full, wr, stride), xi = __shfl_down_sync(full, wi, stride);
                    if (l < stride) {
                        wr = __fadd_rn(wr, xr);
                        wi = __fadd_rn(wi, xi);
                    }
                }
                if (l == 0) {
                    const float direct_r = peak_r[1], direct_i = peak_i[1];
                    float out_r = wr, out_i = wi;
                    if (peak_r[0] >= __fmul_rn(fabsf(direct_r), 32.0f)) {
                        out_r = direct_r;
                    }
                    if (peak_i[0] >= __fmul_rn(fabsf(direct_i), 32.0f)) {
                        out_i = direct_i;
                    }
                    C[(size_t)j * n + i] = make_float2(out_r, out_i);
                }
            }
        }
        __syncthreads();  // every read of this output's staged vectors and sums is done
    }
}

}  // namespace

// bridge = (floor(n/128)*128^2 + (n mod 128)^2) / (18 n^2), in FP32 as the
// reference forms it (cgemm3m_rounding_kernel.cpp:96-100).
static float bridge_term(int n)
{
    const int tail = n % 128;
    volatile float a = (float)(n / 128) * (float)(128 * 128);
    volatile float b = a + (float)(tail * tail);
    volatile float d = 18.0f * (float)n;
    volatile float e = d * (float)n;
    return b / e;
}

// Layout of the rounding region (Plan::round_off): path n^2 floats | rows of
// op(A) n^2 complex | columns of op(B) n^2 complex | energies 2n floats |
// flags: one bit per output (written whole by the selection), then one count
// per 16 x 16 tile, kStatWords counters, the exact recompute's fallback bits
// (one per output) and a byte per op(A) row and op(B) column marking those the
// per-output kernels read, all zeroed before every selection | tensor-core
// forms: the exact recompute's exponents, residue planes and product residues
// (OzLayout).
struct RoundLayout {
    float* path;
    float2* rows_a;
    float2* rows_b;
    float2* lanes_a;  // lane-major copies (per-output recompute)
    float2* lanes_b;
    float* energy;
    uint32_t* flag_bits;
    uint32_t* tile_count;
    uint32_t* stats;
    uint32_t* fallback_bits;
    uint8_t* need;      // rows of op(A), then columns of op(B), the per-output kernels read
    uint8_t* band;      // [kMaxBands] op(A) row bands, then [kMaxBands] op(B) column bands, of 256
                        // whose tiles the form's products read (tensor-core forms)
    size_t zero_bytes;  // tile_count + stats + fallback_bits + need + band, one memset
    OzLayout oz;
};

static size_t flag_words(int n) { return ((size_t)n * n + 31) / 32; }
static size_t need_words(int n) { return ((size_t)2 * n + 3) / 4; }
constexpr int kMaxBands = 16;  // 256-row bands of the largest gated order, 4096
static size_t band_words() { return (size_t)2 * kMaxBands / 4; }
static size_t tile_words(int n)
{
    const size_t t = (size_t)(n + kTile - 1) / kTile;
    return t * t;
}

// Row stride of the packed op(A) rows and op(B) columns: n rounded up to even,
// so that every row starts on a 16-byte boundary (the replay stages them with
// 2-D tensor copies, whose row stride must be a multiple of 16 bytes).
static int row_pitch(int n) { return n + (n & 1); }

// Region offsets of the rounding region (shared by the layout and its size).
struct RoundOffsets {
    size_t path, rows_a, rows_b, lanes_a, lanes_b, energy, flags, oz, end;
};

static RoundOffsets round_offsets(int n, int form, std::vector<size_t>* guards)
{
    const size_t nn = (size_t)n * n;
    const size_t rows = (size_t)n * row_pitch(n);
    RoundOffsets o{};
    size_t off = 0;
    o.path = off;
    off = next_region(off, nn * 4, guards);
    o.rows_a = off;
    off = next_region(off, rows * 8, guards);
    o.rows_b = off;
    off = next_region(off, rows * 8, guards);
    const size_t lanes = (size_t)n * kLanes * (((n + kLanes - 1) / kLanes) | 1);
    o.lanes_a = off;
    off = next_region(off, lanes * 8, guards);
    o.lanes_b = off;
    off = next_region(off, lanes * 8, guards);
    o.energy = off;
    off = next_region(off, (size_t)2 * n * 4, guards);
    o.flags = off;
    off = next_region(off, (2 * flag_words(n) + tile_words(n) + kStatWords + need_words(n) + band_words()) * 4,
                      guards);
    o.oz = off;
    if (form != CG3M_FORM_FP32) {
        std::vector<size_t> inner;
        off += oz_layout(n, nullptr, &inner).bytes;
        if (guards != nullptr) {
            for (size_t g : inner) {
                guards->push_back(o.oz + g);
            }
        }
    }
    o.end = off;
    return o;
}

static RoundLayout round_layout(const Plan& plan, void* ws, int n)
{
    uint8_t* b = static_cast<uint8_t*>(ws) + plan.round_off;
    const RoundOffsets o = round_offsets(n, plan.form, nullptr);
    RoundLayout L;
    L.path = reinterpret_cast<float*>(b + o.path);
    L.rows_a = reinterpret_cast<float2*>(b + o.rows_a);
    L.rows_b = reinterpret_cast<float2*>(b + o.rows_b);
    L.lanes_a = reinterpret_cast<float2*>(b + o.lanes_a);
    L.lanes_b = reinterpret_cast<float2*>(b + o.lanes_b);
    L.energy = reinterpret_cast<float*>(b + o.energy);
    L.flag_bits = reinterpret_cast<uint32_t*>(b + o.flags);
    L.tile_count = L.flag_bits + flag_words(n);
    L.stats = L.tile_count + tile_words(n);
    L.fallback_bits = L.stats + kStatWords;
    L.need = reinterpret_cast<uint8_t*>(L.fallback_bits + flag_words(n));
    L.band = L.need + need_words(n) * 4;
    L.zero_bytes = (tile_words(n) + kStatWords + flag_words(n) + need_words(n) + band_words()) * 4;
    if (plan.form != CG3M_FORM_FP32) {
        L.oz = oz_layout(n, b + o.oz);
    }
    return L;
}

uint32_t* rounding_stats_ptr(const Plan& plan, void* ws, int n) { return round_layout(plan, ws, n).stats; }

size_t rounding_bytes(int n, int form, std::vector<size_t>* guards) { return round_offsets(n, form, guards).end; }

cudaError_t launch_gemm_with_path(cudaStream_t s, const Problem& p, const Plan& plan, void* ws, int* status)
{
    const RoundLayout L = round_layout(plan, ws, p.n);
    if (plan.form == CG3M_FORM_FP32) {
        return launch_gemm_fp32_path(s, p, plan, ws, L.path, status);
    }
    const LeadSelect sel{L.energy, bridge_term(p.n), kConfidence * kConfidence, L.flag_bits,
                         L.tile_count, L.stats};
    return launch_gemm_tc_path(s, p, plan, ws, sel, status);
}

// The replay's staging copies: op(A) rows or op(B) columns as an n x n array of
// 8-byte complex elements with the even row pitch; a box is w K terms of 16
// rows.
static bool replay_tensor_map(CUtensorMap* map, const float2* rows, int n, int w)
{
    const uint64_t dims[2] = {(uint64_t)n, (uint64_t)n};
    const uint64_t strides[1] = {(uint64_t)row_pitch(n) * sizeof(float2)};
    const uint32_t box[2] = {(uint32_t)w, (uint32_t)kTile};
    return encode_tensor_map(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, dims, strides, box,
                             CU_TENSOR_MAP_SWIZZLE_NONE, rows);
}

// The replay instance for this order's chunk length ch = ceil(span / kChunks).
template <int CH>
static cudaError_t launch_replay(cudaStream_t s, int n, int span, const RoundLayout& L, float2* C, int* status)
{
    if ((span + kChunks - 1) / kChunks != CH) {
        if constexpr (CH < kChunk) {
            return launch_replay<CH + 1>(s, n, span, L, C, status);
        } else {
            return cudaErrorInvalidValue;  // lanes longer than the staged boxes (n > 4096)
        }
    }
    static_assert(box_width(CH) <= kBoxMax, "box wider than its staging slot");
    CUtensorMap tm_a, tm_b;
    if (!replay_tensor_map(&tm_a, L.rows_a, n, box_width(CH)) ||
        !replay_tensor_map(&tm_b, L.rows_b, n, box_width(CH))) {
        return cudaErrorInvalidValue;
    }
    const int tiles = (n + kTile - 1) / kTile;
    cudaError_t err = cudaFuncSetAttribute(recompute_fp32_tiled<CH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)kRecomputeSmem);
    if (err != cudaSuccess) {
        return err;
    }
    recompute_fp32_tiled<CH><<<tiles * tiles, 512, kRecomputeSmem, s>>>(tm_a, tm_b, n, span, L.flag_bits,
                                                                       L.tile_count, L.stats, C, status);
    return cudaGetLastError();
}

int rounding_prep_kernels(int form)
{
    return form == CG3M_FORM_FP32 ? 2 : 1;  // FP32: packed rows, energies; tensor-core forms: residues
}

// Tensor-core forms: zero the selection's outputs (its flag words too, which
// take per-bit atomics when n is not a multiple of 32), then the packed rows
// with the leading planes and the energies, all before the risk-plane GEMM
// that applies the selection.
cudaError_t launch_rounding_pack(cudaStream_t s, const Problem& p, const Plan& plan, void* ws,
                                 const std::function<void()>& mark)
{
    const int n = p.n;
    const RoundLayout L = round_layout(plan, ws, n);
    const int pitch = row_pitch(n);
    cudaError_t err = cudaMemsetAsync(L.flag_bits, 0, L.zero_bytes + flag_words(n) * 4, s);
    if (err == cudaSuccess) {
        err = launch_pack_rows(s, p, L.rows_a, L.rows_b, pitch, &plan, ws);
        mark();
    }
    if (err == cudaSuccess) {
        const int span = ((n + kLanes - 1) / kLanes) | 1;
        energy_kernel<<<2 * n, kLanes, 0, s>>>(L.rows_a, L.rows_b, n, pitch, span, L.energy);
        err = cudaGetLastError();
        mark();
    }
    return err;
}

cudaError_t launch_rounding_prep(cudaStream_t s, const Problem& p, const Plan& plan, void* ws, int* launched,
                                 const std::function<void(int)>& mark)
{
    const int n = p.n;
    const int pitch = row_pitch(n);
    const RoundLayout L = round_layout(plan, ws, n);
    const int span = ((n + kLanes - 1) / kLanes) | 1;
    int count = 0;
    cudaError_t err = cudaSuccess;
    if (plan.form == CG3M_FORM_FP32) {  // the tensor-core forms packed their rows and energies first
        err = launch_pack_rows(s, p, L.rows_a, L.rows_b, pitch);
        mark(++count);
    }
    if (err == cudaSuccess && plan.form == CG3M_FORM_FP32) {
        energy_kernel<<<2 * n, kLanes, 0, s>>>(L.rows_a, L.rows_b, n, pitch, span,
                                                                        L.energy);
        err = cudaGetLastError();
        mark(++count);
    }
    if (err == cudaSuccess && plan.form != CG3M_FORM_FP32) {
        err = launch_ozaki_split(s, n, pitch, L.rows_a, L.rows_b, L.oz);
        mark(++count);
    }
    if (launched != nullptr) {
        *launched = count;
    }
    return err;
}

cudaError_t launch_rounding_finish(cudaStream_t s, const Problem& p, const Plan& plan, void* ws, int* status,
                                   int* launched, const std::function<void(int)>& mark)
{
    const int n = p.n;
    const RoundLayout L = round_layout(plan, ws, n);
    const int span = ((n + kLanes - 1) / kLanes) | 1;
    int count = 0;
    cudaError_t err = cudaSuccess;
    if (plan.form == CG3M_FORM_FP32) {  // the tensor-core forms' risk-plane GEMM selected already
        err = cudaMemsetAsync(L.tile_count, 0, L.zero_bytes, s);
    }
    if (err == cudaSuccess && plan.form == CG3M_FORM_FP32) {
        select_kernel<<<148 * 8, 256, 0, s>>>(n, static_cast<const float2*>(p.C), L.energy, L.path, bridge_term(n),
                                              L.flag_bits, L.tile_count, L.stats);
        err = cudaGetLastError();
        mark(++count);
    }
    // Dense tiles, then the flagged outputs of sparse tiles one by one; both
    // read the same per-tile counts, so each flagged output is recomputed by
    // exactly one of them.
    const int tiles16 = (n + kTile - 1) / kTile;
    float2* C = static_cast<float2*>(p.C);
    const int exact_gn = plan.form == CG3M_FORM_FP32 ? 1 : ozaki_tile_n(n) / kTile;
    const int pitch = row_pitch(n);
    // lane-major copies of the rows and columns the per-output kernels read
    auto lanes = [&]() {
        const bool tc = plan.form != CG3M_FORM_FP32;
        lanes_needed_kernel<<<148 * 4, 256, 0, s>>>(n, tc ? 1 : 0, L.flag_bits, L.fallback_bits, L.tile_count,
                                                    tc ? L.oz.tile_ran : nullptr, L.oz.y_pad / kOzakiTile, L.need);
        cudaError_t e = cudaGetLastError();
        mark(++count);
        if (e == cudaSuccess) {
            lane_major_kernel<<<2 * n, 256, (size_t)n * sizeof(float2), s>>>(n, pitch, span, L.rows_a, L.rows_b,
                                                                             L.lanes_a, L.lanes_b, L.need);
            e = cudaGetLastError();
            mark(++count);
        }
        return e;
    };
    auto sparse = [&](auto kernel, const uint32_t* bits) {
        // one block per 16 x 16 tile: several tiles per block (4, or a grid-
        // stride walk) saved ~0.02 ms of block launches where no tile has work
        // but made the reference's data (~7 flagged outputs per tile) 1.6-2.5x slower
        kernel<<<tiles16 * tiles16, kLanes, 0, s>>>(n, span, L.lanes_a, L.lanes_b, bits, L.tile_count, L.stats, C,
                                                    exact_gn);
        const cudaError_t e = cudaGetLastError();
        mark(++count);
        return e;
    };
    if (plan.form == CG3M_FORM_FP32) {
        if (err == cudaSuccess) {
            err = launch_replay<kChunkMin>(s, n, span, L, C, status);
            mark(++count);
        }
        if (err == cudaSuccess) {
            err = lanes();
        }
        if (err == cudaSuccess) {
            err = sparse(recompute_sparse<kSparseFp32>, L.flag_bits);
        }
    } else {
        // The path GEMM's C came from the leading split planes alone: the
        // form's own products now run on every tile the exact recompute does
        // not take, and the exact recompute writes every output of its tiles.
        // The rest of the form's planes is packed for the bands those tiles read.
        const int bands = (n + kOzakiTile - 1) / kOzakiTile;
        if (err == cudaSuccess && bands > kMaxBands) {
            err = cudaErrorInvalidValue;  // beyond the gated orders
        }
        if (err == cudaSuccess) {
            band_need_kernel<<<dim3(bands, bands), 256, 0, s>>>(n, L.tile_count, L.band, L.band + kMaxBands);
            err = cudaGetLastError();
            mark(++count);
        }
        if (err == cudaSuccess) {
            err = launch_pack(s, p, plan, ws, L.band, L.band + kMaxBands);
            mark(++count);
        }
        if (err == cudaSuccess) {
            err = launch_gemm_tc_tiles(s, p, plan, ws, status, L.tile_count);
            mark(++count);
        }
        if (err == cudaSuccess) {
            int oz_launched = 0;
            const int before = count;
            err = launch_ozaki_tiles(s, n, L.oz, L.tile_count, L.stats, L.fallback_bits, C, status,
                                     &oz_launched, [&](int i) { mark(before + i); });
            count += oz_launched;
        }
        if (err == cudaSuccess) {
            err = lanes();
        }
        if (err == cudaSuccess) {
            err = sparse(recompute_sparse<kSparseFp64>, L.flag_bits);
        }
        if (err == cudaSuccess) {
            err = sparse(recompute_sparse<kFallbackFp64>, L.fallback_bits);
        }
    }
    if (launched != nullptr) {
        *launched = count;
    }
    return err;
}

}  // namespace cg3m
