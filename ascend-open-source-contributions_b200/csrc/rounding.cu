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
// conflict-free); a grid-stride select that sets one bit per flagged output
// and one word per 16 x 16 output tile (each flagged output is recomputed
// independently, so no ordering is needed to keep the result bits fixed); the
// recompute works on
// output tiles so operand rows are staged once per tile instead of once per
// output, and skips tiles with no flagged output.  FP32 form: the reference's
// segmented replay, one output per thread over 16 x 16 tiles, with the 64
// lane sums in shared memory and the lane reductions and the inclusive lane
// scan in fixed orders.  Tensor-core forms: flagged outputs are recomputed
// in FP64 over 64 x 64 tiles (K in order) and rounded once to FP32.
#include <cstring>
#include <functional>

#include "cg3m_internal.h"

namespace cg3m {

cudaError_t launch_pack_rows(cudaStream_t stream, const Problem& p, void* rows_a, void* rows_b);
cudaError_t launch_gemm_fp32_path(cudaStream_t stream, const Problem& pr, const Plan& plan, void* ws, float* path,
                                  int* status);
cudaError_t launch_gemm_tc_path(cudaStream_t stream, const Problem& pr, const Plan& plan, void* ws, float* path,
                                int* status);

namespace {

constexpr int kLanes = 64;
constexpr int kTile = 16;             // flag granule: 16 x 16 outputs
constexpr int kMaxSpan = 65;          // ceil(4096/64) | 1
constexpr float kConfidence = 3.75f;  // CGEMM_ROUNDING_CONFIDENCE, cgemm_host.cpp:37

// ---- 2. energies ----------------------------------------------------------------

__global__ void __launch_bounds__(kLanes) energy_kernel(const float2* __restrict__ rows_a,
                                                        const float2* __restrict__ rows_b, int n, int span,
                                                        float* __restrict__ energy)
{
    extern __shared__ float2 row[];
    __shared__ float lanes[kLanes];
    const int r = blockIdx.x;
    const float2* src = r < n ? rows_a + (size_t)r * n : rows_b + (size_t)(r - n) * n;
    for (int k = threadIdx.x; k < n; k += kLanes) {
        row[k] = src[k];
    }
    __syncthreads();
    const int l = threadIdx.x;
    float e = 0.0f;
    for (int s = 0; s < span; ++s) {
        const int k = l * span + s;
        if (k >= n) {
            break;
        }
        const float2 x = row[k];
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

__global__ void select_kernel(int n, const float2* __restrict__ C, const float* __restrict__ energy,
                              const float* __restrict__ path, float bridge, uint32_t* __restrict__ flag_bits,
                              uint32_t* __restrict__ tile_flags, uint32_t* __restrict__ count)
{
    const size_t total = (size_t)n * n;
    const int tiles = (n + kTile - 1) / kTile;
    const float conf2 = __fmul_rn(kConfidence, kConfidence);
    uint32_t local = 0;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(idx / n), i = (int)(idx - (size_t)j * n);
        const float2 c = C[idx];
        const float re = fabsf(c.x), im = fabsf(c.y);
        const float magnitude = re > im ? re : im;
        const float variance =
            __fmul_rn(0x1p-48f, __fadd_rn(path[idx], __fmul_rn(__fmul_rn(energy[i], energy[n + j]), bridge)));
        const bool sel = !isfinite(magnitude) || !isfinite(variance) || __fmul_rn(conf2, variance) >= 0.0001f;
        if (sel) {
            atomicOr(&flag_bits[idx >> 5], 1u << (idx & 31));
            atomicOr(&tile_flags[(j / kTile) * tiles + i / kTile], 1u);
            ++local;
        }
    }
    atomicAdd(count, local);
}

__device__ __forceinline__ bool flagged(const uint32_t* bits, size_t idx)
{
    return (bits[idx >> 5] >> (idx & 31)) & 1u;
}

// ---- 4a. FP32 segmented replay (FastSegmentDot) ---------------------------------------

struct Cf {
    float r, i;
};

// One 3M term with the fused identity (ThreeProductTerms, :192-208).
__device__ __forceinline__ Cf term(float2 x, float2 y)
{
    const float p = __fmul_rn(__fadd_rn(x.x, x.y), y.x);
    const float q = __fmul_rn(x.x, __fsub_rn(y.y, y.x));
    const float rr = __fmul_rn(x.y, __fadd_rn(y.x, y.y));
    return Cf{__fsub_rn(p, rr), __fadd_rn(p, q)};
}

// FP32 segmented replay of one 16 x 16 output tile with 512 threads: two per
// output, the lower half of the block summing K lanes 0..31 and the upper half
// lanes 32..63 (lane l holds k in [l*span, (l+1)*span)), both halves on the
// same lane step at a time while the next step's op(A) rows and op(B) columns
// are copied into shared memory.  The 64 lane sums of each output sit in
// shared memory (S[l][output]); the lower-half thread computes the reduction,
// the inclusive scan and the final selection, and both halves replay their
// lanes seeded with the scanned prefixes -- all in the oracle's fixed orders.
// Only flagged outputs are written.
__device__ __forceinline__ void cp_async8(void* dst, const void* src, int src_bytes)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Shared memory of recompute_fp32_tiled: the 64 lane sums (real, imaginary)
// of the tile's 256 outputs, then two staging buffers, each with the operand
// slices (16 rows of op(A) and 16 columns of op(B), span K terms each) of two
// lanes, one for each half of the block.
constexpr size_t kLaneSumBytes = (size_t)2 * kLanes * 256 * sizeof(float);
constexpr size_t kStageElems = (size_t)kMaxSpan * kTile;  // float2 per operand per buffer
constexpr int kStageIters = (kTile * kMaxSpan + 511) / 512;  // staging elements per thread
constexpr size_t kRecomputeSmem = kLaneSumBytes + 2 * 2 * 2 * kStageElems * sizeof(float2);

__global__ void __launch_bounds__(512) recompute_fp32_tiled(int n, int span, const float2* __restrict__ rows_a,
                                                            const float2* __restrict__ rows_b,
                                                            const uint32_t* __restrict__ flag_bits,
                                                            const uint32_t* __restrict__ tile_flags,
                                                            float2* __restrict__ C)
{
    extern __shared__ __align__(16) float lane_sums[];  // [2][64][256]: real then imaginary
    float* sr = lane_sums;
    float* si = lane_sums + kLanes * 256;
    float2* stage_base = reinterpret_cast<float2*>(reinterpret_cast<char*>(lane_sums) + kLaneSumBytes);
    const int tiles = (n + kTile - 1) / kTile;
    if (tile_flags[blockIdx.x] == 0) {
        return;
    }
    const int i0 = (blockIdx.x % tiles) * kTile, j0 = (blockIdx.x / tiles) * kTile;
    const int tid = threadIdx.x;
    // Thread (o, half): output o of the 16 x 16 tile, K lanes [32*half, 32*half + 32).
    // A warp covers 8 rows x 4 columns of the tile, so each of its operand
    // reads touches at most 8 distinct shared addresses.
    const int o = tid & 255, half = tid >> 8;
    const int ti = (o & 7) | (((o >> 5) & 1) << 3), tj = ((o >> 3) & 3) | ((o >> 6) << 2);
    const int i = i0 + ti, j = j0 + tj;
    // Buffer b holds, for both halves h, xs[r][q] and ys[r][q] of lane
    // 32h + step at slot(b, h, 0) and slot(b, h, 1), rows span apart: span is
    // odd, so the rows a warp reads at one q fall in distinct bank pairs, and
    // consecutive threads stage consecutive q of one row.
    auto slot = [&](int b, int h, int op) { return stage_base + (size_t)((b * 2 + h) * 2 + op) * kStageElems; };
    auto lane_count = [&](int l) { return max(0, min(span, n - l * span)); };
    // Staging element e = tid + 512u of a lane slice (u < staged): row
    // r = e / span, K offset q = e % span, shared offset e.  These are fixed for
    // the launch; a step only moves the source by the lane's K start.  A row
    // outside the matrix gets q = span, which fails every q < count test.
    const int slice = kTile * span;
    const int staged = tid < slice ? (slice - tid + 511) / 512 : 0;
    const float2* src_a[kStageIters];
    const float2* src_b[kStageIters];
    int qa[kStageIters], qb[kStageIters];
#pragma unroll
    for (int u = 0; u < kStageIters; ++u) {
        const int e = tid + 512 * u;
        const int r = e / span, q = e - r * span;
        const bool in_a = u < staged && i0 + r < n, in_b = u < staged && j0 + r < n;
        src_a[u] = in_a ? rows_a + (size_t)(i0 + r) * n + q : rows_a;
        src_b[u] = in_b ? rows_b + (size_t)(j0 + r) * n + q : rows_b;
        qa[u] = in_a ? q : span;
        qb[u] = in_b ? q : span;
    }
    // Asynchronous copy of lanes step and 32 + step into buffer b; positions
    // past the end of K or past the matrix read as zero.
    auto issue = [&](int step, int b) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int l = step + 32 * h;
            const int k0 = l * span;
            const int cnt = lane_count(l);
            float2* X = slot(b, h, 0) + tid;
            float2* Y = slot(b, h, 1) + tid;
#pragma unroll
            for (int u = 0; u < kStageIters; ++u) {
                if (u < staged) {
                    const bool okx = qa[u] < cnt, oky = qb[u] < cnt;
                    cp_async8(X + 512 * u, okx ? (const void*)(src_a[u] + k0) : rows_a, okx ? 8 : 0);
                    cp_async8(Y + 512 * u, oky ? (const void*)(src_b[u] + k0) : rows_b, oky ? 8 : 0);
                }
            }
        }
        cp_async_commit();
    };
    // pass 1: lane sums (the next lane pair is copied while this one is summed)
    issue(0, 0);
    for (int step = 0; step < kLanes / 2; ++step) {
        cp_async_wait_all();
        __syncthreads();  // this step staged by every thread; the previous step's buffer is free
        if (step + 1 < kLanes / 2) {
            issue(step + 1, (step + 1) & 1);
        }
        const int l = step + 32 * half;
        const int cnt = lane_count(l);
        const float2* X = slot(step & 1, half, 0);
        const float2* Y = slot(step & 1, half, 1);
        Cf acc{0.0f, 0.0f};
#pragma unroll 8
        for (int q = 0; q < cnt; ++q) {
            const Cf t = term(X[ti * span + q], Y[tj * span + q]);
            acc.r = __fadd_rn(acc.r, t.r);
            acc.i = __fadd_rn(acc.i, t.i);
        }
        sr[l * 256 + o] = acc.r;
        si[l * 256 + o] = acc.i;
    }
    __syncthreads();  // all 64 lane sums of every output are in place
    float direct_r = 0.0f, direct_i = 0.0f, max_r = 0.0f, max_i = 0.0f;
    if (half == 0) {
        // direct reduction (pairwise, stride 32 .. 1) in registers
        float vr[kLanes], vi[kLanes];
#pragma unroll
        for (int l = 0; l < kLanes; ++l) {
            vr[l] = sr[l * 256 + o];
            vi[l] = si[l * 256 + o];
        }
#pragma unroll
        for (int stride = kLanes / 2; stride >= 1; stride /= 2) {
#pragma unroll
            for (int l = 0; l < stride; ++l) {
                vr[l] = __fadd_rn(vr[l], vr[l + stride]);
                vi[l] = __fadd_rn(vi[l], vi[l + stride]);
            }
        }
        direct_r = vr[0];
        direct_i = vi[0];
        // inclusive Hillis-Steele scan in place: new[l] = s[l] + s[l-d] for l >= d
        for (int d = 1; d < kLanes; d *= 2) {
            for (int l = kLanes - 1; l >= d; --l) {
                sr[l * 256 + o] = __fadd_rn(sr[l * 256 + o], sr[(l - d) * 256 + o]);
                si[l * 256 + o] = __fadd_rn(si[l * 256 + o], si[(l - d) * 256 + o]);
            }
        }
        for (int l = 0; l < kLanes; ++l) {
            const float ar = fabsf(sr[l * 256 + o]), ai = fabsf(si[l * 256 + o]);
            max_r = ar > max_r ? ar : max_r;
            max_i = ai > max_i ? ai : max_i;
        }
    }
    __syncthreads();  // scanned prefixes in place; every thread is done with the last buffer
    // pass 2: replay each lane seeded with the previous lanes' prefix.  The
    // upper half starts from the prefix of lane 31, read before the lower half
    // overwrites it (after at least 31 more barriers).
    float prev_r = half == 0 ? 0.0f : sr[31 * 256 + o];
    float prev_i = half == 0 ? 0.0f : si[31 * 256 + o];
    issue(0, 0);
    for (int step = 0; step < kLanes / 2; ++step) {
        cp_async_wait_all();
        __syncthreads();
        if (step + 1 < kLanes / 2) {
            issue(step + 1, (step + 1) & 1);
        }
        const int l = step + 32 * half;
        const int cnt = lane_count(l);
        const float2* X = slot(step & 1, half, 0);
        const float2* Y = slot(step & 1, half, 1);
        const float init_r = prev_r, init_i = prev_i;
        prev_r = sr[l * 256 + o];
        prev_i = si[l * 256 + o];
        float r = __fadd_rn(init_r, 0.0f), im = __fadd_rn(init_i, 0.0f);
#pragma unroll 8
        for (int q = 0; q < cnt; ++q) {
            const Cf t = term(X[ti * span + q], Y[tj * span + q]);
            r = __fadd_rn(r, t.r);
            im = __fadd_rn(im, t.i);
        }
        sr[l * 256 + o] = __fsub_rn(r, init_r);
        si[l * 256 + o] = __fsub_rn(im, init_i);
    }
    __syncthreads();  // every replayed lane is in place
    if (half == 0) {
        float vr[kLanes], vi[kLanes];
#pragma unroll
        for (int l = 0; l < kLanes; ++l) {
            vr[l] = sr[l * 256 + o];
            vi[l] = si[l * 256 + o];
        }
#pragma unroll
        for (int stride = kLanes / 2; stride >= 1; stride /= 2) {
#pragma unroll
            for (int l = 0; l < stride; ++l) {
                vr[l] = __fadd_rn(vr[l], vr[l + stride]);
                vi[l] = __fadd_rn(vi[l], vi[l + stride]);
            }
        }
        float bridged_r = vr[0], bridged_i = vi[0];
        if (max_r >= __fmul_rn(fabsf(direct_r), 32.0f)) {
            bridged_r = direct_r;
        }
        if (max_i >= __fmul_rn(fabsf(direct_i), 32.0f)) {
            bridged_i = direct_i;
        }
        if (i < n && j < n) {
            const size_t idx = (size_t)j * n + i;
            if (flagged(flag_bits, idx)) {
                C[idx] = make_float2(bridged_r, bridged_i);
            }
        }
    }
}

// ---- 4b. FP64 recompute (tensor-core forms) -----------------------------------------

// FP64 product of one 64 x 64 output tile (each thread 4 x 4 outputs, K in
// order), computed only when one of its 16 x 16 flag granules is set; flagged
// outputs are rounded once to FP32 and written.
constexpr int kT64 = 64;

// Operand slabs of 16 K terms, converted to FP64 once while staging (each
// value feeds 16 threads), double-buffered with the next slab held in
// registers during the current slab's DFMAs.
constexpr size_t kFp64Slab = (size_t)16 * kT64;  // double2 per operand per buffer
constexpr size_t kFp64Smem = 2 * 2 * kFp64Slab * sizeof(double2);

__global__ void __launch_bounds__(256, 2) recompute_fp64_tiled(int n, const float2* __restrict__ rows_a,
                                                            const float2* __restrict__ rows_b,
                                                            const uint32_t* __restrict__ flag_bits,
                                                            const uint32_t* __restrict__ tile_flags,
                                                            float2* __restrict__ C)
{
    extern __shared__ __align__(16) double2 slabs[];  // [buffer][x | y][16][64]
    const int tiles16 = (n + kTile - 1) / kTile;
    const int tiles64 = (n + kT64 - 1) / kT64;
    const int i0 = (blockIdx.x % tiles64) * kT64, j0 = (blockIdx.x / tiles64) * kT64;
    uint32_t any = 0;
    for (int q = 0; q < 16; ++q) {
        const int gi = i0 / kTile + (q & 3), gj = j0 / kTile + (q >> 2);
        if (gi < tiles16 && gj < tiles16) {
            any |= tile_flags[gj * tiles16 + gi];
        }
    }
    if (any == 0) {
        return;
    }
    const int tid = threadIdx.x;
    // Thread (ti, tj) owns rows ti + 16a and columns tj + 16b (a, b < 4): for a
    // fixed a the 16 row values a warp reads are 256 consecutive bytes.
    const int ti = tid & 15, tj = tid >> 4;
    double ar[4][4], ai[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            ar[a][b] = 0.0;
            ai[a][b] = 0.0;
        }
    // Element e = tid + 256*u of a slab: row r = e >> 4, K offset q = e & 15.
    float2 vx[4], vy[4];
    auto load = [&](int k0) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = tid + 256 * u;
            const int r = e >> 4, q = e & 15;
            const int k = k0 + q;
            vx[u] = (k < n && i0 + r < n) ? rows_a[(size_t)(i0 + r) * n + k] : make_float2(0.0f, 0.0f);
            vy[u] = (k < n && j0 + r < n) ? rows_b[(size_t)(j0 + r) * n + k] : make_float2(0.0f, 0.0f);
        }
    };
    load(0);
    const int slabs_n = (n + 15) / 16;
    for (int t = 0; t < slabs_n; ++t) {
        double2* xs = slabs + (size_t)(t & 1) * 2 * kFp64Slab;
        double2* ys = xs + kFp64Slab;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = tid + 256 * u;
            const int r = e >> 4, q = e & 15;
            xs[q * kT64 + r] = make_double2((double)vx[u].x, (double)vx[u].y);
            ys[q * kT64 + r] = make_double2((double)vy[u].x, (double)vy[u].y);
        }
        // Buffer t&1 was last read in slab t-2; this barrier also orders slab
        // t-1's reads before slab t+1's writes.
        __syncthreads();
        if (t + 1 < slabs_n) {
            load((t + 1) * 16);
        }
#pragma unroll 2
        for (int q = 0; q < 16; ++q) {
            double2 x[4], y[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                x[a] = xs[q * kT64 + ti + 16 * a];
                y[a] = ys[q * kT64 + tj + 16 * a];
            }
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    ar[a][b] = fma(x[a].x, y[b].x, fma(-x[a].y, y[b].y, ar[a][b]));
                    ai[a][b] = fma(x[a].x, y[b].y, fma(x[a].y, y[b].x, ai[a][b]));
                }
        }
    }
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        const int j = j0 + tj + 16 * b;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int i = i0 + ti + 16 * a;
            if (i < n && j < n) {
                const size_t idx = (size_t)j * n + i;
                if (flagged(flag_bits, idx)) {
                    C[idx] = make_float2((float)ar[a][b], (float)ai[a][b]);
                }
            }
        }
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
// flags (one bit per output, then one word per 16 x 16 tile, then the flagged
// count), zeroed before every selection.
struct RoundLayout {
    float* path;
    float2* rows_a;
    float2* rows_b;
    float* energy;
    uint32_t* flag_bits;
    uint32_t* tile_flags;
    uint32_t* count;
    size_t flag_bytes;  // flag_bits + tile_flags + count, one memset
};

static size_t flag_words(int n) { return ((size_t)n * n + 31) / 32; }
static size_t tile_words(int n)
{
    const size_t t = (size_t)(n + kTile - 1) / kTile;
    return t * t;
}

static RoundLayout round_layout(const Plan& plan, void* ws, int n)
{
    uint8_t* b = static_cast<uint8_t*>(ws) + plan.round_off;
    const size_t nn = (size_t)n * n;
    RoundLayout L;
    size_t off = 0;
    L.path = reinterpret_cast<float*>(b + off);
    off = align_up(off + nn * 4, kRegionAlign);
    L.rows_a = reinterpret_cast<float2*>(b + off);
    off = align_up(off + nn * 8, kRegionAlign);
    L.rows_b = reinterpret_cast<float2*>(b + off);
    off = align_up(off + nn * 8, kRegionAlign);
    L.energy = reinterpret_cast<float*>(b + off);
    off = align_up(off + (size_t)2 * n * 4, kRegionAlign);
    L.flag_bits = reinterpret_cast<uint32_t*>(b + off);
    L.tile_flags = L.flag_bits + flag_words(n);
    L.count = L.tile_flags + tile_words(n);
    L.flag_bytes = (flag_words(n) + tile_words(n) + 1) * 4;
    return L;
}

size_t rounding_bytes(int n)
{
    const size_t nn = (size_t)n * n;
    size_t off = 0;
    off = align_up(off + nn * 4, kRegionAlign);
    off = align_up(off + nn * 8, kRegionAlign);
    off = align_up(off + nn * 8, kRegionAlign);
    off = align_up(off + (size_t)2 * n * 4, kRegionAlign);
    off = align_up(off + (flag_words(n) + tile_words(n) + 1) * 4, kRegionAlign);
    return off;
}

cudaError_t launch_gemm_with_path(cudaStream_t s, const Problem& p, const Plan& plan, void* ws, int* status)
{
    const RoundLayout L = round_layout(plan, ws, p.n);
    return plan.form == CG3M_FORM_FP32 ? launch_gemm_fp32_path(s, p, plan, ws, L.path, status)
                                       : launch_gemm_tc_path(s, p, plan, ws, L.path, status);
}

cudaError_t launch_rounding(cudaStream_t s, const Problem& p, const Plan& plan, void* ws, int*, int* launched,
                            const std::function<void(int)>& mark)
{
    const int n = p.n;
    const RoundLayout L = round_layout(plan, ws, n);
    const int span = ((n + kLanes - 1) / kLanes) | 1;
    int count = 0;
    cudaError_t err = launch_pack_rows(s, p, L.rows_a, L.rows_b);
    mark(++count);
    if (err == cudaSuccess) {
        energy_kernel<<<2 * n, kLanes, (size_t)n * sizeof(float2), s>>>(L.rows_a, L.rows_b, n, span, L.energy);
        err = cudaGetLastError();
        mark(++count);
    }
    if (err == cudaSuccess) {
        err = cudaMemsetAsync(L.flag_bits, 0, L.flag_bytes, s);
    }
    if (err == cudaSuccess) {
        select_kernel<<<148 * 8, 256, 0, s>>>(n, static_cast<const float2*>(p.C), L.energy, L.path, bridge_term(n),
                                              L.flag_bits, L.tile_flags, L.count);
        err = cudaGetLastError();
        mark(++count);
    }
    if (err == cudaSuccess) {
        if (plan.form == CG3M_FORM_FP32) {
            const int tiles = (n + kTile - 1) / kTile;
            const size_t smem = kRecomputeSmem;
            err = cudaFuncSetAttribute(recompute_fp32_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (err == cudaSuccess) {
                recompute_fp32_tiled<<<tiles * tiles, 512, smem, s>>>(n, span, L.rows_a, L.rows_b, L.flag_bits,
                                                                     L.tile_flags, static_cast<float2*>(p.C));
            }
        } else {
            const int tiles = (n + kT64 - 1) / kT64;
            err = cudaFuncSetAttribute(recompute_fp64_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kFp64Smem);
            if (err == cudaSuccess) {
                recompute_fp64_tiled<<<tiles * tiles, 256, kFp64Smem, s>>>(n, L.rows_a, L.rows_b, L.flag_bits,
                                                                            L.tile_flags, static_cast<float2*>(p.C));
            }
        }
        if (err == cudaSuccess) {
            err = cudaGetLastError();
        }
        mark(++count);
    }
    if (launched != nullptr) {
        *launched = count;
    }
    return err;
}

}  // namespace cg3m
