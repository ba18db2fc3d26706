// gemm_tc.cu -- the three real products on the 5th-generation tensor cores
// (tcgen05) with FP32 accumulators in TMEM: the precision forms 3xTF32 and
// split-BF16 (x6 / x9 products).
//
// Reference counterpart: gemm_cgemm_fused_kernel (blas/gemm/arch35/
// cgemm_compute_kernel.cpp:879-896), whose Cube unit keeps the three products
// of one output tile in three L0C accumulators (:602) and whose vector cores
// merge them and write C (:748-760).  The reference computes them in FP32 with
// HF32 disabled (:356); here the products run on tensor cores with each FP32
// operand split into TF32 or BF16 terms, which restores FP32-level products
// while the accumulation stays FP32.
//
// B200 design.  One CTA per 128 x BN output tile (cta_group::1, M = 128,
// N = BN = 128), 320 threads:
//   warp 0       TMA producer: per K-block and component c in {re, im, sum}
//                one 3-D box for A (all split planes of c) and one for B,
//                128-byte rows with the 128-byte swizzle, into a 192 KB
//                ring (3 stages for 3xTF32, 2 for split-BF16; 64-byte rows
//                give deeper rings but measured slower);
//   warp 1       allocates TMEM (512 columns; 256 for BN = 64); one lane
//                issues every tcgen05.mma: accumulator c (columns
//                [BN*c, BN*c + BN)) +=
//                sum over split pairs (i, j) of A_c,i * B_c,j, smallest terms
//                first; tcgen05.commit releases each ring slot;
//   warps 2-9    epilogue: after every 128-term K segment, tcgen05.ld of
//                P0, P1, P2 (one TMEM lane = one output row, BN/2 columns per
//                warp), Re_s = P0-P1, Im_s = P2-(P0+P1) added to running Re,
//                Im in registers with round-to-nearest FP32; at the end
//                alpha/beta and a column-major C store in which each warp
//                instruction writes 32 consecutive rows of one column.
// Why segments: the tensor core aligns the products of one MMA and the
// accumulator to the largest exponent and truncates, a bias that grows
// linearly with the number of MMAs chained into one accumulator.  Over a
// 4096-term K (1536 chained MMAs for 3xTF32) that costs ~15x the error of a
// round-to-nearest FP32 chain; restarting the accumulators every 128 terms
// (the reference's own segment length for this shape, cgemm_host.cpp:257-260)
// and merging segments on the CUDA cores brings the error below plain FP32.
// Operand planes are K-major ([row][k]) and split by the pack kernel, so the
// sums Ar+Ai and Br+Bi are formed in FP32 before any rounding to TF32/BF16.
// Every wait on an mbarrier is bounded; a timeout sets the status word, the
// CTA stops issuing work, waits for what is in flight, frees TMEM and exits.
#include <cuda_bf16.h>

#include "cg3m_internal.h"
#include "epilogue.cuh"
#include "ptx.cuh"

// The rounding-correction gate's risk plane comes from gemm3m_lead_path_kernel
// below: the leading split planes in the four-multiplication form, 128 x 128
// tiles, the running sums in TMEM and both risk integrals per output in
// registers (MergeProductsWithPath, cgemm_compute_kernel.cpp:432-474).
namespace cg3m {
namespace {

constexpr int TILE_M = 128;                     // M of the MMA and rows of the output tile
constexpr int ROW_BYTES = 128;                  // one K-block row of one plane (128-byte swizzle)
constexpr int A_PLANE = TILE_M * ROW_BYTES;     // 16 KB: one A plane, 128 rows
constexpr int RING_BYTES = 192 * 1024;          // operand ring; stages = RING_BYTES / stage size
constexpr int kEpilogueWarps = 8;
constexpr int kThreads = (2 + kEpilogueWarps) * 32;
// 10 warps land 3/3/2/2 on the SM's four sub-partitions, whose register files
// hold 16K registers each: 3 warps x 32 threads x 168 registers is the most
// that still launches, so each epilogue thread keeps 2 x 64 running sums
// (BN = 128) and streams TMEM through 8-column pieces.

template <int FORM>
struct TcCfg;

template <>
struct TcCfg<CG3M_FORM_TF32X3> {
    static constexpr int S = 2;        // split planes per component (hi, lo)
    static constexpr int ZS = 2;       // planes per component in the packed layout
    static constexpr int BK = 32;      // K elements per 128-byte row
    static constexpr int NPAIRS = 3;   // lo*hi, hi*lo, hi*hi
    static constexpr uint32_t FMT = 2; // TF32
    __device__ static int2 pair(int q) { return q == 0 ? make_int2(1, 0) : q == 1 ? make_int2(0, 1) : make_int2(0, 0); }
};

template <>
struct TcCfg<CG3M_FORM_BF16X6> {
    static constexpr int S = 3;        // b0, b1, b2
    static constexpr int ZS = 3;
    static constexpr int BK = 64;
    static constexpr int NPAIRS = 6;   // b_i*b_j with i+j <= 2, smallest first
    static constexpr uint32_t FMT = 1; // BF16
    __device__ static int2 pair(int q)
    {
        switch (q) {
            case 0: return make_int2(2, 0);
            case 1: return make_int2(1, 1);
            case 2: return make_int2(0, 2);
            case 3: return make_int2(1, 0);
            case 4: return make_int2(0, 1);
            default: return make_int2(0, 0);
        }
    }
};

template <>
struct TcCfg<CG3M_FORM_BF16X9> {
    static constexpr int S = 3;
    static constexpr int ZS = 3;
    static constexpr int BK = 64;
    static constexpr int NPAIRS = 9;   // all b_i*b_j, smallest first
    static constexpr uint32_t FMT = 1;
    __device__ static int2 pair(int q)
    {
        switch (q) {
            case 0: return make_int2(2, 2);
            case 1: return make_int2(2, 1);
            case 2: return make_int2(1, 2);
            case 3: return make_int2(2, 0);
            case 4: return make_int2(1, 1);
            case 5: return make_int2(0, 2);
            case 6: return make_int2(1, 0);
            case 7: return make_int2(0, 1);
            default: return make_int2(0, 0);
        }
    }
};

// The leading split plane alone (one tensor pass over the form's packed
// planes, ZS of them per component): the risk plane of the tensor-core forms'
// rounding pass.  The pass recomputes exactly every output of a tile it finds
// dense and runs the form's own products on the other tiles, so this product
// only feeds the selection, whose risk estimate needs a few significant bits.
constexpr int kLeadTf32 = 100;
constexpr int kLeadBf16 = 101;

template <>
struct TcCfg<kLeadTf32> {
    static constexpr int ZS = 2;       // planes per component in the packed layout (plane 0 is read)
    static constexpr int BK = 32;
    static constexpr uint32_t FMT = 2;
};

template <>
struct TcCfg<kLeadBf16> {
    static constexpr int ZS = 3;
    static constexpr int BK = 64;
    static constexpr uint32_t FMT = 1;
};

// Geometry of one instantiation: output tile 128 x BN.
template <int FORM, int BN>
struct TcGeom {
    using Cfg = TcCfg<FORM>;
    static constexpr int B_PLANE = BN * ROW_BYTES;
    static constexpr int STAGE_BYTES = Cfg::S * (A_PLANE + B_PLANE);
    static constexpr int STAGES = RING_BYTES / STAGE_BYTES;
    static constexpr int COLS = BN / 2;                        // columns per epilogue thread
    static constexpr int TMEM_COLS = 4 * BN;                   // 3 accumulators + the spare block
    static constexpr size_t SMEM = (size_t)STAGES * STAGE_BYTES + 1024 + 256;
    static_assert(TMEM_COLS == 256 || TMEM_COLS == 512, "TMEM allocation must be a power of two");
};

struct TcParams {
    int m, n, k;
    int span, parts;
    int tiles_m, tiles_n;
    EpiParams epi;
    float2* C;
    int ldc;
    float* partial;
    int ppitch;
    size_t pplane;
    int* status;
    int seg_blocks;  // K-blocks per accumulation segment
    int cluster_merge;  // pair kernel: the `parts` pairs of a tile form one cluster and merge on chip
    // pair kernel in the rounding pass: the per-16 x 16 flagged counts; pair
    // tiles inside a 256 x 256 tile the exact recompute takes are skipped
    const uint32_t* skip_count;
    // gemm3m_lead_path_kernel: the rounding pass's selection in its epilogue
    const float* energy;   // [n] op(A) rows, then [n] op(B) columns
    float bridge, conf2;
    uint32_t* flag_bits;   // one bit per output (column-major index), zeroed beforehand
    uint32_t* tile_count;  // flagged outputs per 16 x 16 tile, zeroed beforehand
    uint32_t* stats;
};

// Loads from a shared::cluster address (a peer block's shared memory).
__device__ __forceinline__ float ld_dsmem_f32(uint32_t addr)
{
    float v;
    asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(addr) : "memory");
    return v;
}
__device__ __forceinline__ int ld_dsmem_s32(uint32_t addr)
{
    int v;
    asm volatile("ld.shared::cluster.s32 %0, [%1];" : "=r"(v) : "r"(addr) : "memory");
    return v;
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle (layout type 2),
// 8-row groups 8 x 128 = 1024 bytes apart (SBO), leading offset unused (1),
// descriptor version 1.  Consecutive MMAs along K advance the start address by
// 32 bytes inside the swizzled row, as the hardware swizzles on absolute
// address bits and every plane tile starts on a 1024-byte boundary.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)((8 * ROW_BYTES) >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// Instruction descriptor: FP32 accumulate, A/B format, both K-major, M = 128, N = BN.
template <uint32_t FMT, int BN>
__device__ __forceinline__ uint32_t instr_desc()
{
    return (1u << 4) | (FMT << 7) | (FMT << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(TILE_M >> 4) << 24);
}

// d/9 * (old^2 + old*new + new^2) added to the integral (MergeProductsWithPath).
__device__ __forceinline__ float risk_step(float integral, float old, float nw, float w)
{
    float t = __fmul_rn(old, old);
    t = __fmaf_rn(old, nw, t);
    t = __fmaf_rn(nw, nw, t);
    return __fadd_rn(integral, __fmul_rn(t, w));
}

// One segment of the risk integral summed by parts (gemm3m_lead_path_kernel):
// before the last segment acc += s_new (2 s_new + s_old); the last one turns
// acc into the integral, wfull (acc - s_old^2) + w (s_old^2 + s_old s_new + s_new^2).
template <bool LAST>
__device__ __forceinline__ float risk_part(float acc, float old, float nw, float w, float wfull)
{
    if constexpr (!LAST) {
        return __fmaf_rn(nw, __fmaf_rn(nw, 2.0f, old), acc);
    } else {
        return risk_step(__fmul_rn(wfull, __fsub_rn(acc, __fmul_rn(old, old))), old, nw, w);
    }
}

// One segment's drain of an epilogue thread's COLS columns: Re_s and Im_s
// merge into the running sums in TMEM (round-to-nearest FP32) and both risk
// integrals advance.  STEP 0: the first segment of several (the running sums
// start at the segment's sums), 1: a middle one, 2: the last one, which
// closes the integrals (first says whether it is also the first).
template <int COLS, int STEP>
__device__ __forceinline__ void lead_drain(uint32_t seg_re, uint32_t seg_im, uint32_t run_re, uint32_t run_im,
                                           bool first, float w, float wfull, float* ir, float* ii)
{
#pragma unroll
    for (int part = 0; part < 2; ++part) {
        const uint32_t sa = part == 0 ? seg_re : seg_im, ra = part == 0 ? run_re : run_im;
        float* acc = part == 0 ? ir : ii;
#pragma unroll
        for (int cb = 0; cb < COLS; cb += 8) {
            float v[8], r[8];
            if constexpr (STEP == 0) {
                tmem_ld8(sa + (uint32_t)cb, v);
            } else {
                tmem_ld8x2(sa + (uint32_t)cb, ra + (uint32_t)cb, v, r);
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if constexpr (STEP == 0) {
                    acc[cb + j] = __fmul_rn(v[j], __fmul_rn(v[j], 2.0f));  // s_1 (2 s_1 + s_0), s_0 = 0
                    r[j] = v[j];
                } else if constexpr (STEP == 1) {
                    const float nw = __fadd_rn(r[j], v[j]);
                    acc[cb + j] = risk_part<false>(acc[cb + j], r[j], nw, w, wfull);
                    r[j] = nw;
                } else {
                    const float old = first ? 0.0f : r[j];
                    const float nw = first ? v[j] : __fadd_rn(r[j], v[j]);
                    acc[cb + j] = risk_part<true>(first ? 0.0f : acc[cb + j], old, nw, w, wfull);
                    r[j] = nw;
                }
            }
            tmem_st8(ra + (uint32_t)cb, r);
        }
    }
}

template <int FORM, int BN>
__global__ void __launch_bounds__(kThreads, 1)
    gemm3m_tc_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                     const TcParams p)
{
    using Cfg = TcCfg<FORM>;
    using G = TcGeom<FORM, BN>;
    constexpr int STAGES = G::STAGES;
    constexpr int STAGE_BYTES = G::STAGE_BYTES;
    constexpr int KSTEPS = ROW_BYTES / 32;  // 32 bytes of K per MMA: 8 tf32 or 16 bf16
    constexpr int COLS = G::COLS;

    extern __shared__ uint8_t smem_raw[];
    uint8_t* ring = align_shared<1024>(smem_raw);
    uint64_t* full = reinterpret_cast<uint64_t*>(ring + STAGES * STAGE_BYTES);
    uint64_t* empty = full + STAGES;
    uint64_t* acc_full = empty + STAGES;  // [3] MMA -> epilogue: product c of the segment is in TMEM
    uint64_t* acc_free = acc_full + 3;    // [3] epilogue -> MMA: accumulator c may be overwritten
    uint64_t* mma_done = acc_free + 3;    // every MMA of the CTA has completed
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_done + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;

    constexpr int GM = 8;
    const int pid = blockIdx.x;
    const int in_group = GM * p.tiles_n;
    const int first_m = (pid / in_group) * GM;
    const int gsz = min(p.tiles_m - first_m, GM);
    const int tm = first_m + (pid % in_group) % gsz;
    const int tn = (pid % in_group) / gsz;
    const int m0 = tm * TILE_M, n0 = tn * BN;
    const int part = blockIdx.y;
    const int kbeg = part * p.span;
    const int kend = min(p.k, kbeg + p.span);
    const int kblocks = (kend - kbeg + Cfg::BK - 1) / Cfg::BK;
    const int seg_blocks = p.seg_blocks;
    const int segments = (kblocks + seg_blocks - 1) / seg_blocks;

    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int c = 0; c < 3; ++c) {
            mbar_init(&acc_full[c], 1);
            mbar_init(&acc_free[c], kEpilogueWarps);
        }
        mbar_init(mma_done, 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 1) {
        tmem_alloc(tmem_slot, G::TMEM_COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    // Work order (producer and MMA issuer walk it identically): for each K
    // segment, for each component c in {re, im, sum}, for each K-block of the
    // segment, one ring stage holding component c's split planes of A and B.
    if (warp == 0) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            tma_prefetch_desc(&tmA);
            tma_prefetch_desc(&tmB);
            int it = 0;
            bool stop = false;
            for (int seg = 0; seg < segments && !stop; ++seg) {
                const int kb0 = seg * seg_blocks, kb1 = min(kblocks, kb0 + seg_blocks);
                for (int c = 0; c < 3 && !stop; ++c) {
                    for (int kb = kb0; kb < kb1; ++kb, ++it) {
                        const int s = it % STAGES;
                        if ((it >= STAGES && !mbar_wait(&empty[s], ((it / STAGES) - 1) & 1, p.status)) ||
                            *abort_flag) {
                            *abort_flag = 1;
                            stop = true;
                            break;
                        }
                        uint8_t* st = ring + s * STAGE_BYTES;
                        mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
                        tma_load_3d(st, &tmA, &full[s], kbeg + kb * Cfg::BK, m0, c * Cfg::ZS);
                        tma_load_3d(st + Cfg::S * A_PLANE, &tmB, &full[s], kbeg + kb * Cfg::BK, n0, c * Cfg::ZS);
                    }
                }
            }
            for (int j = it > STAGES ? it - STAGES : 0; j < it; ++j) {
                mbar_wait(&full[j % STAGES], (j / STAGES) & 1, p.status);
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            const uint32_t idesc = instr_desc<Cfg::FMT, BN>();
            int it = 0;
            bool stop = false;
            for (int seg = 0; seg < segments && !stop; ++seg) {
                const int kb0 = seg * seg_blocks, kb1 = min(kblocks, kb0 + seg_blocks);
                for (int c = 0; c < 3 && !stop; ++c) {
                    if (seg > 0) {
                        if (!mbar_wait(&acc_free[c], (seg - 1) & 1, p.status)) {
                            *abort_flag = 1;
                            stop = true;
                            break;
                        }
                        tc_fence_after();
                    }
                    const uint32_t d = tmem + (uint32_t)(c * BN);
                    for (int kb = kb0; kb < kb1; ++kb, ++it) {
                        const int s = it % STAGES;
                        if (!mbar_wait(&full[s], (it / STAGES) & 1, p.status)) {
                            *abort_flag = 1;
                            stop = true;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t a_base = smem_u32(ring + s * STAGE_BYTES);
                        const uint32_t b_base = a_base + Cfg::S * A_PLANE;
#pragma unroll
                        for (int kk = 0; kk < KSTEPS; ++kk) {
#pragma unroll
                            for (int q = 0; q < Cfg::NPAIRS; ++q) {
                                const int2 ij = Cfg::pair(q);
                                const uint64_t ad = smem_desc(a_base + ij.x * A_PLANE + kk * 32);
                                const uint64_t bd = smem_desc(b_base + ij.y * G::B_PLANE + kk * 32);
                                const uint32_t acc = (kb > kb0 || kk > 0 || q > 0) ? 1u : 0u;
                                if constexpr (Cfg::FMT == 2) {
                                    umma_tf32(d, ad, bd, idesc, acc);
                                } else {
                                    umma_f16(d, ad, bd, idesc, acc);
                                }
                            }
                        }
                        umma_commit(&empty[s]);
                    }
                    if (!stop && c > 0) {
                        // Fires when every MMA issued so far has completed: after c == 1
                        // both P0 and P1 of the segment are final, after c == 2 all three.
                        umma_commit(&acc_full[c]);
                    }
                }
            }
            umma_commit(mma_done);
            mbar_wait(mma_done, 0, p.status);  // nothing may still write TMEM when it is freed
        }
    } else {
        // ---------------- epilogue warps 2..9 ----------------
        // TMEM lane quadrant = warp % 4; warps 2-5 take the first BN/2 columns,
        // warps 6-9 the second half, of every accumulator and of the spare block.
        const int quad = warp & 3;
        const int half = (warp - 2) >> 2;
        const int row = m0 + quad * 32 + lane;
        const uint32_t lane_addr = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(half * COLS);
        const uint32_t spare = lane_addr + (uint32_t)(3 * BN);
        float re[COLS], im[COLS];
        bool go = true;
        for (int seg = 0; seg < segments && go; ++seg) {
            // P0 and P1 complete: Re_s = P0 - P1 joins the running sum; P0 + P1
            // parks in the spare columns so both accumulators can be reused.
            bool ready = mbar_wait(&acc_full[1], seg & 1, p.status);
            tc_fence_after();
            go = __all_sync(0xffffffffu, ready && !*abort_flag);
            if (!go) {
                break;
            }
#pragma unroll
            for (int cb = 0; cb < COLS; cb += 8) {
                float v0[8], v1[8];
                tmem_ld8x2(lane_addr + (uint32_t)cb, lane_addr + (uint32_t)(BN + cb), v0, v1);
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const float rs = __fsub_rn(v0[j], v1[j]);
                    v1[j] = __fadd_rn(v0[j], v1[j]);
                    re[cb + j] = seg == 0 ? rs : __fadd_rn(re[cb + j], rs);
                }
                tmem_st8(spare + (uint32_t)cb, v1);
            }
            tmem_wait_st();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&acc_free[0]);
                mbar_arrive(&acc_free[1]);
            }
            // P2 complete: Im_s = P2 - (P0 + P1).
            ready = mbar_wait(&acc_full[2], seg & 1, p.status);
            tc_fence_after();
            go = __all_sync(0xffffffffu, ready && !*abort_flag);
            if (!go) {
                break;
            }
#pragma unroll
            for (int cb = 0; cb < COLS; cb += 8) {
                float v2[8], u[8];
                tmem_ld8x2(lane_addr + (uint32_t)(2 * BN + cb), spare + (uint32_t)cb, v2, u);
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const float is = __fsub_rn(v2[j], u[j]);
                    im[cb + j] = seg == 0 ? is : __fadd_rn(im[cb + j], is);
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&acc_free[2]);
            }
        }
        if (go && row < p.m) {
#pragma unroll
            for (int j = 0; j < COLS; ++j) {
                const int col = n0 + half * COLS + j;
                if (col < p.n) {
                    if (p.parts == 1) {
                        float2* cp = p.C + (size_t)col * p.ldc + row;
                        *cp = epilogue_value(re[j], im[j], p.epi, cp);
                    } else {
                        const size_t o = (size_t)col * p.ppitch + row;
                        p.partial[(size_t)(2 * part) * p.pplane + o] = re[j];
                        p.partial[(size_t)(2 * part + 1) * p.pplane + o] = im[j];
                    }
                }
            }
        }
    }
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, G::TMEM_COLS);
    }
}

// ---------------------------------------------------------------------------
// Risk path of the tensor-core forms' rounding pass: one CTA per 128 x 128
// output tile over the leading split plane of the real and imaginary
// components only (the sum planes are not read).  Per K-block one ring stage
// holds A_re, A_im, B_re, B_im (16 KB each) and one thread issues, per 32-byte
// K step,
//   Re += A_re B_re + (-A_im) B_im   (the second with the negate-A bit)
//   Im += A_re B_im + A_im B_re
// into TMEM columns [0, 128) and [128, 256); the running sums live in columns
// [256, 384) and [384, 512).  After every K segment the epilogue merges Re_s
// and Im_s into the running sums with round-to-nearest FP32 and advances both
// risk integrals of its 32 outputs (registers) by d/9 (s_old^2 + s_old s_new
// + s_new^2), as MergeProductsWithPath does (cgemm_compute_kernel.cpp:432-474).
// The four-multiplication products read 2.25x fewer operand bytes per output
// than the three-multiplication ones over 128 x 64 tiles (the register-resident
// running state of that form caps its tile width), and the risk estimate,
// which needs a few significant bits of the running sums, does not tell the
// two apart.  The K range is never partitioned: the risk plane needs the whole
// chain.  The epilogue then applies the selection itself (flag words, 16 x
// 16 tile counts, the flagged total); C and the risk plane are not written.
constexpr int kLeadBN = 128;
// 16 epilogue warps (four per TMEM lane quadrant, 32 columns each) hide the
// TMEM load latency four ways per sub-partition; 18 warps launch at up to 96
// registers a thread (five warps on the busiest sub-partition's 16K).
constexpr int kLeadEpiWarps = 16;
constexpr int kLeadThreads = (2 + kLeadEpiWarps) * 32;
constexpr int kLeadStage = 4 * A_PLANE;                 // 64 KB
constexpr int kLeadStages = RING_BYTES / kLeadStage;    // 3
constexpr size_t kLeadSmem = (size_t)kLeadStages * kLeadStage + 1024 + 256;
constexpr uint32_t kNegateA = 1u << 13;                 // instruction descriptor: negate the A operand

template <int LEAD>
__global__ void __launch_bounds__(kLeadThreads, 1)
    gemm3m_lead_path_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                            const TcParams p)
{
    using Cfg = TcCfg<LEAD>;
    constexpr int KSTEPS = ROW_BYTES / 32;
    constexpr int COLS = kLeadBN / (kLeadEpiWarps / 4);  // columns per epilogue thread

    extern __shared__ uint8_t smem_raw[];
    uint8_t* ring = align_shared<1024>(smem_raw);
    uint64_t* full = reinterpret_cast<uint64_t*>(ring + kLeadStages * kLeadStage);
    uint64_t* empty = full + kLeadStages;
    uint64_t* acc_full = empty + kLeadStages;  // MMA -> epilogue: Re_s and Im_s of the segment are in TMEM
    uint64_t* acc_free = acc_full + 1;         // epilogue -> MMA: both may be overwritten
    uint64_t* mma_done = acc_free + 1;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_done + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;

    constexpr int GM = 8;
    const int pid = blockIdx.x;
    const int in_group = GM * p.tiles_n;
    const int first_m = (pid / in_group) * GM;
    const int gsz = min(p.tiles_m - first_m, GM);
    const int tm = first_m + (pid % in_group) % gsz;
    const int tn = (pid % in_group) / gsz;
    const int m0 = tm * TILE_M, n0 = tn * kLeadBN;
    const int kblocks = (p.k + Cfg::BK - 1) / Cfg::BK;
    const int seg_blocks = p.seg_blocks;
    const int segments = (kblocks + seg_blocks - 1) / seg_blocks;

    if (tid == 0) {
        for (int s = 0; s < kLeadStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(acc_full, 1);
        mbar_init(acc_free, kLeadEpiWarps);
        mbar_init(mma_done, 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 1) {
        tmem_alloc(tmem_slot, 512);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        // ---------------- TMA producer: one stage per K-block ----------------
        if (lane == 0) {
            tma_prefetch_desc(&tmA);
            tma_prefetch_desc(&tmB);
            int it = 0;
            for (; it < kblocks; ++it) {
                const int s = it % kLeadStages;
                if ((it >= kLeadStages && !mbar_wait(&empty[s], ((it / kLeadStages) - 1) & 1, p.status)) ||
                    *abort_flag) {
                    *abort_flag = 1;
                    break;
                }
                uint8_t* st = ring + s * kLeadStage;
                const int k = it * Cfg::BK;
                mbar_arrive_expect_tx(&full[s], kLeadStage);
                tma_load_3d(st, &tmA, &full[s], k, m0, 0);
                tma_load_3d(st + A_PLANE, &tmA, &full[s], k, m0, Cfg::ZS);
                tma_load_3d(st + 2 * A_PLANE, &tmB, &full[s], k, n0, 0);
                tma_load_3d(st + 3 * A_PLANE, &tmB, &full[s], k, n0, Cfg::ZS);
            }
            for (int j = it > kLeadStages ? it - kLeadStages : 0; j < it; ++j) {
                mbar_wait(&full[j % kLeadStages], (j / kLeadStages) & 1, p.status);
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            const uint32_t idesc = instr_desc<Cfg::FMT, kLeadBN>();
            const uint32_t idesc_neg = idesc | kNegateA;
            const uint32_t d_re = tmem, d_im = tmem + (uint32_t)kLeadBN;
            int it = 0;
            bool stop = false;
            for (int seg = 0; seg < segments && !stop; ++seg) {
                if (seg > 0) {
                    if (!mbar_wait(acc_free, (seg - 1) & 1, p.status)) {
                        *abort_flag = 1;
                        break;
                    }
                    tc_fence_after();
                }
                const int kb0 = seg * seg_blocks, kb1 = min(kblocks, kb0 + seg_blocks);
                for (int kb = kb0; kb < kb1; ++kb, ++it) {
                    const int s = it % kLeadStages;
                    if (!mbar_wait(&full[s], (it / kLeadStages) & 1, p.status)) {
                        *abort_flag = 1;
                        stop = true;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t base = smem_u32(ring + s * kLeadStage);
#pragma unroll
                    for (int kk = 0; kk < KSTEPS; ++kk) {
                        const uint64_t a_re = smem_desc(base + kk * 32);
                        const uint64_t a_im = smem_desc(base + A_PLANE + kk * 32);
                        const uint64_t b_re = smem_desc(base + 2 * A_PLANE + kk * 32);
                        const uint64_t b_im = smem_desc(base + 3 * A_PLANE + kk * 32);
                        const uint32_t acc = (kb > kb0 || kk > 0) ? 1u : 0u;
                        if constexpr (Cfg::FMT == 2) {
                            umma_tf32(d_re, a_re, b_re, idesc, acc);
                            umma_tf32(d_re, a_im, b_im, idesc_neg, 1u);
                            umma_tf32(d_im, a_re, b_im, idesc, acc);
                            umma_tf32(d_im, a_im, b_re, idesc, 1u);
                        } else {
                            umma_f16(d_re, a_re, b_re, idesc, acc);
                            umma_f16(d_re, a_im, b_im, idesc_neg, 1u);
                            umma_f16(d_im, a_re, b_im, idesc, acc);
                            umma_f16(d_im, a_im, b_re, idesc, 1u);
                        }
                    }
                    umma_commit(&empty[s]);
                }
                if (!stop) {
                    umma_commit(acc_full);
                }
            }
            umma_commit(mma_done);
            mbar_wait(mma_done, 0, p.status);  // nothing may still write TMEM when it is freed
        }
    } else {
        // ---------------- epilogue warps 2.. ----------------
        // TMEM lane quadrant = warp % 4; warps 2-5 take the first COLS columns
        // of the tile, warps 6-9 the next, and so on.
        const int quad = warp & 3;
        const int group = (warp - 2) >> 2;
        const int row = m0 + quad * 32 + lane;
        const uint32_t lane_addr = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(group * COLS);
        const uint32_t seg_re = lane_addr, seg_im = lane_addr + kLeadBN;
        const uint32_t run_re = lane_addr + 2 * kLeadBN, run_im = lane_addr + 3 * kLeadBN;
        // Risk integrals by parts: with s_0 = 0 and equal weights w = d/9 on
        // the full segments,
        //   sum_{k<K} w (s_{k-1}^2 + s_{k-1} s_k + s_k^2)
        //     = w (sum_{k<K} s_k (2 s_k + s_{k-1}) - s_{K-1}^2),
        // so a full segment costs two FMAs per part and the last one (of depth
        // d_K <= d) closes the sum with the whole step of weight d_K / 9.
        float ir[COLS], ii[COLS];
        const float wfull = __fdiv_rn((float)(seg_blocks * Cfg::BK), 9.0f);
        bool go = true;
        for (int seg = 0; seg < segments && go; ++seg) {
            const int t0 = seg * seg_blocks * Cfg::BK;
            const int depth = min(p.k, t0 + seg_blocks * Cfg::BK) - t0;
            const float w = __fdiv_rn((float)depth, 9.0f);
            const bool last = seg == segments - 1;
            const bool ready = mbar_wait(acc_full, seg & 1, p.status);
            tc_fence_after();
            go = __all_sync(0xffffffffu, ready && !*abort_flag);
            if (!go) {
                break;
            }
            if (last) {
                lead_drain<COLS, 2>(seg_re, seg_im, run_re, run_im, seg == 0, w, wfull, ir, ii);
            } else if (seg == 0) {
                lead_drain<COLS, 0>(seg_re, seg_im, run_re, run_im, true, w, wfull, ir, ii);
            } else {
                lead_drain<COLS, 1>(seg_re, seg_im, run_re, run_im, false, w, wfull, ir, ii);
            }
            tmem_wait_st();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(acc_free);
            }
        }
        if (go) {
            // The selection (select_kernel's predicate on this product's sums and
            // risk plane): C and the risk plane are not written, as the form's
            // products or the exact recompute overwrite every output later.
            const bool row_ok = row < p.m;
            const float ei = row_ok ? __ldg(p.energy + row) : 0.0f;
            const int rbase = m0 + quad * 32;          // the warp's 32 rows
            const int cbase = n0 + group * COLS;       // this thread's 32 columns
            const bool words = (p.n & 31) == 0;        // then the warp's rows of a column are one flag word
            uint32_t cnt00 = 0, cnt01 = 0, cnt10 = 0, cnt11 = 0, total = 0;  // [row tile][column tile]
#pragma unroll
            for (int cb = 0; cb < COLS; cb += 8) {
                float re[8], im[8];
                tmem_ld8x2(run_re + (uint32_t)cb, run_im + (uint32_t)cb, re, im);
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int col = cbase + cb + j;
                    bool sel = false;
                    if (row_ok && col < p.n) {
                        const float ar = fabsf(re[j]), ai = fabsf(im[j]);
                        const float magnitude = ar > ai ? ar : ai;
                        const float risk = ir[cb + j] > ii[cb + j] ? ir[cb + j] : ii[cb + j];
                        const float ej = __ldg(p.energy + p.n + col);
                        const float variance =
                            __fmul_rn(0x1p-48f, __fadd_rn(risk, __fmul_rn(__fmul_rn(ei, ej), p.bridge)));
                        sel = !isfinite(magnitude) || !isfinite(variance) || __fmul_rn(p.conf2, variance) >= 0.0001f;
                    }
                    const uint32_t word = __ballot_sync(0xffffffffu, sel);
                    if (words) {
                        if (lane == 0 && col < p.n && rbase < p.m) {
                            p.flag_bits[((size_t)col * p.n + rbase) >> 5] = word;
                        }
                    } else if (sel) {
                        const size_t idx = (size_t)col * p.n + row;
                        atomicOr(&p.flag_bits[idx >> 5], 1u << (idx & 31));
                    }
                    const uint32_t lo = (uint32_t)__popc(word & 0xFFFFu), hi = (uint32_t)__popc(word >> 16);
                    if ((cb + j) < 16) {
                        cnt00 += lo;
                        cnt10 += hi;
                    } else {
                        cnt01 += lo;
                        cnt11 += hi;
                    }
                    total += lo + hi;
                }
            }
            if (lane == 0 && total != 0) {
                const int g16 = (p.n + 15) / 16;
                const size_t ti = (size_t)(rbase >> 4), tj = (size_t)(cbase >> 4);
                if (cnt00) atomicAdd(&p.tile_count[tj * g16 + ti], cnt00);
                if (cnt10) atomicAdd(&p.tile_count[tj * g16 + ti + 1], cnt10);
                if (cnt01) atomicAdd(&p.tile_count[(tj + 1) * g16 + ti], cnt01);
                if (cnt11) atomicAdd(&p.tile_count[(tj + 1) * g16 + ti + 1], cnt11);
                atomicAdd(&p.stats[kStatFlagged], total);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, 512);
    }
}

// ---------------------------------------------------------------------------
// CTA-pair variant (the main path): a cluster of two CTAs computes a 256 x 128
// output tile with cta_group::2 MMAs (M = 256).  CTA r holds rows
// [128r, 128r + 128) of the A tile and columns [64r, 64r + 64) of the B tile
// in its own shared memory; the even CTA's single MMA thread multiplies the
// pair's operands into both CTAs' TMEM (each CTA's accumulators hold its own
// 128 rows x all 128 columns).  Per CTA and K-block this moves 3/4 of the
// operand bytes of the single-CTA kernel for the same MMA work, which leaves
// room for a 3-stage ring (split-BF16) in 216 KB.
//   - both producers load into their own shared memory; the transaction bytes
//     of both land on the even CTA's `full` barrier, whose producer alone
//     arms it with the pair's byte count;
//   - MMA completion is committed to `empty`, `acc_full` and `mma_done` in
//     both CTAs (multicast commit); the odd CTA's epilogue warps arrive on the
//     even CTA's `acc_free` (16 arrivals per phase);
//   - TMEM (512 columns) is allocated and freed by warp 1 of both CTAs;
//   - a cluster barrier after set-up and before tear-down keeps both CTAs'
//     barriers and shared memory alive while the peer may use them.
// All mbarrier waits are bounded as in the single-CTA kernel.
constexpr int PAIR_BN = 128;       // N of the pair MMA (B columns per pair tile)
constexpr int PAIR_BHALF = 64;     // B columns staged by each CTA
constexpr int PAIR_RING = 216 * 1024;

template <int FORM>
struct PairGeom {
    using Cfg = TcCfg<FORM>;
    static constexpr int B_PLANE = PAIR_BHALF * ROW_BYTES;            // 8 KB
    static constexpr int STAGE_BYTES = Cfg::S * (A_PLANE + B_PLANE);   // per CTA
    static constexpr int STAGES = PAIR_RING / STAGE_BYTES;
    static constexpr int COLS = PAIR_BN / 2;
    static constexpr int TMEM_COLS = 4 * PAIR_BN;
    static constexpr size_t SMEM = (size_t)STAGES * STAGE_BYTES + 1024 + 256;
};

template <int FORM>
__global__ void __launch_bounds__(kThreads, 1)
    gemm3m_tc_pair_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                          const TcParams p)
{
    using Cfg = TcCfg<FORM>;
    using G = PairGeom<FORM>;
    constexpr int STAGES = G::STAGES;
    constexpr int STAGE_BYTES = G::STAGE_BYTES;
    constexpr int KSTEPS = ROW_BYTES / 32;
    constexpr int COLS = G::COLS;
    constexpr int BN = PAIR_BN;
    static_assert((size_t)2 * TILE_M * BN * sizeof(float) <= (size_t)STAGES * STAGE_BYTES,
                  "merge partials must fit the ring below the barriers");

    extern __shared__ uint8_t smem_raw[];
    uint8_t* ring = align_shared<1024>(smem_raw);
    uint64_t* full = reinterpret_cast<uint64_t*>(ring + STAGES * STAGE_BYTES);
    uint64_t* empty = full + STAGES;
    uint64_t* acc_full = empty + STAGES;  // [3]
    uint64_t* acc_free = acc_full + 3;    // [3] (used in the even CTA)
    uint64_t* mma_done = acc_free + 3;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_done + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    // The cluster is the CTA pair (1 x 2), or with an on-chip K merge the pairs
    // of all partitions of the tile (2 x parts): ranks 2q and 2q + 1 are the
    // pair of partition q, so the pair role is rank bit 0.
    const uint32_t crank = cluster_ctarank();
    const uint32_t rank = crank & 1u;     // role in the pair: 0 even (MMA issuer), 1 odd
    const uint32_t base = crank & ~1u;    // cluster rank of this pair's even CTA
    const uint16_t pair_mask = (uint16_t)(0x3u << base);
    const bool leader = rank == 0;
    __shared__ int merge_fail;

    constexpr int GM = 4;  // pair tiles per L2 group along m
    const int pid = blockIdx.x >> 1;
    const int tiles_m2 = p.tiles_m;  // pair tiles (256 rows) along m
    const int in_group = GM * p.tiles_n;
    const int first_m = (pid / in_group) * GM;
    const int gsz = min(tiles_m2 - first_m, GM);
    const int tm = first_m + (pid % in_group) % gsz;
    const int tn = (pid % in_group) / gsz;
    const int m0 = tm * 2 * TILE_M + (int)rank * TILE_M;  // this CTA's rows
    const int n0 = tn * BN;
    const int part = blockIdx.y;
    const int kbeg = part * p.span;
    const int kend = min(p.k, kbeg + p.span);
    const int kblocks = (kend - kbeg + Cfg::BK - 1) / Cfg::BK;
    const int seg_blocks = p.seg_blocks;
    const int segments = (kblocks + seg_blocks - 1) / seg_blocks;

    if (p.skip_count != nullptr) {
        // Rounding pass: the exact recompute writes every output of the
        // 256 x 256 tile holding this pair tile when one of its 16 x 16 count
        // tiles is dense (its own test, ozaki.cu); both CTAs read the same
        // counts and leave together, before any barrier or TMEM is touched.
        const int g16 = (p.n + 15) / 16;
        const int et = (tn * BN) / kOzakiTile;
        bool dense = false;
        if (tid < 256) {
            const int gi = tm * 16 + tid % 16;
            const int gj = et * 16 + tid / 16;
            if (gi < g16 && gj < g16) {
                dense = p.skip_count[(size_t)gj * g16 + gi] > kSparseMax;
            }
        }
        if (__syncthreads_or(dense)) {
            return;
        }
    }

    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int c = 0; c < 3; ++c) {
            mbar_init(&acc_full[c], 1);
            mbar_init(&acc_free[c], 2 * kEpilogueWarps);
        }
        mbar_init(mma_done, 1);
        *abort_flag = 0;
        merge_fail = 0;
        fence_mbar_init();
    }
    if (warp == 1) {
        tmem_alloc_pair(tmem_slot, G::TMEM_COLS);
        tmem_relinquish_pair();
    }
    tc_fence_before();
    cluster_sync();  // both CTAs' barriers initialised, TMEM allocated in both
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        // ---------------- TMA producer (both CTAs) ----------------
        if (lane == 0) {
            tma_prefetch_desc(&tmA);
            tma_prefetch_desc(&tmB);
            int it = 0;
            bool stop = false;
            for (int seg = 0; seg < segments && !stop; ++seg) {
                const int kb0 = seg * seg_blocks, kb1 = min(kblocks, kb0 + seg_blocks);
                for (int c = 0; c < 3 && !stop; ++c) {
                    for (int kb = kb0; kb < kb1; ++kb, ++it) {
                        const int s = it % STAGES;
                        if ((it >= STAGES && !mbar_wait(&empty[s], ((it / STAGES) - 1) & 1, p.status)) ||
                            *abort_flag) {
                            *abort_flag = 1;
                            stop = true;
                            break;
                        }
                        uint8_t* st = ring + s * STAGE_BYTES;
                        const uint32_t bar = mapa_shared(smem_u32(&full[s]), base);
                        if (leader) {
                            mbar_arrive_expect_tx(&full[s], 2 * STAGE_BYTES);
                        }
                        tma_load_3d_pair(st, &tmA, bar, kbeg + kb * Cfg::BK, m0, c * Cfg::ZS);
                        tma_load_3d_pair(st + Cfg::S * A_PLANE, &tmB, bar, kbeg + kb * Cfg::BK,
                                         n0 + (int)rank * PAIR_BHALF, c * Cfg::ZS);
                    }
                }
            }
            if (leader) {
                for (int j = it > STAGES ? it - STAGES : 0; j < it; ++j) {
                    mbar_wait(&full[j % STAGES], (j / STAGES) & 1, p.status);
                }
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer (even CTA) ----------------
        if (leader && lane == 0) {
            const uint32_t idesc = (1u << 4) | (Cfg::FMT << 7) | (Cfg::FMT << 10) | ((uint32_t)(BN >> 3) << 17) |
                                   ((uint32_t)((2 * TILE_M) >> 4) << 24);
            int it = 0;
            bool stop = false;
            for (int seg = 0; seg < segments && !stop; ++seg) {
                const int kb0 = seg * seg_blocks, kb1 = min(kblocks, kb0 + seg_blocks);
                for (int c = 0; c < 3 && !stop; ++c) {
                    if (seg > 0) {
                        if (!mbar_wait_cluster(&acc_free[c], (seg - 1) & 1, p.status)) {
                            *abort_flag = 1;
                            stop = true;
                            break;
                        }
                        tc_fence_after();
                    }
                    const uint32_t d = tmem + (uint32_t)(c * BN);
                    for (int kb = kb0; kb < kb1; ++kb, ++it) {
                        const int s = it % STAGES;
                        if (!mbar_wait(&full[s], (it / STAGES) & 1, p.status)) {
                            *abort_flag = 1;
                            stop = true;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t a_base = smem_u32(ring + s * STAGE_BYTES);
                        const uint32_t b_base = a_base + Cfg::S * A_PLANE;
#pragma unroll
                        for (int kk = 0; kk < KSTEPS; ++kk) {
#pragma unroll
                            for (int q = 0; q < Cfg::NPAIRS; ++q) {
                                const int2 ij = Cfg::pair(q);
                                const uint64_t ad = smem_desc(a_base + ij.x * A_PLANE + kk * 32);
                                const uint64_t bd = smem_desc(b_base + ij.y * G::B_PLANE + kk * 32);
                                const uint32_t acc = (kb > kb0 || kk > 0 || q > 0) ? 1u : 0u;
                                if constexpr (Cfg::FMT == 2) {
                                    umma_tf32_pair(d, ad, bd, idesc, acc);
                                } else {
                                    umma_f16_pair(d, ad, bd, idesc, acc);
                                }
                            }
                        }
                        umma_commit_pair(&empty[s], pair_mask);
                    }
                    if (!stop && c > 0) {
                        umma_commit_pair(&acc_full[c], pair_mask);
                    }
                }
            }
            umma_commit_pair(mma_done, pair_mask);
            mbar_wait(mma_done, 0, p.status);  // nothing may still write TMEM when it is freed
        }
    } else {
        // ---------------- epilogue warps 2..9 (both CTAs) ----------------
        const int quad = warp & 3;
        const int half = (warp - 2) >> 2;
        const int row = m0 + quad * 32 + lane;
        const uint32_t lane_addr = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(half * COLS);
        const uint32_t spare = lane_addr + (uint32_t)(3 * BN);
        const uint32_t free0 = mapa_shared(smem_u32(&acc_free[0]), base);
        const uint32_t free1 = mapa_shared(smem_u32(&acc_free[1]), base);
        const uint32_t free2 = mapa_shared(smem_u32(&acc_free[2]), base);
        float re[COLS], im[COLS];
        bool go = true;
        for (int seg = 0; seg < segments && go; ++seg) {
            bool ready = mbar_wait(&acc_full[1], seg & 1, p.status);
            tc_fence_after();
            go = __all_sync(0xffffffffu, ready && !*abort_flag);
            if (!go) {
                break;
            }
#pragma unroll
            for (int cb = 0; cb < COLS; cb += 8) {
                float v0[8], v1[8];
                tmem_ld8x2(lane_addr + (uint32_t)cb, lane_addr + (uint32_t)(BN + cb), v0, v1);
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const float rs = __fsub_rn(v0[j], v1[j]);
                    v1[j] = __fadd_rn(v0[j], v1[j]);
                    re[cb + j] = seg == 0 ? rs : __fadd_rn(re[cb + j], rs);
                }
                tmem_st8(spare + (uint32_t)cb, v1);
            }
            tmem_wait_st();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive_cluster(free0);
                mbar_arrive_cluster(free1);
            }
            ready = mbar_wait(&acc_full[2], seg & 1, p.status);
            tc_fence_after();
            go = __all_sync(0xffffffffu, ready && !*abort_flag);
            if (!go) {
                break;
            }
#pragma unroll
            for (int cb = 0; cb < COLS; cb += 8) {
                float v2[8], u[8];
                tmem_ld8x2(lane_addr + (uint32_t)(2 * BN + cb), spare + (uint32_t)cb, v2, u);
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const float is = __fsub_rn(v2[j], u[j]);
                    im[cb + j] = seg == 0 ? is : __fadd_rn(im[cb + j], is);
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive_cluster(free2);
            }
        }
        if (p.cluster_merge) {
            // This partition's (Re, Im) of the CTA's 128 rows x 128 columns go to
            // the ring, free once the last segment's products are read (every
            // MMA, and so every copy into the ring, is complete by then).
            if (!go) {
                merge_fail = 1;
            } else {
                float* part_re = reinterpret_cast<float*>(ring);
                float* part_im = part_re + TILE_M * BN;
                const int rl = quad * 32 + lane;
#pragma unroll
                for (int j = 0; j < COLS; ++j) {
                    const int cl = half * COLS + j;
                    part_re[cl * TILE_M + rl] = re[j];
                    part_im[cl * TILE_M + rl] = im[j];
                }
            }
        } else if (go && row < p.m) {
#pragma unroll
            for (int j = 0; j < COLS; ++j) {
                const int col = n0 + half * COLS + j;
                if (col < p.n) {
                    if (p.parts == 1) {
                        float2* cp = p.C + (size_t)col * p.ldc + row;
                        *cp = epilogue_value(re[j], im[j], p.epi, cp);
                    } else {
                        const size_t o = (size_t)col * p.ppitch + row;
                        p.partial[(size_t)(2 * part) * p.pplane + o] = re[j];
                        p.partial[(size_t)(2 * part + 1) * p.pplane + o] = im[j];
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    cluster_sync();  // the even CTA's MMAs are complete; neither CTA's memory is used any more
    if (p.cluster_merge) {
        // K merge across the tile's pairs: CTA (pair role r, partition q) sums
        // the q-th slice of its 128 x 128 half-tile over partitions 0, 1, ... in
        // order (the merge kernel's arithmetic), reading the same role's CTA of
        // every partition (cluster rank r + 2q'), then applies alpha/beta.
        // Every thread of every CTA reaches both cluster barriers.
        const uint32_t re_local = smem_u32(ring), im_local = re_local + 4u * TILE_M * BN;
        int bad = 0;
        for (int q = 0; q < p.parts; ++q) {
            const uint32_t peer = rank + 2u * (uint32_t)q;
            bad |= ld_dsmem_s32(mapa_shared(smem_u32(&merge_fail), peer));
            bad |= ld_dsmem_s32(mapa_shared(smem_u32((const void*)abort_flag), peer));
        }
        if (!bad) {
            const int per = (TILE_M * BN + p.parts - 1) / p.parts;
            const int e_end = min(TILE_M * BN, (part + 1) * per);
            for (int e = part * per + tid; e < e_end; e += kThreads) {
                const int rl = e % TILE_M, cl = e / TILE_M;
                const int row = m0 + rl, col = n0 + cl;
                if (row >= p.m || col >= p.n) {
                    continue;
                }
                float vre = ld_dsmem_f32(mapa_shared(re_local + 4u * e, rank));
                float vim = ld_dsmem_f32(mapa_shared(im_local + 4u * e, rank));
                for (int q = 1; q < p.parts; ++q) {
                    const uint32_t peer = rank + 2u * (uint32_t)q;
                    vre = __fadd_rn(vre, ld_dsmem_f32(mapa_shared(re_local + 4u * e, peer)));
                    vim = __fadd_rn(vim, ld_dsmem_f32(mapa_shared(im_local + 4u * e, peer)));
                }
                float2* cp = p.C + (size_t)col * p.ldc + row;
                *cp = epilogue_value(vre, vim, p.epi, cp);
            }
        }
        cluster_sync();  // no CTA leaves while others may still read its shared memory
    }
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc_pair(tmem, G::TMEM_COLS);
    }
}

template <int FORM>
cudaError_t launch_pair(cudaStream_t stream, const Problem& pr, const Plan& plan, void* ws, int* status,
                        const uint32_t* skip_count = nullptr)
{
    using Cfg = TcCfg<FORM>;
    using G = PairGeom<FORM>;
    const bool bf16 = Cfg::FMT == 1;
    const size_t elem = bf16 ? 2 : 4;
    uint8_t* w = static_cast<uint8_t*>(ws);
    CUtensorMap ta, tb;
    const CUtensorMapDataType dt = bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    {
        const uint64_t dims[3] = {(uint64_t)pr.k, (uint64_t)pr.m, (uint64_t)(3 * Cfg::ZS)};
        const uint64_t strides[2] = {(uint64_t)plan.pitch_a * elem, (uint64_t)plan.plane_a_elems * elem};
        const uint32_t box[3] = {(uint32_t)Cfg::BK, (uint32_t)TILE_M, (uint32_t)Cfg::S};
        if (!encode_tensor_map(&ta, dt, 3, dims, strides, box, CU_TENSOR_MAP_SWIZZLE_128B, w + plan.planes_a_off)) {
            return cudaErrorInvalidValue;
        }
    }
    {
        const uint64_t dims[3] = {(uint64_t)pr.k, (uint64_t)pr.n, (uint64_t)(3 * Cfg::ZS)};
        const uint64_t strides[2] = {(uint64_t)plan.pitch_b * elem, (uint64_t)plan.plane_b_elems * elem};
        const uint32_t box[3] = {(uint32_t)Cfg::BK, (uint32_t)PAIR_BHALF, (uint32_t)Cfg::S};
        if (!encode_tensor_map(&tb, dt, 3, dims, strides, box, CU_TENSOR_MAP_SWIZZLE_128B, w + plan.planes_b_off)) {
            return cudaErrorInvalidValue;
        }
    }
    TcParams p{};
    p.m = pr.m;
    p.n = pr.n;
    p.k = pr.k;
    p.span = plan.span;
    p.parts = plan.parts;
    p.tiles_m = ceil_div(pr.m, 2 * TILE_M);  // pair tiles
    p.tiles_n = ceil_div(pr.n, PAIR_BN);
    p.epi = EpiParams{pr.ar, pr.ai, pr.br, pr.bi, plan.unit ? 1 : 0, plan.beta_zero ? 1 : 0};
    p.C = static_cast<float2*>(pr.C);
    p.ldc = pr.ldc;
    p.partial = reinterpret_cast<float*>(w + plan.partial_off);
    p.ppitch = plan.partial_pitch;
    p.pplane = plan.partial_plane_elems;
    p.status = status;
    p.seg_blocks = plan.tc_segment > 0 ? (plan.tc_segment + Cfg::BK - 1) / Cfg::BK : 64 / Cfg::BK;
    if (p.seg_blocks < 1) {
        p.seg_blocks = 1;
    }
    p.skip_count = skip_count;
    p.cluster_merge = plan.cluster_merge ? 1 : 0;
    if (p.cluster_merge && (plan.parts < 2 || plan.parts > 4)) {
        return cudaErrorInvalidValue;  // clusters of at most 8 CTAs: up to 4 pairs
    }
    static_assert((size_t)2 * TILE_M * PAIR_BN * sizeof(float) <= (size_t)PAIR_RING,
                  "merge partials exceed the ring");
    auto kernel = gemm3m_tc_pair_kernel<FORM>;
    cudaError_t err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::SMEM);
    if (err != cudaSuccess) {
        return err;
    }
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)(2 * p.tiles_m * p.tiles_n), (unsigned)plan.parts);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = G::SMEM;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = p.cluster_merge ? (unsigned)plan.parts : 1u;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    err = cudaLaunchKernelEx(&cfg, kernel, ta, tb, p);
    return err != cudaSuccess ? err : cudaGetLastError();
}

template <int FORM, int BN>
cudaError_t launch_form(cudaStream_t stream, const Problem& pr, const Plan& plan, void* ws, int* status)
{
    using Cfg = TcCfg<FORM>;
    using G = TcGeom<FORM, BN>;
    const bool bf16 = Cfg::FMT == 1;
    const size_t elem = bf16 ? 2 : 4;
    uint8_t* w = static_cast<uint8_t*>(ws);
    CUtensorMap ta, tb;
    const CUtensorMapDataType dt = bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    {
        const uint64_t dims[3] = {(uint64_t)pr.k, (uint64_t)pr.m, (uint64_t)(3 * Cfg::ZS)};
        const uint64_t strides[2] = {(uint64_t)plan.pitch_a * elem, (uint64_t)plan.plane_a_elems * elem};
        const uint32_t box[3] = {(uint32_t)Cfg::BK, (uint32_t)TILE_M, (uint32_t)Cfg::S};
        if (!encode_tensor_map(&ta, dt, 3, dims, strides, box, CU_TENSOR_MAP_SWIZZLE_128B, w + plan.planes_a_off)) {
            return cudaErrorInvalidValue;
        }
    }
    {
        const uint64_t dims[3] = {(uint64_t)pr.k, (uint64_t)pr.n, (uint64_t)(3 * Cfg::ZS)};
        const uint64_t strides[2] = {(uint64_t)plan.pitch_b * elem, (uint64_t)plan.plane_b_elems * elem};
        const uint32_t box[3] = {(uint32_t)Cfg::BK, (uint32_t)BN, (uint32_t)Cfg::S};
        if (!encode_tensor_map(&tb, dt, 3, dims, strides, box, CU_TENSOR_MAP_SWIZZLE_128B, w + plan.planes_b_off)) {
            return cudaErrorInvalidValue;
        }
    }
    TcParams p{};
    p.m = pr.m;
    p.n = pr.n;
    p.k = pr.k;
    p.span = plan.span;
    p.parts = plan.parts;
    p.tiles_m = ceil_div(pr.m, TILE_M);
    p.tiles_n = ceil_div(pr.n, BN);
    p.epi = EpiParams{pr.ar, pr.ai, pr.br, pr.bi, plan.unit ? 1 : 0, plan.beta_zero ? 1 : 0};
    p.C = static_cast<float2*>(pr.C);
    p.ldc = pr.ldc;
    p.partial = reinterpret_cast<float*>(w + plan.partial_off);
    p.ppitch = plan.partial_pitch;
    p.pplane = plan.partial_plane_elems;
    p.status = status;
    p.seg_blocks = plan.tc_segment > 0 ? (plan.tc_segment + Cfg::BK - 1) / Cfg::BK : 64 / Cfg::BK;
    if (p.seg_blocks < 1) {
        p.seg_blocks = 1;
    }
    auto kernel = gemm3m_tc_kernel<FORM, BN>;
    cudaError_t err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::SMEM);
    if (err != cudaSuccess) {
        return err;
    }
    const dim3 grid((unsigned)(p.tiles_m * p.tiles_n), (unsigned)plan.parts);
    kernel<<<grid, kThreads, G::SMEM, stream>>>(ta, tb, p);
    return cudaGetLastError();
}

template <int LEAD>
cudaError_t launch_lead_path(cudaStream_t stream, const Problem& pr, const Plan& plan, void* ws, int* status,
                             const LeadSelect& sel)
{
    using Cfg = TcCfg<LEAD>;
    const bool bf16 = Cfg::FMT == 1;
    const size_t elem = bf16 ? 2 : 4;
    uint8_t* w = static_cast<uint8_t*>(ws);
    CUtensorMap ta, tb;
    const CUtensorMapDataType dt = bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    {
        const uint64_t dims[3] = {(uint64_t)pr.k, (uint64_t)pr.m, (uint64_t)(3 * Cfg::ZS)};
        const uint64_t strides[2] = {(uint64_t)plan.pitch_a * elem, (uint64_t)plan.plane_a_elems * elem};
        const uint32_t box[3] = {(uint32_t)Cfg::BK, (uint32_t)TILE_M, 1u};
        if (!encode_tensor_map(&ta, dt, 3, dims, strides, box, CU_TENSOR_MAP_SWIZZLE_128B, w + plan.planes_a_off)) {
            return cudaErrorInvalidValue;
        }
    }
    {
        const uint64_t dims[3] = {(uint64_t)pr.k, (uint64_t)pr.n, (uint64_t)(3 * Cfg::ZS)};
        const uint64_t strides[2] = {(uint64_t)plan.pitch_b * elem, (uint64_t)plan.plane_b_elems * elem};
        const uint32_t box[3] = {(uint32_t)Cfg::BK, (uint32_t)kLeadBN, 1u};
        if (!encode_tensor_map(&tb, dt, 3, dims, strides, box, CU_TENSOR_MAP_SWIZZLE_128B, w + plan.planes_b_off)) {
            return cudaErrorInvalidValue;
        }
    }
    TcParams p{};
    p.m = pr.m;
    p.n = pr.n;
    p.k = pr.k;
    p.span = pr.k;
    p.parts = 1;
    p.tiles_m = ceil_div(pr.m, TILE_M);
    p.tiles_n = ceil_div(pr.n, kLeadBN);
    p.epi = EpiParams{pr.ar, pr.ai, pr.br, pr.bi, plan.unit ? 1 : 0, plan.beta_zero ? 1 : 0};
    p.C = static_cast<float2*>(pr.C);
    p.ldc = pr.ldc;
    p.status = status;
    p.seg_blocks = plan.tc_segment > 0 ? (plan.tc_segment + Cfg::BK - 1) / Cfg::BK : 64 / Cfg::BK;
    if (p.seg_blocks < 1) {
        p.seg_blocks = 1;
    }
    p.energy = sel.energy;
    p.bridge = sel.bridge;
    p.conf2 = sel.conf2;
    p.flag_bits = sel.flag_bits;
    p.tile_count = sel.tile_count;
    p.stats = sel.stats;
    auto kernel = gemm3m_lead_path_kernel<LEAD>;
    cudaError_t err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLeadSmem);
    if (err != cudaSuccess) {
        return err;
    }
    kernel<<<(unsigned)(p.tiles_m * p.tiles_n), kLeadThreads, kLeadSmem, stream>>>(ta, tb, p);
    return cudaGetLastError();
}

}  // namespace

#ifndef CG3M_TC_PAIR
#define CG3M_TC_PAIR 1
#endif

cudaError_t launch_gemm_tc(cudaStream_t stream, const Problem& pr, const Plan& plan, void* ws, int* status)
{
    // CTA pairs whenever the output has more than one 128-row tile; a single
    // row tile would leave the odd CTA of every pair without rows.
    if (CG3M_TC_PAIR && pr.m > TILE_M) {
        switch (plan.form) {
            case CG3M_FORM_TF32X3: return launch_pair<CG3M_FORM_TF32X3>(stream, pr, plan, ws, status);
            case CG3M_FORM_BF16X6: return launch_pair<CG3M_FORM_BF16X6>(stream, pr, plan, ws, status);
            case CG3M_FORM_BF16X9: return launch_pair<CG3M_FORM_BF16X9>(stream, pr, plan, ws, status);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (plan.form) {
        case CG3M_FORM_TF32X3: return launch_form<CG3M_FORM_TF32X3, 128>(stream, pr, plan, ws, status);
        case CG3M_FORM_BF16X6: return launch_form<CG3M_FORM_BF16X6, 128>(stream, pr, plan, ws, status);
        case CG3M_FORM_BF16X9: return launch_form<CG3M_FORM_BF16X9, 128>(stream, pr, plan, ws, status);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_gemm_tc_path(cudaStream_t stream, const Problem& pr, const Plan& plan, void* ws,
                                const LeadSelect& sel, int* status)
{
    switch (plan.form) {
        case CG3M_FORM_TF32X3: return launch_lead_path<kLeadTf32>(stream, pr, plan, ws, status, sel);
        case CG3M_FORM_BF16X6:
        case CG3M_FORM_BF16X9: return launch_lead_path<kLeadBf16>(stream, pr, plan, ws, status, sel);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_gemm_tc_tiles(cudaStream_t stream, const Problem& pr, const Plan& plan, void* ws, int* status,
                                 const uint32_t* tile_count)
{
    if (!CG3M_TC_PAIR || pr.m <= TILE_M || plan.parts != 1 || tile_count == nullptr) {
        return cudaErrorInvalidValue;  // the rounding pass's orders (2048..4096) always have two row tiles
    }
    switch (plan.form) {
        case CG3M_FORM_TF32X3: return launch_pair<CG3M_FORM_TF32X3>(stream, pr, plan, ws, status, tile_count);
        case CG3M_FORM_BF16X6: return launch_pair<CG3M_FORM_BF16X6>(stream, pr, plan, ws, status, tile_count);
        case CG3M_FORM_BF16X9: return launch_pair<CG3M_FORM_BF16X9>(stream, pr, plan, ws, status, tile_count);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace cg3m
