// gemm_fp32.cu -- plain FP32 3M GEMM (the drop-in form), its split-K merge and
// the beta-only scaling kernel.
//
// Reference counterparts:
//   products  gemm_cgemm_products_kernel  blas/gemm/arch35/cgemm_compute_kernel.cpp:350-366
//   fused     gemm_cgemm_fused_kernel                         cgemm_compute_kernel.cpp:879-896
//   epilogue  gemm_cgemm_epilogue_kernel / CgemmEpilogueVf     cgemm_epilogue_kernel.cpp:232-332
//   alpha=0   HandleCgemmAlphaZero                            cgemm_host.cpp:636-663
//
// B200 design.  One CTA owns a BM x BN tile of complex outputs and computes all
// three real products of it on the CUDA cores with FFMA, so the epilogue
// (Re = P0-P1, Im = (P2-P0)-P1, alpha, beta, interleave, ldc store) runs from
// registers with no workspace round trip -- the reference's "fused" kernel for
// every alpha/beta.  Operand planes (Ar, Ai, Ar+Ai / Br, Bi, Br+Bi, MN-major)
// are staged by TMA: one 3-D box per operand per K-tile carries all three
// planes, into a STAGES-deep ring guarded by full/empty mbarriers.  A producer
// warp issues the copies; the consumer warps each own a 32x32 sub-tile, every
// thread an 8 x 4 complex micro-tile (96 FP32 accumulators).  Each output's
// K terms are accumulated by one thread in increasing k -- a fixed order, so
// results are bitwise reproducible.  For long-K, few-tile shapes the K range is
// split into partitions (grid.y); each writes (Re_p, Im_p) planes and a merge
// kernel sums them in partition order before alpha/beta.
#include "cg3m_internal.h"
#include "epilogue.cuh"
#include "ptx.cuh"

namespace cg3m {

namespace {

struct Fp32Params {
    int m, n, k;
    int span, parts;
    int tiles_m, tiles_n;
    EpiParams epi;
    float2* C;
    int ldc;
    float* partial;  // [part][2][n][ppitch]
    int ppitch;
    size_t pplane;
    int* status;
    int cluster_merge;  // the `parts` partitions of a tile form one cluster and merge on chip
};

template <int BM, int BN>
struct Fp32Cfg {
    static constexpr int BK = 16;
    static constexpr int STAGES = 4;
    static constexpr int WARPS_M = BM / 32;
    static constexpr int WARPS_N = BN / 32;
    static constexpr int CONSUMER_WARPS = WARPS_M * WARPS_N;
    static constexpr int THREADS = (CONSUMER_WARPS + 1) * 32;
    static constexpr int A_STAGE = 3 * BK * BM;  // floats
    static constexpr int B_STAGE = 3 * BK * BN;
    static constexpr size_t SMEM = size_t(STAGES) * (A_STAGE + B_STAGE) * 4 + 2 * STAGES * 8 + 1024;
};

template <int BM, int BN>
__global__ void __launch_bounds__(Fp32Cfg<BM, BN>::THREADS, 1)
    gemm3m_fp32_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                       const Fp32Params p)
{
    using Cfg = Fp32Cfg<BM, BN>;
    constexpr int BK = Cfg::BK, STAGES = Cfg::STAGES;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* base = align_shared<1024>(smem_raw);
    float* sA = reinterpret_cast<float*>(base);
    float* sB = sA + STAGES * Cfg::A_STAGE;
    uint64_t* full = reinterpret_cast<uint64_t*>(sB + STAGES * Cfg::B_STAGE);
    uint64_t* empty = full + STAGES;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;

    // Grouped rasterisation: 8 row-tiles per group keeps the operand panels of
    // concurrently running CTAs resident in L2.
    constexpr int GM = 8;
    const int pid = blockIdx.x;
    const int in_group = GM * p.tiles_n;
    const int first_m = (pid / in_group) * GM;
    const int gsz = min(p.tiles_m - first_m, GM);
    const int tm = first_m + (pid % in_group) % gsz;
    const int tn = (pid % in_group) / gsz;
    const int m0 = tm * BM, n0 = tn * BN;
    const int part = blockIdx.y;
    const int kbeg = part * p.span;
    const int kend = min(p.k, kbeg + p.span);
    const int ktiles = (kend - kbeg + BK - 1) / BK;

    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], Cfg::CONSUMER_WARPS);
        }
        fence_mbar_init();
    }
    __syncthreads();

    if (warp == Cfg::CONSUMER_WARPS) {
        // ---------------- producer ----------------
        if (lane == 0) {
            tma_prefetch_desc(&tmA);
            tma_prefetch_desc(&tmB);
            int issued = 0;
            for (int kt = 0; kt < ktiles; ++kt) {
                const int s = kt % STAGES;
                if (kt >= STAGES && !mbar_wait(&empty[s], ((kt / STAGES) - 1) & 1, p.status)) {
                    break;
                }
                mbar_arrive_expect_tx(&full[s], (Cfg::A_STAGE + Cfg::B_STAGE) * 4);
                tma_load_3d(sA + s * Cfg::A_STAGE, &tmA, &full[s], m0, kbeg + kt * BK, 0);
                tma_load_3d(sB + s * Cfg::B_STAGE, &tmB, &full[s], n0, kbeg + kt * BK, 0);
                ++issued;
            }
            // Drain: the last STAGES copies may still be landing in shared memory.
            for (int kt = issued > STAGES ? issued - STAGES : 0; kt < issued; ++kt) {
                mbar_wait(&full[kt % STAGES], (kt / STAGES) & 1, p.status);
            }
        }
    } else {
        // ---------------- consumers ----------------
        const int wm = warp % Cfg::WARPS_M, wn = warp / Cfg::WARPS_M;
        const int lm = lane & 3, ln = lane >> 2;
        const int tm0 = wm * 32 + lm * 8;  // 8 rows
        const int tn0 = wn * 32 + ln * 4;  // 4 columns
        float p0[8][4], p1[8][4], p2[8][4];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                p0[i][j] = 0.0f;
                p1[i][j] = 0.0f;
                p2[i][j] = 0.0f;
            }
        }
        bool ok = true;
        for (int kt = 0; kt < ktiles; ++kt) {
            const int s = kt % STAGES;
            if (!mbar_wait(&full[s], (kt / STAGES) & 1, p.status)) {
                ok = false;
                break;
            }
            const float* a = sA + s * Cfg::A_STAGE + tm0;
            const float* b = sB + s * Cfg::B_STAGE + tn0;
#pragma unroll
            for (int kk = 0; kk < BK; ++kk) {
                float x[8], y[4];
                // plane 0: Ar * Br
                *reinterpret_cast<float4*>(&x[0]) = *reinterpret_cast<const float4*>(a + kk * BM);
                *reinterpret_cast<float4*>(&x[4]) = *reinterpret_cast<const float4*>(a + kk * BM + 4);
                *reinterpret_cast<float4*>(&y[0]) = *reinterpret_cast<const float4*>(b + kk * BN);
#pragma unroll
                for (int i = 0; i < 8; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) p0[i][j] = __fmaf_rn(x[i], y[j], p0[i][j]);
                // plane 1: Ai * Bi
                *reinterpret_cast<float4*>(&x[0]) = *reinterpret_cast<const float4*>(a + (BK + kk) * BM);
                *reinterpret_cast<float4*>(&x[4]) = *reinterpret_cast<const float4*>(a + (BK + kk) * BM + 4);
                *reinterpret_cast<float4*>(&y[0]) = *reinterpret_cast<const float4*>(b + (BK + kk) * BN);
#pragma unroll
                for (int i = 0; i < 8; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) p1[i][j] = __fmaf_rn(x[i], y[j], p1[i][j]);
                // plane 2: (Ar+Ai) * (Br+Bi)
                *reinterpret_cast<float4*>(&x[0]) = *reinterpret_cast<const float4*>(a + (2 * BK + kk) * BM);
                *reinterpret_cast<float4*>(&x[4]) = *reinterpret_cast<const float4*>(a + (2 * BK + kk) * BM + 4);
                *reinterpret_cast<float4*>(&y[0]) = *reinterpret_cast<const float4*>(b + (2 * BK + kk) * BN);
#pragma unroll
                for (int i = 0; i < 8; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) p2[i][j] = __fmaf_rn(x[i], y[j], p2[i][j]);
            }
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&empty[s]);
            }
        }
        if (ok) {
            const int row0 = m0 + tm0, col0 = n0 + tn0;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int col = col0 + j;
                if (col >= p.n) {
                    continue;
                }
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int row = row0 + i;
                    if (row >= p.m) {
                        continue;
                    }
                    const float re = __fsub_rn(p0[i][j], p1[i][j]);
                    const float im = __fsub_rn(__fsub_rn(p2[i][j], p0[i][j]), p1[i][j]);
                    if (p.parts == 1) {
                        float2* cp = p.C + (size_t)col * p.ldc + row;
                        *cp = epilogue_at(re, im, p.epi, cp, row, col);
                    } else {
                        const size_t o = (size_t)col * p.ppitch + row;
                        p.partial[(size_t)(2 * part) * p.pplane + o] = re;
                        p.partial[(size_t)(2 * part + 1) * p.pplane + o] = im;
                    }
                }
            }
        }
    }
    __syncthreads();  // no CTA retires while its copies may still land
}

// ---------------------------------------------------------------------------
// Warp-specialised 128 x 64 variant (the packed engine's tile).  A warp's
// 128-bit shared-memory load costs four wavefronts whether or not its lanes
// share addresses, so the 8 x 4 complex micro-tile above (nine loads per 96
// FFMA) is bound by shared-memory wavefronts at about two thirds of the FFMA
// rate.  Here each of the three real products P0 = Ar.Br, P1 = Ai.Bi,
// P2 = (Ar+Ai).(Br+Bi) has its own four consumer warps, and every thread an
// 8 x 8 real micro-tile of one product: four 128-bit loads per 64 FMAs, the
// ratio at which the SM's FMA pipe and shared-memory wavefronts balance.  The
// FMAs issue as 32 packed pairs (two independent FP32 FMAs per instruction,
// each rounded to nearest), which halves the issue slots they take.
// Each product's K terms are still one thread's FFMA chain in increasing k,
// so the bits are those of the kernel above.  After the K loop the three
// products meet in shared memory (over the drained stage ring) and all 384
// consumer threads form Re = P0 - P1, Im = (P2 - P0) - P1, apply alpha/beta
// and store with coalesced column-major writes.
// ---------------------------------------------------------------------------
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

#ifndef CG3M_FP32_WS_UNROLL
#define CG3M_FP32_WS_UNROLL 16
#endif
namespace ws {
constexpr int BM = 128, BN = 64, BK = 16, STAGES = 4;
constexpr int KK_UNROLL = CG3M_FP32_WS_UNROLL;  // K terms per unrolled step (16 measured fastest)
constexpr int WARPS = 12;  // 4 per product; thread 0 also issues the copies
constexpr int THREADS = WARPS * 32;
constexpr int A_STAGE = 3 * BK * BM, B_STAGE = 3 * BK * BN;  // floats
constexpr size_t RING = size_t(STAGES) * (A_STAGE + B_STAGE) * 4;
constexpr size_t SMEM = RING + 2 * STAGES * 8 + 1024;
static_assert((size_t)3 * BM * BN * 4 <= RING, "product exchange exceeds the stage ring");
}  // namespace ws

// Twelve warps fall three to each of the SM's four sub-partitions (16K
// registers each), so 168 registers per thread is the launch limit; a
// thirteenth (producer) warp would cut it to 128.  Thread 0 therefore issues
// the TMA copies itself: the first STAGES K-tiles up front, then the refill of
// each stage once every warp has released it.
__global__ void __launch_bounds__(ws::THREADS, 1)
    gemm3m_fp32_ws_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                          const Fp32Params p)
{
    using namespace ws;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* base = align_shared<1024>(smem_raw);
    float* sA = reinterpret_cast<float*>(base);
    float* sB = sA + STAGES * A_STAGE;
    uint64_t* full = reinterpret_cast<uint64_t*>(sB + STAGES * B_STAGE);
    uint64_t* empty = full + STAGES;
    __shared__ int failed;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;

    constexpr int GM = 8;  // grouped rasterisation, as the kernel above
    const int pid = blockIdx.x;
    const int in_group = GM * p.tiles_n;
    const int first_m = (pid / in_group) * GM;
    const int gsz = min(p.tiles_m - first_m, GM);
    const int tm = first_m + (pid % in_group) % gsz;
    const int tn = (pid % in_group) / gsz;
    const int m0 = tm * BM, n0 = tn * BN;
    const int part = blockIdx.y;
    const int kbeg = part * p.span;
    const int kend = min(p.k, kbeg + p.span);
    const int ktiles = (kend - kbeg + BK - 1) / BK;

    auto issue = [&](int kt) {
        const int s = kt % STAGES;
        mbar_arrive_expect_tx(&full[s], (A_STAGE + B_STAGE) * 4);
        tma_load_3d(sA + s * A_STAGE, &tmA, &full[s], m0, kbeg + kt * BK, 0);
        tma_load_3d(sB + s * B_STAGE, &tmB, &full[s], n0, kbeg + kt * BK, 0);
    };
    int issued = 0;  // thread 0 only
    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], WARPS);
        }
        fence_mbar_init();
        failed = 0;
        tma_prefetch_desc(&tmA);
        tma_prefetch_desc(&tmB);
        for (; issued < STAGES && issued < ktiles; ++issued) {
            issue(issued);
        }
    }
    __syncthreads();

    // Warp w: product w / 4, warp tile 64 x 32 at (64 (w & 1), 32 ((w & 3) >> 1)); lane
    // (mi, ni) = (lane & 7, lane >> 3): rows am + {0..3, 32..35}, columns bn + {0..3, 16..19}.
    const int plane = warp >> 2, wq = warp & 3;
    const int am = (wq & 1) * 64 + (lane & 7) * 4;
    const int bn = (wq >> 1) * 32 + (lane >> 3) * 4;
    // acc[i][jj] = (P(row i, col 2jj), P(row i, col 2jj + 1)): one packed FMA
    // (__ffma2_rn: two independent round-to-nearest FMAs) updates both.
    float2 acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            acc[i][jj] = make_float2(0.0f, 0.0f);
        }
    }
    bool ok = true;
    int consumed = 0;
    for (int kt = 0; kt < ktiles; ++kt) {
        const int s = kt % STAGES;
        if (!mbar_wait(&full[s], (kt / STAGES) & 1, p.status)) {
            ok = false;
            break;
        }
        consumed = kt + 1;
        const float* a = sA + s * A_STAGE + plane * BK * BM + am;
        const float* b = sB + s * B_STAGE + plane * BK * BN + bn;
#pragma unroll KK_UNROLL
        for (int kk = 0; kk < BK; ++kk) {
            float x[8];
            float2 y[4];
            *reinterpret_cast<float4*>(&x[0]) = *reinterpret_cast<const float4*>(a + kk * BM);
            *reinterpret_cast<float4*>(&x[4]) = *reinterpret_cast<const float4*>(a + kk * BM + 32);
            *reinterpret_cast<float4*>(&y[0]) = *reinterpret_cast<const float4*>(b + kk * BN);
            *reinterpret_cast<float4*>(&y[2]) = *reinterpret_cast<const float4*>(b + kk * BN + 16);
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const float2 xi = make_float2(x[i], x[i]);
#pragma unroll
                for (int jj = 0; jj < 4; ++jj) acc[i][jj] = __ffma2_rn(xi, y[jj], acc[i][jj]);
            }
        }
        __syncwarp();
        if (lane == 0) {
            mbar_arrive(&empty[s]);
        }
        // Refill stage s with K-tile kt + STAGES once all twelve warps have released it.
        if (tid == 0 && issued < ktiles) {
            if (!mbar_wait(&empty[s], (kt / STAGES) & 1, p.status)) {
                ok = false;
                break;
            }
            issue(issued);
            ++issued;
        }
    }
    if (tid == 0) {
        // Copies this thread issued but no longer waits for (after a timeout) must land
        // before the ring is reused or the CTA retires.
        for (int kt = consumed; kt < issued; ++kt) {
            mbar_wait(&full[kt % STAGES], (kt / STAGES) & 1, p.status);
        }
    }
    if (!ok) {
        failed = 1;
    }
    // Every warp is past its last stage read and every copy has landed: the
    // ring becomes the exchange P[plane][col][row].
    __syncthreads();
    float* P = sA;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int col = bn + (j < 4 ? j : 12 + j);
        auto v = [&](int i) { return (j & 1) ? acc[i][j >> 1].y : acc[i][j >> 1].x; };
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            *reinterpret_cast<float4*>(P + (size_t)(plane * BN + col) * BM + am + 32 * h) =
                make_float4(v(4 * h), v(4 * h + 1), v(4 * h + 2), v(4 * h + 3));
        }
    }
    __syncthreads();
    if (!p.cluster_merge) {
        if (failed) {
            return;
        }
        for (int e = tid; e < BM * BN; e += THREADS) {
            const int r = e % BM, c = e / BM;
            const int row = m0 + r, col = n0 + c;
            if (row >= p.m || col >= p.n) {
                continue;
            }
            const float q0 = P[(0 * BN + c) * BM + r], q1 = P[(1 * BN + c) * BM + r];
            const float q2 = P[(2 * BN + c) * BM + r];
            const float re = __fsub_rn(q0, q1);
            const float im = __fsub_rn(__fsub_rn(q2, q0), q1);
            if (p.parts == 1) {
                float2* cp = p.C + (size_t)col * p.ldc + row;
                *cp = epilogue_at(re, im, p.epi, cp, row, col);
            } else {
                const size_t o = (size_t)col * p.ppitch + row;
                p.partial[(size_t)(2 * part) * p.pplane + o] = re;
                p.partial[(size_t)(2 * part + 1) * p.pplane + o] = im;
            }
        }
        return;
    }
    // K split merged through the cluster (grid.y = cluster.y = parts): this
    // partition's (Re, Im) replace planes 0 and 1 in place (element e read and
    // written by one thread), a cluster barrier publishes them, and block q
    // sums the q-th slice of the tile over partitions 0, 1, ... in order -- the
    // merge kernel's arithmetic -- reading its peers' shared memory, then
    // applies alpha/beta.  Every thread of every block reaches both barriers.
    for (int e = tid; e < BM * BN; e += THREADS) {
        const float q0 = P[e], q1 = P[BN * BM + e], q2 = P[2 * BN * BM + e];
        P[e] = __fsub_rn(q0, q1);
        P[BN * BM + e] = __fsub_rn(__fsub_rn(q2, q0), q1);
    }
    cluster_sync();
    const uint32_t re_local = smem_u32(P), im_local = smem_u32(P + BN * BM);
    int bad = 0;
    for (int q = 0; q < p.parts; ++q) {
        bad |= ld_dsmem_s32(mapa_shared(smem_u32(&failed), q));
    }
    if (!bad) {
        const int per = (BM * BN + p.parts - 1) / p.parts;
        const int e_end = min(BM * BN, (part + 1) * per);
        for (int e = part * per + tid; e < e_end; e += THREADS) {
            const int r = e % BM, c = e / BM;
            const int row = m0 + r, col = n0 + c;
            if (row >= p.m || col >= p.n) {
                continue;
            }
            float re = ld_dsmem_f32(mapa_shared(re_local + 4u * e, 0));
            float im = ld_dsmem_f32(mapa_shared(im_local + 4u * e, 0));
            for (int q = 1; q < p.parts; ++q) {
                re = __fadd_rn(re, ld_dsmem_f32(mapa_shared(re_local + 4u * e, q)));
                im = __fadd_rn(im, ld_dsmem_f32(mapa_shared(im_local + 4u * e, q)));
            }
            float2* cp = p.C + (size_t)col * p.ldc + row;
            *cp = epilogue_at(re, im, p.epi, cp, row, col);
        }
    }
    cluster_sync();  // no block leaves while others may still read its shared memory
}

// ---------------------------------------------------------------------------
// Path-tracking variant for the rounding-correction gate (square n in
// [2048, 4096], contiguous, alpha = 1, beta = 0).  Reference: cgemm3m_path_kernel
// and MergeProductsWithPath, blas/gemm/arch35/cgemm_compute_kernel.cpp:432-474,
// 897-927: K is cut into 128-term parts accumulated from zero, merged in order
// into the running sum s, and each part of depth d adds
// d/9 * (s_old^2 + s_old*s_new + s_new^2) to the real and imaginary integrals;
// path = max(I_re, I_im).  Each thread keeps a 4 x 4 complex micro-tile (three
// product accumulators, the running sums and both integrals), CTA tile 64 x 64.
// Only the real and imaginary planes are staged: the third operand of the
// identity (Re + Im) is formed in registers with the same round-to-nearest
// add the pack kernel uses for that plane, so the products keep their bits
// while shared-memory reads (this kernel's limit) drop by a third.
// ---------------------------------------------------------------------------
constexpr int kRiskSegment = 128;

struct PathParams {
    int n;
    int tiles;
    float2* C;    // ldc = n
    float* path;  // ld = n
    int* status;
};

__global__ void __launch_bounds__(288, 1)
    gemm3m_fp32_path_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                            const PathParams p)
{
    constexpr int BM = 64, BN = 64, BK = 16, STAGES = 4, CONSUMER_WARPS = 8;
    constexpr int A_STAGE = 2 * BK * BM, B_STAGE = 2 * BK * BN;  // planes 0 (Re) and 1 (Im)
    extern __shared__ uint8_t smem_raw[];
    uint8_t* base = align_shared<1024>(smem_raw);
    float* sA = reinterpret_cast<float*>(base);
    float* sB = sA + STAGES * A_STAGE;
    uint64_t* full = reinterpret_cast<uint64_t*>(sB + STAGES * B_STAGE);
    uint64_t* empty = full + STAGES;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // Tiles run in bands of BAND tile rows, rows fastest within a band, so the
    // band's op(A) planes stay in L2 while its columns go by.
    constexpr int BAND = 8;
    const int band = blockIdx.x / (BAND * p.tiles), first = band * BAND;
    const int rows_in_band = min(BAND, p.tiles - first), in_band = blockIdx.x - band * BAND * p.tiles;
    const int tm = first + in_band % rows_in_band, tn = in_band / rows_in_band;
    const int m0 = tm * BM, n0 = tn * BN;
    const int ktiles = (p.n + BK - 1) / BK;
    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], CONSUMER_WARPS);
        }
        fence_mbar_init();
    }
    __syncthreads();
    if (warp == CONSUMER_WARPS) {
        if (lane == 0) {
            int issued = 0;
            for (int kt = 0; kt < ktiles; ++kt) {
                const int s = kt % STAGES;
                if (kt >= STAGES && !mbar_wait(&empty[s], ((kt / STAGES) - 1) & 1, p.status)) {
                    break;
                }
                mbar_arrive_expect_tx(&full[s], (A_STAGE + B_STAGE) * 4);
                tma_load_3d(sA + s * A_STAGE, &tmA, &full[s], m0, kt * BK, 0);
                tma_load_3d(sB + s * B_STAGE, &tmB, &full[s], n0, kt * BK, 0);
                ++issued;
            }
            for (int kt = issued > STAGES ? issued - STAGES : 0; kt < issued; ++kt) {
                mbar_wait(&full[kt % STAGES], (kt / STAGES) & 1, p.status);
            }
        }
    } else {
        // warp -> 32 x 16 sub-tile (lanes 8 x 4), thread -> 4 x 4 outputs
        const int wm = warp & 1, wn = warp >> 1;
        const int tm0 = wm * 32 + (lane & 7) * 4;
        const int tn0 = wn * 16 + (lane >> 3) * 4;
        // Product accumulators in column pairs: p0[i][jj] = (P0(row i, col 2jj),
        // P0(row i, col 2jj + 1)), updated by one packed FMA (__ffma2_rn: two
        // independent round-to-nearest FMAs).
        float2 p0[4][2], p1[4][2], p2[4][2];
        float sr[4][4], si[4][4], ir[4][4], ii[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
#pragma unroll
            for (int jj = 0; jj < 2; ++jj) {
                p0[i][jj] = p1[i][jj] = p2[i][jj] = make_float2(0.0f, 0.0f);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                sr[i][j] = si[i][j] = ir[i][j] = ii[i][j] = 0.0f;
            }
        }
        bool ok = true;
        int seg_terms = 0;
        for (int kt = 0; kt < ktiles; ++kt) {
            const int s = kt % STAGES;
            if (!mbar_wait(&full[s], (kt / STAGES) & 1, p.status)) {
                ok = false;
                break;
            }
            const float* a = sA + s * A_STAGE + tm0;
            const float* b = sB + s * B_STAGE + tn0;
            const int kvalid = min(BK, p.n - kt * BK);
#pragma unroll
            for (int kk = 0; kk < BK; ++kk) {
                float x0[4], x1[4], x2[4];
                float2 y0[2], y1[2], y2[2];
                *reinterpret_cast<float4*>(x0) = *reinterpret_cast<const float4*>(a + kk * BM);
                *reinterpret_cast<float4*>(x1) = *reinterpret_cast<const float4*>(a + (BK + kk) * BM);
                *reinterpret_cast<float4*>(y0) = *reinterpret_cast<const float4*>(b + kk * BN);
                *reinterpret_cast<float4*>(y1) = *reinterpret_cast<const float4*>(b + (BK + kk) * BN);
                // Re + Im of each operand (the pack kernel's third plane, same rounding);
                // packed adds of loaded values, so nothing can be contracted.
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const float2 s = __fadd2_rn(make_float2(x0[2 * h], x0[2 * h + 1]),
                                                make_float2(x1[2 * h], x1[2 * h + 1]));
                    x2[2 * h] = s.x;
                    x2[2 * h + 1] = s.y;
                    y2[h] = __fadd2_rn(y0[h], y1[h]);
                }
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const float2 a0 = make_float2(x0[i], x0[i]), a1 = make_float2(x1[i], x1[i]),
                                 a2 = make_float2(x2[i], x2[i]);
#pragma unroll
                    for (int jj = 0; jj < 2; ++jj) {
                        p0[i][jj] = __ffma2_rn(a0, y0[jj], p0[i][jj]);
                        p1[i][jj] = __ffma2_rn(a1, y1[jj], p1[i][jj]);
                        p2[i][jj] = __ffma2_rn(a2, y2[jj], p2[i][jj]);
                    }
                }
            }
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&empty[s]);
            }
            seg_terms += kvalid;
            // A segment closes every 128 terms (8 K-tiles) and at the end of K.
            if (seg_terms == kRiskSegment || kt == ktiles - 1) {
                const float w = __fdiv_rn((float)seg_terms, 9.0f);
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const float q0 = (j & 1) ? p0[i][j >> 1].y : p0[i][j >> 1].x;
                        const float q1 = (j & 1) ? p1[i][j >> 1].y : p1[i][j >> 1].x;
                        const float q2 = (j & 1) ? p2[i][j >> 1].y : p2[i][j >> 1].x;
                        const float nr = __fadd_rn(sr[i][j], __fsub_rn(q0, q1));
                        const float ni = __fadd_rn(si[i][j], __fsub_rn(__fsub_rn(q2, q0), q1));
                        float t = __fmul_rn(sr[i][j], sr[i][j]);
                        t = __fmaf_rn(sr[i][j], nr, t);
                        t = __fmaf_rn(nr, nr, t);
                        ir[i][j] = __fadd_rn(ir[i][j], __fmul_rn(t, w));
                        t = __fmul_rn(si[i][j], si[i][j]);
                        t = __fmaf_rn(si[i][j], ni, t);
                        t = __fmaf_rn(ni, ni, t);
                        ii[i][j] = __fadd_rn(ii[i][j], __fmul_rn(t, w));
                        sr[i][j] = nr;
                        si[i][j] = ni;
                    }
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int jj = 0; jj < 2; ++jj) {
                        p0[i][jj] = p1[i][jj] = p2[i][jj] = make_float2(0.0f, 0.0f);
                    }
                seg_terms = 0;
            }
        }
        if (ok) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int col = n0 + tn0 + j;
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int row = m0 + tm0 + i;
                    if (row < p.n && col < p.n) {
                        const size_t o = (size_t)col * p.n + row;
                        p.C[o] = make_float2(sr[i][j], si[i][j]);
                        p.path[o] = ir[i][j] > ii[i][j] ? ir[i][j] : ii[i][j];
                    }
                }
            }
        }
    }
    __syncthreads();
}

// Sum of the partition partials in increasing partition order, then alpha/beta.
__global__ void merge_kernel(int m, int n, int parts, const float* __restrict__ partial, int ppitch, size_t pplane,
                             EpiParams e, float2* C, int ldc)
{
    const size_t total = (size_t)m * n;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        const int col = (int)(idx / m), row = (int)(idx - (size_t)col * m);
        const size_t o = (size_t)col * ppitch + row;
        float re = partial[o], im = partial[pplane + o];
        for (int q = 1; q < parts; ++q) {
            re = __fadd_rn(re, partial[(size_t)(2 * q) * pplane + o]);
            im = __fadd_rn(im, partial[(size_t)(2 * q + 1) * pplane + o]);
        }
        float2* cp = C + (size_t)col * ldc + row;
        *cp = epilogue_at(re, im, e, cp, row, col);
    }
}

// k == 0 or alpha == 0: C = beta*C (beta == 0: C = 0 without reading C).
__global__ void beta_scale_kernel(int m, int n, float br, float bi, float2* C, int ldc)
{
    const size_t total = (size_t)m * n;
    const bool zero = br == 0.0f && bi == 0.0f;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        const int col = (int)(idx / m), row = (int)(idx - (size_t)col * m);
        float2* cp = C + (size_t)col * ldc + row;
        if (zero) {
            *cp = make_float2(0.0f, 0.0f);
        } else {
            const float2 c = *cp;
            *cp = make_float2(__fsub_rn(__fmul_rn(br, c.x), __fmul_rn(bi, c.y)),
                              __fadd_rn(__fmul_rn(br, c.y), __fmul_rn(bi, c.x)));
        }
    }
}

int elementwise_blocks(size_t total)
{
    const size_t blocks = (total + 255) / 256;
    return (int)(blocks < 148 * 16 ? (blocks == 0 ? 1 : blocks) : 148 * 16);
}

// Epilogue parameters of an FP32 call; a cg3mCgemm call with alpha = 1,
// beta = 0 (plan.repair) also carries what the non-finite repair reads.
EpiParams fp32_epilogue(const Problem& pr, const Plan& plan)
{
    EpiParams e{pr.ar, pr.ai, pr.br, pr.bi, plan.unit ? 1 : 0, plan.beta_zero ? 1 : 0};
    if (plan.repair) {
        e.repair = 1;
        e.ta = pr.transa;
        e.tb = pr.transb;
        e.k = pr.k;
        e.lda = pr.lda;
        e.ldb = pr.ldb;
        e.A = static_cast<const float2*>(pr.A);
        e.B = static_cast<const float2*>(pr.B);
    }
    return e;
}

template <int BM, int BN>
cudaError_t launch_fp32_tile(cudaStream_t stream, const Problem& pr, const Plan& plan, void* ws, int* status)
{
    using Cfg = Fp32Cfg<BM, BN>;
    uint8_t* w = static_cast<uint8_t*>(ws);
    CUtensorMap ta, tb;
    {
        const uint64_t dims[3] = {(uint64_t)pr.m, (uint64_t)pr.k, 3};
        const uint64_t strides[2] = {(uint64_t)plan.pitch_a * 4, (uint64_t)plan.plane_a_elems * 4};
        const uint32_t box[3] = {BM, Cfg::BK, 3};
        if (!encode_tensor_map(&ta, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, dims, strides, box,
                               CU_TENSOR_MAP_SWIZZLE_NONE, w + plan.planes_a_off)) {
            return cudaErrorInvalidValue;
        }
    }
    {
        const uint64_t dims[3] = {(uint64_t)pr.n, (uint64_t)pr.k, 3};
        const uint64_t strides[2] = {(uint64_t)plan.pitch_b * 4, (uint64_t)plan.plane_b_elems * 4};
        const uint32_t box[3] = {BN, Cfg::BK, 3};
        if (!encode_tensor_map(&tb, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, dims, strides, box,
                               CU_TENSOR_MAP_SWIZZLE_NONE, w + plan.planes_b_off)) {
            return cudaErrorInvalidValue;
        }
    }
    Fp32Params p{};
    p.m = pr.m;
    p.n = pr.n;
    p.k = pr.k;
    p.span = plan.span;
    p.parts = plan.parts;
    p.tiles_m = ceil_div(pr.m, BM);
    p.tiles_n = ceil_div(pr.n, BN);
    p.epi = fp32_epilogue(pr, plan);
    p.C = static_cast<float2*>(pr.C);
    p.ldc = pr.ldc;
    p.partial = reinterpret_cast<float*>(w + plan.partial_off);
    p.ppitch = plan.partial_pitch;
    p.pplane = plan.partial_plane_elems;
    p.status = status;
    const dim3 grid((unsigned)(p.tiles_m * p.tiles_n), (unsigned)plan.parts);
    if constexpr (BM == ws::BM && BN == ws::BN) {
        cudaError_t err = cudaFuncSetAttribute(gemm3m_fp32_ws_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)ws::SMEM);
        if (err != cudaSuccess) {
            return err;
        }
        p.cluster_merge = plan.cluster_merge ? 1 : 0;
        if (!p.cluster_merge) {
            gemm3m_fp32_ws_kernel<<<grid, ws::THREADS, ws::SMEM, stream>>>(ta, tb, p);
            return cudaGetLastError();
        }
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = grid;
        cfg.blockDim = dim3(ws::THREADS, 1, 1);
        cfg.dynamicSmemBytes = ws::SMEM;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 1;
        attr[0].val.clusterDim.y = (unsigned)plan.parts;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        err = cudaLaunchKernelEx(&cfg, gemm3m_fp32_ws_kernel, ta, tb, p);
        return err != cudaSuccess ? err : cudaGetLastError();
    } else {
        auto kernel = gemm3m_fp32_kernel<BM, BN>;
        cudaError_t err =
            cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::SMEM);
        if (err != cudaSuccess) {
            return err;
        }
        kernel<<<grid, Cfg::THREADS, Cfg::SMEM, stream>>>(ta, tb, p);
        return cudaGetLastError();
    }
}

}  // namespace

cudaError_t launch_gemm_fp32(cudaStream_t stream, const Problem& pr, const Plan& plan, void* ws, int* status)
{
    if (plan.tile_m == 128 && plan.tile_n == 64) {
        return launch_fp32_tile<128, 64>(stream, pr, plan, ws, status);
    }
    if (plan.tile_m == 64 && plan.tile_n == 64) {
        return launch_fp32_tile<64, 64>(stream, pr, plan, ws, status);
    }
    if (plan.tile_m == 64 && plan.tile_n == 32) {
        return launch_fp32_tile<64, 32>(stream, pr, plan, ws, status);
    }
    return launch_fp32_tile<32, 32>(stream, pr, plan, ws, status);
}

cudaError_t launch_gemm_fp32_path(cudaStream_t stream, const Problem& pr, const Plan& plan, void* ws, float* path,
                                  int* status)
{
    constexpr int BM = 64, BN = 64, BK = 16, STAGES = 4;
    uint8_t* w = static_cast<uint8_t*>(ws);
    CUtensorMap ta, tb;
    {
        const uint64_t dims[3] = {(uint64_t)pr.m, (uint64_t)pr.k, 3};
        const uint64_t strides[2] = {(uint64_t)plan.pitch_a * 4, (uint64_t)plan.plane_a_elems * 4};
        const uint32_t box[3] = {BM, BK, 2};  // planes 0 and 1; the kernel forms plane 2
        if (!encode_tensor_map(&ta, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, dims, strides, box,
                               CU_TENSOR_MAP_SWIZZLE_NONE, w + plan.planes_a_off)) {
            return cudaErrorInvalidValue;
        }
    }
    {
        const uint64_t dims[3] = {(uint64_t)pr.n, (uint64_t)pr.k, 3};
        const uint64_t strides[2] = {(uint64_t)plan.pitch_b * 4, (uint64_t)plan.plane_b_elems * 4};
        const uint32_t box[3] = {BN, BK, 2};
        if (!encode_tensor_map(&tb, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, dims, strides, box,
                               CU_TENSOR_MAP_SWIZZLE_NONE, w + plan.planes_b_off)) {
            return cudaErrorInvalidValue;
        }
    }
    PathParams p{pr.n, ceil_div(pr.n, BM), static_cast<float2*>(pr.C), path, status};
    const size_t smem = (size_t)STAGES * 2 * BK * (BM + BN) * 4 + 2 * STAGES * 8 + 1024;
    cudaError_t err =
        cudaFuncSetAttribute(gemm3m_fp32_path_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) {
        return err;
    }
    gemm3m_fp32_path_kernel<<<p.tiles * p.tiles, 288, smem, stream>>>(ta, tb, p);
    return cudaGetLastError();
}

cudaError_t launch_merge(cudaStream_t stream, const Problem& pr, const Plan& plan, void* ws)
{
    const float* partial = reinterpret_cast<const float*>(static_cast<uint8_t*>(ws) + plan.partial_off);
    const EpiParams e = fp32_epilogue(pr, plan);
    merge_kernel<<<elementwise_blocks((size_t)pr.m * pr.n), 256, 0, stream>>>(
        pr.m, pr.n, plan.parts, partial, plan.partial_pitch, plan.partial_plane_elems, e, static_cast<float2*>(pr.C),
        pr.ldc);
    return cudaGetLastError();
}

cudaError_t launch_beta_scale(cudaStream_t stream, int m, int n, float br, float bi, void* C, int ldc)
{
    beta_scale_kernel<<<elementwise_blocks((size_t)m * n), 256, 0, stream>>>(m, n, br, bi, static_cast<float2*>(C),
                                                                             ldc);
    return cudaGetLastError();
}

}  // namespace cg3m
