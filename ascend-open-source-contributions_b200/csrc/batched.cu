// batched.cu -- many cgemm3m problems of uneven shape and mixed op() in one
// persistent launch (the batching form).
//
// Reference hooks for batched 3M: LaunchCgemm3mOnchipBatches /
// LaunchCgemm3mUnitBatches (blas/gemm/arch35/cgemm_host.cpp:749-782,
// gemm_host_common.h:84-97), used by aclblasCgemm3mStridedBatched
// (cann_ops_blas.h:652).  The reference batches equal shapes only; this form
// takes a heterogeneous list, and like the reference's on-chip batch kernel
// (cgemm_onchip_kernel.h:84 ProducePanel) it deinterleaves inside the GEMM
// instead of through a workspace.
//
// Design.  One persistent kernel (grid = SM count x resident blocks) pulls
// tasks from a device list through an atomic counter; a task is (problem,
// output tile, K partition), and the list is sorted by decreasing work so the
// schedule ends on small tasks.  A task stages op(A) and op(B) straight from
// the caller's interleaved complex matrices into shared-memory planes re, im,
// fl(re+im) (op() and conjugation applied while staging, the next K-block
// prefetched into registers during the current one's FFMAs), runs the 3M FFMA
// micro-kernel of the drop-in (one thread per output, K in increasing order,
// fmaf into P0, P1, P2 from +0), and either applies alpha/beta and stores, or
// writes its partition's (Re, Im) partials and counts in on a per-tile counter;
// the last partition to arrive merges all partitions in partition order with
// the merge arithmetic of the drop-in and stores.  No block ever waits on
// another.  Each output is thus a fixed function of the inputs and its K
// split, bit-identical to the drop-in called with the same k_partitions.
//
// Tile (128x64, 64x64, 64x32, 32x32) and K split are chosen per problem from a
// policy table; the autotuner times every candidate policy on the device with
// the caller's A and B and a scratch C, keeps the fastest and caches it per
// batch signature (device, ops, shapes).  Execute may replay a captured CUDA
// graph holding the counter reset and the one kernel.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "cg3m_internal.h"
#include "epilogue.cuh"
#include "ptx.cuh"

namespace cg3m {
namespace {

constexpr int kThreads = 256;
constexpr int BK = 16;
#ifndef CG3M_BATCH_UNROLL
#define CG3M_BATCH_UNROLL 4
#endif
constexpr int kUnroll = CG3M_BATCH_UNROLL;  // K terms unrolled in the FFMA loop

// Product modes: the standard 3M identity (P0 = Ar.Br, P1 = Ai.Bi,
// P2 = (Ar+Ai).(Br+Bi); Re = P0 - P1, Im = (P2 - P0) - P1) or four real
// products (Re = Ar.Br - Ai.Bi, Im = Ar.Bi + Ai.Br).
constexpr int kMode3M = 0;
constexpr int kMode4M = 1;

struct BProblem {
    int ta, tb, m, n, k;  // k = 0: beta-scale only (k == 0 or alpha == 0)
    EpiParams epi;
    const float2* A;
    const float2* B;
    float2* C;
    int lda, ldb, ldc;
    int tile;    // index into the tile shapes below
    int repair;  // recompute non-finite products with explicit FP32 four-product terms
    int parts, span, tiles_m, tiles_n, ppitch;
    size_t partial_off;  // floats into the partial arena
    size_t counter_off;  // words into the tile counters
};

struct BTask {
    int problem, tile, part, pad;
};

// Tile shapes (BM x BN): 0: 128x64, 1: 64x64, 2: 128x32, 3: 32x128, 4: 64x32, 5: 32x32.
// The four-product mode does not use tile 0 (its accumulators would not fit).
constexpr int kTileCount = 6;
__host__ __device__ constexpr int tile_bm(int t)
{
    return (t == 0 || t == 2) ? 128 : (t == 1 || t == 4) ? 64 : 32;
}
__host__ __device__ constexpr int tile_bn(int t)
{
    return t == 3 ? 128 : (t == 0 || t == 1) ? 64 : 32;
}

template <int BM, int BN, int MODE>
struct Cfg {
    static constexpr int MT = BM / 16, NT = BN / 16;  // outputs per thread along m, n
    static constexpr int VA = MT >= 4 ? 4 : MT, HA = MT / VA;
    static constexpr int VB = NT >= 4 ? 4 : NT, HB = NT / VB;
    static constexpr int SA = BM + 4, SB = BN + 4;  // padded plane strides (floats)
    static constexpr int EA = BM * BK / kThreads, EB = BN * BK / kThreads;  // elements per thread per K-block
    static constexpr int COMPS = MODE == kMode3M ? 3 : 2;                      // planes per operand
    static constexpr int A_FLOATS = COMPS * BK * SA, B_FLOATS = COMPS * BK * SB;
    static constexpr int ACC = MODE == kMode3M ? 3 : 4;                        // accumulators per output
};

// Shared memory: kStages raw stages of interleaved complex elements (as
// copied, one slot per (thread, element)), then two plane buffers.
constexpr int kStages = 4;
constexpr int kRawElems = (128 + 64) * BK;  // largest BM + BN of any tile, times BK
constexpr int kPlaneFloats = 3 * BK * (128 + 4) + 3 * BK * (64 + 4);
constexpr size_t kSmemBytes = (size_t)kStages * kRawElems * sizeof(float2) + 2 * (size_t)kPlaneFloats * sizeof(float);

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// 8-byte asynchronous copy global -> shared; src_bytes = 0 writes zeros
// (the source is then not read).
__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src, int src_bytes)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// One operand's share of a K-block for this thread (q = 0 .. E-1).  The
// source's contiguous dimension goes to consecutive threads: rows
// ("rows_contig": op(A) in {N, R}, op(B) in {T, C}; r = e % R, kk = e / R with
// e = tid + q*kThreads) or K (8 consecutive K of 4 rows per warp; row
// 16q + r0(tid), K index kk0(tid)).
//   rows_contig: X[(row0 + r) + k*ld]      else: X[k + (row0 + r)*ld]
struct Feed {
    const float2* origin;  // the matrix (source of the zero-byte copies)
    const float2* base;    // element q = 0 at K-block 0
    long long qstep;       // element offset between consecutive q
    long long kbstep;      // element offset between consecutive K-blocks
    int r, kk;             // block coordinates of element q = 0
    int rq, kq;            // coordinate steps between consecutive q
    int rows;              // valid rows of this tile
    float conj;            // -1 for op C / R
};

template <int R>
__device__ __forceinline__ Feed make_feed(const float2* X, int ld, bool rows_contig, int row0, int rows, int kbeg,
                                          float conj)
{
    Feed f;
    const int tid = threadIdx.x;
    if (rows_contig) {
        f.r = tid % R;
        f.kk = tid / R;
        f.rq = 0;
        f.kq = kThreads / R;
        f.base = X + (long long)(row0 + f.r) + (long long)(kbeg + f.kk) * ld;
        f.qstep = (long long)f.kq * ld;
        f.kbstep = (long long)BK * ld;
    } else {
        // Each warp covers 4 rows x 8 consecutive K: 64-byte global segments,
        // and conflict-free plane stores (row stride = 4 banks mod 32).
        f.kk = (tid % 8) + 8 * ((tid / 32) % 2);
        f.r = ((tid / 8) % 4) + 4 * (tid / 64);
        f.rq = kThreads / BK;
        f.kq = 0;
        f.base = X + (long long)(kbeg + f.kk) + (long long)(row0 + f.r) * ld;
        f.qstep = (long long)f.rq * ld;
        f.kbstep = BK;
    }
    f.origin = X;
    f.rows = rows;
    f.conj = conj;
    return f;
}

// Issue this thread's copies of K-block kb into raw slot `raw`; elements past
// the tile or past the partition's K range read as zero.
template <int E>
__device__ __forceinline__ void issue(const Feed& f, float2* raw, int kb, int krel_end)
{
    const float2* src = f.base + (long long)kb * f.kbstep;
#pragma unroll
    for (int q = 0; q < E; ++q) {
        const int r = f.r + q * f.rq;
        const int kk = kb * BK + f.kk + q * f.kq;
        const bool ok = r < f.rows && kk < krel_end;
        cp_async8(smem_u32(raw + threadIdx.x + q * kThreads),
                  ok ? (const void*)(src + q * f.qstep) : (const void*)f.origin, ok ? 8 : 0);
    }
}

// Convert this thread's own elements of a raw slot into the planes
// re, im (conjugated) [, fl(re + im) for 3M] at dst[(c*BK + kk)*S + r].
template <int S, int E, int COMPS>
__device__ __forceinline__ void convert(const Feed& f, const float2* raw, float* dst)
{
#pragma unroll
    for (int q = 0; q < E; ++q) {
        const float2 v = raw[threadIdx.x + q * kThreads];
        const float re = v.x, im = v.y * f.conj;
        const int r = f.r + q * f.rq;
        const int kk = f.kk + q * f.kq;
        dst[(0 * BK + kk) * S + r] = re;
        dst[(1 * BK + kk) * S + r] = im;
        if constexpr (COMPS == 3) {
            dst[(2 * BK + kk) * S + r] = __fadd_rn(re, im);
        }
    }
}

template <int V>
__device__ __forceinline__ void ld_vec(const float* p, float* out)
{
    if constexpr (V == 4) {
        const float4 t = *reinterpret_cast<const float4*>(p);
        out[0] = t.x;
        out[1] = t.y;
        out[2] = t.z;
        out[3] = t.w;
    } else if constexpr (V == 2) {
        const float2 t = *reinterpret_cast<const float2*>(p);
        out[0] = t.x;
        out[1] = t.y;
    } else {
        out[0] = *p;
    }
}

// C = beta*C for k == 0 or alpha == 0 (beta == 0: zeros, C not read).
__device__ __forceinline__ float2 beta_scaled(const EpiParams& e, const float2* cp)
{
    if (e.beta_zero) {
        return make_float2(0.0f, 0.0f);
    }
    const float2 c = *cp;
    return make_float2(__fsub_rn(__fmul_rn(e.br, c.x), __fmul_rn(e.bi, c.y)),
                       __fadd_rn(__fmul_rn(e.br, c.y), __fmul_rn(e.bi, c.x)));
}

// Non-finite repair of one output (repair_four_product, epilogue.cuh).
__device__ float2 repair_product(const BProblem& p, int row, int col)
{
    return repair_four_product(p.A, p.lda, p.ta, p.B, p.ldb, p.tb, p.k, row, col);
}

// Partition product (before alpha/beta) of the accumulators of one output.
template <int MODE>
__device__ __forceinline__ float2 part_product(float q0, float q1, float q2, float q3)
{
    if constexpr (MODE == kMode3M) {
        return make_float2(__fsub_rn(q0, q1), __fsub_rn(__fsub_rn(q2, q0), q1));
    } else {
        return make_float2(__fsub_rn(q0, q1), __fadd_rn(q2, q3));
    }
}

__device__ __forceinline__ bool finite2(float2 v) { return isfinite(v.x) && isfinite(v.y); }

// 16 x 16 threads over the tile; each warp is 8 (along m) x 4 (along n)
// threads, so one vector load of A or B per warp spans at most 128 bytes
// (one shared-memory wavefront).
__device__ __forceinline__ int thread_tx() { return ((threadIdx.x >> 5) & 1) * 8 + (threadIdx.x & 7); }
__device__ __forceinline__ int thread_ty() { return (threadIdx.x >> 6) * 4 + ((threadIdx.x & 31) >> 3); }

// Accumulators: acc[c][i][jj] holds outputs (i, 2jj) and (i, 2jj + 1) of
// accumulator c, updated together by one packed FMA (__ffma2_rn: two
// independent round-to-nearest FP32 FMAs), so each output is still the same
// FMA chain in increasing K.
template <int BM, int BN, int MODE>
using AccTile = float2[Cfg<BM, BN, MODE>::ACC][Cfg<BM, BN, MODE>::MT][Cfg<BM, BN, MODE>::NT / 2];

template <int BM, int BN, int MODE>
__device__ __forceinline__ float acc_at(const AccTile<BM, BN, MODE>& acc, int c, int i, int j)
{
    return (j & 1) ? acc[c][i][j >> 1].y : acc[c][i][j >> 1].x;
}

// Partition product of output (i, j) of this thread.
template <int BM, int BN, int MODE>
__device__ __forceinline__ float2 acc_product(const AccTile<BM, BN, MODE>& acc, int i, int j)
{
    constexpr int L = Cfg<BM, BN, MODE>::ACC - 1;
    return part_product<MODE>(acc_at<BM, BN, MODE>(acc, 0, i, j), acc_at<BM, BN, MODE>(acc, 1, i, j),
                              acc_at<BM, BN, MODE>(acc, 2, i, j), acc_at<BM, BN, MODE>(acc, L, i, j));
}

// The products of K terms [kbeg, kbeg + klen) of the BM x BN tile at (m0, n0),
// accumulated from zero into acc: kStages raw slots of RAWS elements and two
// plane buffers of PLS floats.
template <int BM, int BN, int MODE, int RAWS, int PLS>
__device__ __forceinline__ void accumulate(const BProblem& p, int m0, int n0, int kbeg, int klen, float2* raw,
                                           float* planes, AccTile<BM, BN, MODE>& acc)
{
    using G = Cfg<BM, BN, MODE>;
    static_assert(G::A_FLOATS + G::B_FLOATS <= PLS, "planes exceed their buffer");
    static_assert((BM + BN) * BK <= RAWS, "raw stage exceeds its slot");
    static_assert((BM * BK) % kThreads == 0 && (BN * BK) % kThreads == 0, "whole elements per thread");
    const int nk = (klen + BK - 1) / BK;
    const int tx = thread_tx(), ty = thread_ty();
    const bool na = p.ta == CG3M_OP_N || p.ta == CG3M_OP_R;
    const bool nb = p.tb == CG3M_OP_N || p.tb == CG3M_OP_R;
    const Feed fa = make_feed<BM>(p.A, p.lda, na, m0, min(BM, p.m - m0), kbeg,
                                  (p.ta == CG3M_OP_C || p.ta == CG3M_OP_R) ? -1.0f : 1.0f);
    const Feed fb = make_feed<BN>(p.B, p.ldb, !nb, n0, min(BN, p.n - n0), kbeg,
                                  (p.tb == CG3M_OP_C || p.tb == CG3M_OP_R) ? -1.0f : 1.0f);
#pragma unroll
    for (int c = 0; c < G::ACC; ++c)
#pragma unroll
        for (int i = 0; i < G::MT; ++i)
#pragma unroll
            for (int j = 0; j < G::NT / 2; ++j) {
                acc[c][i][j] = make_float2(0.0f, 0.0f);
            }

    // Prologue: K-blocks 0 .. kStages-2 in flight (one commit group each,
    // empty groups past the end keep the counting uniform).
#pragma unroll
    for (int s = 0; s < kStages - 1; ++s) {
        if (s < nk) {
            float2* slot = raw + s * RAWS;
            issue<G::EA>(fa, slot, s, klen);
            issue<G::EB>(fb, slot + BM * BK, s, klen);
        }
        cp_async_commit();
    }
    for (int kb = 0; kb < nk; ++kb) {
        // Refill the slot converted in the previous iteration (by this same
        // thread: each thread copies and converts only its own elements).
        const int nxt = kb + kStages - 1;
        if (nxt < nk) {
            float2* slot = raw + (nxt % kStages) * RAWS;
            issue<G::EA>(fa, slot, nxt, klen);
            issue<G::EB>(fb, slot + BM * BK, nxt, klen);
        }
        cp_async_commit();
        cp_async_wait<kStages - 1>();  // this thread's copies of K-block kb have landed
        const float2* slot = raw + (kb % kStages) * RAWS;
        float* sA = planes + (kb & 1) * PLS;
        float* sB = sA + G::A_FLOATS;
        convert<G::SA, G::EA, G::COMPS>(fa, slot, sA);
        convert<G::SB, G::EB, G::COMPS>(fb, slot + BM * BK, sB);
        // Plane buffer kb&1 was last read in iteration kb-2; this barrier also
        // orders iteration kb-1's reads before the next iteration's writes.
        __syncthreads();
        const float* a = sA + tx * G::VA;
        const float* b = sB + ty * G::VB;
#pragma unroll kUnroll
        for (int kk = 0; kk < BK; ++kk) {
            float x[G::COMPS][G::MT], y[G::COMPS][G::NT];
#pragma unroll
            for (int c = 0; c < G::COMPS; ++c) {
#pragma unroll
                for (int h = 0; h < G::HA; ++h) {
                    ld_vec<G::VA>(a + (c * BK + kk) * G::SA + h * 16 * G::VA, x[c] + h * G::VA);
                }
#pragma unroll
                for (int h = 0; h < G::HB; ++h) {
                    ld_vec<G::VB>(b + (c * BK + kk) * G::SB + h * 16 * G::VB, y[c] + h * G::VB);
                }
            }
#pragma unroll
            for (int i = 0; i < G::MT; ++i) {
                float2 xb[G::COMPS];
#pragma unroll
                for (int c = 0; c < G::COMPS; ++c) {
                    xb[c] = make_float2(x[c][i], x[c][i]);
                }
#pragma unroll
                for (int jj = 0; jj < G::NT / 2; ++jj) {
                    float2 yp[G::COMPS];
#pragma unroll
                    for (int c = 0; c < G::COMPS; ++c) {
                        yp[c] = make_float2(y[c][2 * jj], y[c][2 * jj + 1]);
                    }
                    if constexpr (MODE == kMode3M) {
                        acc[0][i][jj] = __ffma2_rn(xb[0], yp[0], acc[0][i][jj]);
                        acc[1][i][jj] = __ffma2_rn(xb[1], yp[1], acc[1][i][jj]);
                        acc[2][i][jj] = __ffma2_rn(xb[2], yp[2], acc[2][i][jj]);
                    } else {
                        acc[0][i][jj] = __ffma2_rn(xb[0], yp[0], acc[0][i][jj]);  // Ar.Br
                        acc[1][i][jj] = __ffma2_rn(xb[1], yp[1], acc[1][i][jj]);  // Ai.Bi
                        acc[2][i][jj] = __ffma2_rn(xb[0], yp[1], acc[2][i][jj]);  // Ar.Bi
                        acc[3][i][jj] = __ffma2_rn(xb[1], yp[0], acc[3][i][jj]);  // Ai.Br
                    }
                }
            }
        }
    }
    cp_async_wait<0>();  // only empty groups can remain; keep the count at zero between tasks
}

template <int BM, int BN, int MODE>
__device__ void run_task(const BProblem& prob, int tile, int part, float2* raw, float* planes, float* partials,
                         uint32_t* counters, int* last_flag)
{
    using G = Cfg<BM, BN, MODE>;
    const BProblem p = prob;  // registers: no reloads after barriers
    const int tm = tile % p.tiles_m, tn = tile / p.tiles_m;
    const int m0 = tm * BM, n0 = tn * BN;
    const int kbeg = part * p.span;
    const int kend = min(p.k, kbeg + p.span);
    const int klen = kend > kbeg ? kend - kbeg : 0;
    const int tx = thread_tx(), ty = thread_ty();
    AccTile<BM, BN, MODE> acc;
    accumulate<BM, BN, MODE, kRawElems, kPlaneFloats>(p, m0, n0, kbeg, klen, raw, planes, acc);

    // Output (i, j) of this thread: row m0 + (i / VA)*16*VA + tx*VA + i % VA,
    // column n0 + (j / VB)*16*VB + ty*VB + j % VB.
    if (p.parts == 1) {
#pragma unroll
        for (int j = 0; j < G::NT; ++j) {
            const int col = n0 + (j / G::VB) * 16 * G::VB + ty * G::VB + j % G::VB;
#pragma unroll
            for (int i = 0; i < G::MT; ++i) {
                const int row = m0 + (i / G::VA) * 16 * G::VA + tx * G::VA + i % G::VA;
                if (row < p.m && col < p.n) {
                    float2* cp = p.C + (size_t)col * p.ldc + row;
                    if (p.k == 0) {
                        *cp = beta_scaled(p.epi, cp);
                    } else {
                        float2 v = acc_product<BM, BN, MODE>(acc, i, j);
                        if (p.repair && !finite2(v)) {
                            v = repair_product(p, row, col);
                        }
                        *cp = epilogue_value(v.x, v.y, p.epi, cp);
                    }
                }
            }
        }
        return;
    }

    // K split: store this partition's (Re, Im), count in; the last to arrive merges.
    float* base = partials + p.partial_off;
    const size_t plane = (size_t)p.ppitch * p.n;
#pragma unroll
    for (int j = 0; j < G::NT; ++j) {
        const int col = n0 + (j / G::VB) * 16 * G::VB + ty * G::VB + j % G::VB;
#pragma unroll
        for (int i = 0; i < G::MT; ++i) {
            const int row = m0 + (i / G::VA) * 16 * G::VA + tx * G::VA + i % G::VA;
            if (row < p.m && col < p.n) {
                const size_t o = (size_t)col * p.ppitch + row;
                const float2 v = acc_product<BM, BN, MODE>(acc, i, j);
                __stcg(base + (size_t)(2 * part) * plane + o, v.x);
                __stcg(base + (size_t)(2 * part + 1) * plane + o, v.y);
            }
        }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t* ctr = counters + p.counter_off + tile;
        const uint32_t prev = atomicAdd(ctr, 1u);
        const int last = prev == (uint32_t)(p.parts - 1);
        if (last) {
            *ctr = 0;  // ready for the next execution of the plan
        }
        *last_flag = last;
    }
    __syncthreads();
    if (!*last_flag) {
        return;
    }
    __threadfence();
    // Three outputs per step (the most that fits the kernel's registers) so
    // the loads of one partition for all three are in flight together; each
    // output still adds its partitions in order.
    constexpr int U = 3;
    for (int e0 = threadIdx.x; e0 < BM * BN; e0 += U * kThreads) {
        size_t o[U];
        bool ok[U];
        float re[U], im[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = e0 + u * kThreads;
            const int row = m0 + e % BM, col = n0 + e / BM;
            ok[u] = e < BM * BN && row < p.m && col < p.n;
            o[u] = ok[u] ? (size_t)col * p.ppitch + row : 0;
            re[u] = ok[u] ? __ldcg(base + o[u]) : 0.0f;
            im[u] = ok[u] ? __ldcg(base + plane + o[u]) : 0.0f;
        }
        for (int q = 1; q < p.parts; ++q) {
            float tr[U], ti[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                tr[u] = ok[u] ? __ldcg(base + (size_t)(2 * q) * plane + o[u]) : 0.0f;
                ti[u] = ok[u] ? __ldcg(base + (size_t)(2 * q + 1) * plane + o[u]) : 0.0f;
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                re[u] = __fadd_rn(re[u], tr[u]);
                im[u] = __fadd_rn(im[u], ti[u]);
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (ok[u]) {
                const int e = e0 + u * kThreads;
                const int row = m0 + e % BM, col = n0 + e / BM;
                float2 v = make_float2(re[u], im[u]);
                if (p.repair && !finite2(v)) {
                    v = repair_product(p, row, col);
                }
                float2* cp = p.C + (size_t)col * p.ldc + row;
                *cp = epilogue_value(v.x, v.y, p.epi, cp);
            }
        }
    }
}

template <int MODE>
__device__ __forceinline__ void dispatch_task(const BProblem& p, int tile, int part, float2* raw, float* planes,
                                              float* partials, uint32_t* counters, int* last_flag)
{
    switch (p.tile) {
        case 0:
            if constexpr (MODE == kMode3M) {
                run_task<128, 64, MODE>(p, tile, part, raw, planes, partials, counters, last_flag);
            }
            break;
        case 1: run_task<64, 64, MODE>(p, tile, part, raw, planes, partials, counters, last_flag); break;
        case 2: run_task<128, 32, MODE>(p, tile, part, raw, planes, partials, counters, last_flag); break;
        case 3: run_task<32, 128, MODE>(p, tile, part, raw, planes, partials, counters, last_flag); break;
        case 4: run_task<64, 32, MODE>(p, tile, part, raw, planes, partials, counters, last_flag); break;
        default: run_task<32, 32, MODE>(p, tile, part, raw, planes, partials, counters, last_flag); break;
    }
}

// Heterogeneous batch: tasks from a device list (problem, tile, partition).
__global__ void __launch_bounds__(kThreads) batched_kernel(const BProblem* __restrict__ problems,
                                                           const BTask* __restrict__ tasks, int ntasks,
                                                           int* __restrict__ next, float* partials,
                                                           uint32_t* counters)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* raw = reinterpret_cast<float2*>(smem_raw);
    float* planes = reinterpret_cast<float*>(smem_raw + (size_t)kStages * kRawElems * sizeof(float2));
    __shared__ int task_id;
    __shared__ int last_flag;
    for (;;) {
        __syncthreads();  // the previous task's shared-memory reads are done
        if (threadIdx.x == 0) {
            task_id = atomicAdd(next, 1);
        }
        __syncthreads();
        const int t = task_id;
        if (t >= ntasks) {
            return;
        }
        const BTask tk = tasks[t];
        dispatch_task<kMode3M>(problems[tk.problem], tk.tile, tk.part, raw, planes, partials, counters, &last_flag);
    }
}

// Strided batch (and single problems): batch b's problem is `proto` with
// A + b*sA, B + b*sB, C + b*sC and its own partial / counter ranges; task t
// is (b, tile, part) = (t / per_batch, (t % per_batch) / parts, t % parts).
// counters[0] is the task counter; tile counters follow.
template <int MODE>
__global__ void __launch_bounds__(kThreads) strided_kernel(BProblem proto, long long sA, long long sB, long long sC,
                                                           int batch, size_t partial_stride, float* partials,
                                                           uint32_t* counters)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* raw = reinterpret_cast<float2*>(smem_raw);
    float* planes = reinterpret_cast<float*>(smem_raw + (size_t)kStages * kRawElems * sizeof(float2));
    __shared__ int task_id;
    __shared__ int last_flag;
    const int tiles = proto.tiles_m * proto.tiles_n;
    const int per_batch = tiles * proto.parts;
    const long long ntasks = (long long)per_batch * batch;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) {
            task_id = (int)atomicAdd(counters, 1u);
        }
        __syncthreads();
        const int t = task_id;
        if (t >= ntasks) {
            return;
        }
        const int b = t / per_batch, r = t - b * per_batch;
        BProblem p = proto;
        p.A = proto.A + (long long)b * sA;
        p.B = proto.B + (long long)b * sB;
        p.C = proto.C + (long long)b * sC;
        p.partial_off = (size_t)b * partial_stride;
        p.counter_off = 1 + (size_t)b * tiles;
        dispatch_task<MODE>(p, r / proto.parts, r % proto.parts, raw, planes, partials, counters, &last_flag);
    }
}

// ---- one problem, one launch: K partitions merged through the cluster -------
//
// Block (tile, part) of grid (tiles, parts) computes partition `part` of output
// tile `tile` with the same K loop as the persistent kernels; the partitions
// of a tile form one thread-block cluster (cluster dims 1 x parts).  Each block
// leaves its partition's (Re, Im) in its own shared memory; after a cluster
// barrier, block q merges the q-th slice of the tile's outputs, reading every
// partition's value through distributed shared memory and adding them in
// partition order with the merge arithmetic of the drop-in, then applies
// alpha/beta and stores.  A second cluster barrier keeps every block's shared
// memory in place until all reads are done.  Nothing goes through global
// memory but A, B and C: no workspace, no counters, no second launch.  Both
// barriers are reached by every thread of every block (no early exits).
template <int BM, int BN, int MODE>
struct SingleCfg {
    static constexpr int RAWS = (BM + BN) * BK;  // elements per raw slot
    static constexpr int PLS = Cfg<BM, BN, MODE>::A_FLOATS + Cfg<BM, BN, MODE>::B_FLOATS;
    static constexpr size_t SMEM = (size_t)kStages * RAWS * sizeof(float2) + 2 * (size_t)PLS * sizeof(float);
    static_assert((size_t)2 * BM * BN * sizeof(float) <= (size_t)kStages * RAWS * sizeof(float2),
                  "partials exceed the raw slots");
};

__device__ __forceinline__ float ld_cluster_f32(uint32_t addr)
{
    float v;
    asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(addr) : "memory");
    return v;
}

constexpr int kMaxClusterParts = 8;  // portable cluster size

template <int BM, int BN, int MODE>
__global__ void __launch_bounds__(kThreads) single_kernel(const BProblem p)
{
    using G = Cfg<BM, BN, MODE>;
    using S = SingleCfg<BM, BN, MODE>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* raw = reinterpret_cast<float2*>(smem_raw);
    float* planes = reinterpret_cast<float*>(smem_raw + (size_t)kStages * S::RAWS * sizeof(float2));
    const int tile = blockIdx.x, part = blockIdx.y;
    const int tm = tile % p.tiles_m, tn = tile / p.tiles_m;
    const int m0 = tm * BM, n0 = tn * BN;
    const int kbeg = part * p.span;
    const int kend = min(p.k, kbeg + p.span);
    const int klen = kend > kbeg ? kend - kbeg : 0;
    const int tx = thread_tx(), ty = thread_ty();
    AccTile<BM, BN, MODE> acc;
    accumulate<BM, BN, MODE, S::RAWS, S::PLS>(p, m0, n0, kbeg, klen, raw, planes, acc);

    if (p.parts == 1) {
#pragma unroll
        for (int j = 0; j < G::NT; ++j) {
            const int col = n0 + (j / G::VB) * 16 * G::VB + ty * G::VB + j % G::VB;
#pragma unroll
            for (int i = 0; i < G::MT; ++i) {
                const int row = m0 + (i / G::VA) * 16 * G::VA + tx * G::VA + i % G::VA;
                if (row < p.m && col < p.n) {
                    float2 v =
                        acc_product<BM, BN, MODE>(acc, i, j);
                    if (p.repair && !finite2(v)) {
                        v = repair_product(p, row, col);
                    }
                    float2* cp = p.C + (size_t)col * p.ldc + row;
                    *cp = epilogue_value(v.x, v.y, p.epi, cp);
                }
            }
        }
        return;
    }

    // This partition's (Re, Im) at part_re[e], part_im[e], e = c*BM + r (tile
    // coordinates), over the raw slots: every thread's copies have landed and
    // been converted before the K loop's last barrier.
    float* part_re = reinterpret_cast<float*>(raw);
    float* part_im = part_re + BM * BN;
#pragma unroll
    for (int j = 0; j < G::NT; ++j) {
        const int c = (j / G::VB) * 16 * G::VB + ty * G::VB + j % G::VB;
#pragma unroll
        for (int i = 0; i < G::MT; ++i) {
            const int r = (i / G::VA) * 16 * G::VA + tx * G::VA + i % G::VA;
            const float2 v = acc_product<BM, BN, MODE>(acc, i, j);
            part_re[c * BM + r] = v.x;
            part_im[c * BM + r] = v.y;
        }
    }
    cluster_sync();  // every partition's values are in place and visible to the cluster
    const uint32_t re_local = static_cast<uint32_t>(__cvta_generic_to_shared(part_re));
    const uint32_t im_local = static_cast<uint32_t>(__cvta_generic_to_shared(part_im));
    const int per = (BM * BN + p.parts - 1) / p.parts;  // outputs merged by each block
    const int e_end = min(BM * BN, (part + 1) * per);
    for (int e = part * per + (int)threadIdx.x; e < e_end; e += kThreads) {
        const int r = e % BM, c = e / BM;
        const int row = m0 + r, col = n0 + c;
        float tr[kMaxClusterParts], ti[kMaxClusterParts];
#pragma unroll
        for (int q = 0; q < kMaxClusterParts; ++q) {
            if (q < p.parts) {
                tr[q] = ld_cluster_f32(mapa_shared(re_local + 4u * e, q));
                ti[q] = ld_cluster_f32(mapa_shared(im_local + 4u * e, q));
            }
        }
        float re = tr[0], im = ti[0];
#pragma unroll
        for (int q = 1; q < kMaxClusterParts; ++q) {
            if (q < p.parts) {
                re = __fadd_rn(re, tr[q]);
                im = __fadd_rn(im, ti[q]);
            }
        }
        if (row < p.m && col < p.n) {
            float2 v = make_float2(re, im);
            if (p.repair && !finite2(v)) {
                v = repair_product(p, row, col);
            }
            float2* cp = p.C + (size_t)col * p.ldc + row;
            *cp = epilogue_value(v.x, v.y, p.epi, cp);
        }
    }
    cluster_sync();  // no block leaves while others may still read its shared memory
}

template <int MODE>
cudaError_t launch_single_tile(cudaStream_t s, const BProblem& bp, int tile)
{
    auto run = [&](auto kernel, size_t smem) -> cudaError_t {
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) {
            return e;
        }
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3((unsigned)(bp.tiles_m * bp.tiles_n), (unsigned)bp.parts, 1);
        cfg.blockDim = dim3(kThreads, 1, 1);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 1;
        attr[0].val.clusterDim.y = (unsigned)bp.parts;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        return cudaLaunchKernelEx(&cfg, kernel, bp);
    };
    switch (tile) {
        case 0:
            if constexpr (MODE == kMode3M) {
                return run(single_kernel<128, 64, MODE>, SingleCfg<128, 64, MODE>::SMEM);
            }
            return cudaErrorInvalidValue;
        case 1: return run(single_kernel<64, 64, MODE>, SingleCfg<64, 64, MODE>::SMEM);
        case 2: return run(single_kernel<128, 32, MODE>, SingleCfg<128, 32, MODE>::SMEM);
        case 3: return run(single_kernel<32, 128, MODE>, SingleCfg<32, 128, MODE>::SMEM);
        case 4: return run(single_kernel<64, 32, MODE>, SingleCfg<64, 32, MODE>::SMEM);
        default: return run(single_kernel<32, 32, MODE>, SingleCfg<32, 32, MODE>::SMEM);
    }
}

}  // namespace
}  // namespace cg3m

using namespace cg3m;

struct cg3mBatchPlan {
    int device = -1;
    int count = 0;
    int sm_count = 148;
    int blocks_per_sm = 1;
    std::vector<int> index;  // caller's problem i -> host[] position, -1 for quick returns
    std::vector<BProblem> host;
    std::vector<BTask> tasks;
    BProblem* d_problems = nullptr;
    BTask* d_tasks = nullptr;
    float* d_partials = nullptr;
    uint32_t* d_counters = nullptr;
    int* d_next = nullptr;
    cudaStream_t capture_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~cg3mBatchPlan()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (capture_stream) cudaStreamDestroy(capture_stream);
        cudaFree(d_problems);
        cudaFree(d_tasks);
        cudaFree(d_partials);
        cudaFree(d_counters);
        cudaFree(d_next);
    }
};

namespace {

// One candidate table: the largest tile area allowed and the cap on K
// partitions.  Each problem takes the allowed tile with the least estimated
// time -- padded work (tiles x BM x BN x (k + 16)) over the tile's relative
// FFMA efficiency -- and is split along K only when one of its tile tasks
// would exceed a quarter of the batch's average work per SM (the longest task
// bounds the persistent schedule), keeping >= 128 K terms per partition.
struct Policy {
    int max_area;
    int split_cap;
};

constexpr Policy kPolicies[] = {{8192, 1}, {8192, 2}, {8192, 4}, {8192, 8}, {4096, 1},
                                {4096, 2}, {4096, 4}, {4096, 8}, {2048, 1}, {2048, 4}};
constexpr Policy kDefaultPolicy = {8192, 4};

// Relative FFMA efficiency of each tile shape (per output-element-term).
constexpr double kTileEfficiency[kTileCount] = {1.0, 0.85, 0.8, 0.8, 0.65, 0.45};

int span_for(int k, int parts) { return ceil_div(ceil_div(k, 16), parts) * 16; }

// The allowed tile with the least estimated time for p; returns that time
// (padded work over efficiency) and sets tile, tiles_m, tiles_n.
double choose_tile(BProblem& p, int max_area, int mode)
{
    int best = kTileCount - 1;
    double best_cost = 1e300;
    for (int t = 0; t < kTileCount; ++t) {
        if (tile_bm(t) * tile_bn(t) > max_area || (mode == kMode4M && t == 0)) {
            continue;
        }
        const double work =
            (double)ceil_div(p.m, tile_bm(t)) * ceil_div(p.n, tile_bn(t)) * tile_bm(t) * tile_bn(t) * (p.k + 16);
        const double cost = work / kTileEfficiency[t];
        if (cost < best_cost) {
            best_cost = cost;
            best = t;
        }
    }
    p.tile = best;
    p.tiles_m = ceil_div(p.m, tile_bm(best));
    p.tiles_n = ceil_div(p.n, tile_bn(best));
    return best_cost;
}

// K partitions of p given the schedule's average work per SM.
void choose_parts(BProblem& p, int split_cap, double per_sm)
{
    int parts = 1;
    if (split_cap > 1 && p.k >= 256) {
        const double task = (double)tile_bm(p.tile) * tile_bn(p.tile) * (p.k + 16) / kTileEfficiency[p.tile];
        const int want = (int)std::ceil(task / (0.25 * per_sm));
        parts = std::max(1, std::min({want, split_cap, p.k / 128}));
    }
    p.parts = parts;
    p.span = span_for(p.k, parts);
    while (p.parts > 1 && (p.parts - 1) * p.span >= p.k) {
        --p.parts;
        p.span = span_for(p.k, p.parts);
    }
    if (p.parts == 1) {
        p.span = p.k;
    }
}

void apply_policy(std::vector<BProblem>& ps, const Policy& pol, int sm_count)
{
    double total = 0.0;
    for (auto& p : ps) {
        total += choose_tile(p, pol.max_area, kMode3M);
    }
    const double per_sm = total / std::max(sm_count, 1);
    for (auto& p : ps) {
        choose_parts(p, pol.split_cap, per_sm);
    }
}

// Lays out partials and counters, and lists the tasks by decreasing work.
void build_tasks(std::vector<BProblem>& ps, std::vector<BTask>& tasks, size_t* partial_floats,
                 size_t* counter_words)
{
    std::vector<std::pair<double, BTask>> v;
    size_t pf = 0, cw = 0;
    for (size_t i = 0; i < ps.size(); ++i) {
        BProblem& p = ps[i];
        p.ppitch = (int)align_up((size_t)p.m, 32);
        p.partial_off = pf;
        p.counter_off = cw;
        if (p.parts > 1) {
            pf += (size_t)p.ppitch * p.n * 2 * p.parts;
            cw += (size_t)p.tiles_m * p.tiles_n;
        }
        const double cost =
            (double)tile_bm(p.tile) * tile_bn(p.tile) * ((p.parts > 1 ? p.span : p.k) + 16) / kTileEfficiency[p.tile];
        for (int t = 0; t < p.tiles_m * p.tiles_n; ++t) {
            for (int q = 0; q < p.parts; ++q) {
                v.push_back({cost, BTask{(int)i, t, q, 0}});
            }
        }
    }
    std::stable_sort(v.begin(), v.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    tasks.clear();
    tasks.reserve(v.size());
    for (auto& x : v) {
        tasks.push_back(x.second);
    }
    *partial_floats = pf;
    *counter_words = cw;
}

void release_device(cg3mBatchPlan* plan)
{
    if (plan->exec) {
        cudaGraphExecDestroy(plan->exec);
        plan->exec = nullptr;
    }
    if (plan->graph) {
        cudaGraphDestroy(plan->graph);
        plan->graph = nullptr;
    }
    cudaFree(plan->d_problems);
    cudaFree(plan->d_tasks);
    cudaFree(plan->d_partials);
    cudaFree(plan->d_counters);
    plan->d_problems = nullptr;
    plan->d_tasks = nullptr;
    plan->d_partials = nullptr;
    plan->d_counters = nullptr;
}

// (Re)builds the task list of `ps` under `pol` and uploads it with zeroed
// tile counters.
cudaError_t materialise(cg3mBatchPlan* plan, std::vector<BProblem>& ps, const Policy& pol)
{
    release_device(plan);
    apply_policy(ps, pol, plan->sm_count);
    size_t pf = 0, cw = 0;
    build_tasks(ps, plan->tasks, &pf, &cw);
    cudaError_t e = cudaMalloc(&plan->d_problems, sizeof(BProblem) * std::max<size_t>(1, ps.size()));
    if (e == cudaSuccess) e = cudaMalloc(&plan->d_tasks, sizeof(BTask) * std::max<size_t>(1, plan->tasks.size()));
    if (e == cudaSuccess) e = cudaMalloc(&plan->d_partials, sizeof(float) * std::max<size_t>(1, pf));
    if (e == cudaSuccess) e = cudaMalloc(&plan->d_counters, sizeof(uint32_t) * std::max<size_t>(1, cw));
    if (e == cudaSuccess && plan->d_next == nullptr) e = cudaMalloc(&plan->d_next, sizeof(int));
    if (e == cudaSuccess && !ps.empty())
        e = cudaMemcpy(plan->d_problems, ps.data(), sizeof(BProblem) * ps.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !plan->tasks.empty())
        e = cudaMemcpy(plan->d_tasks, plan->tasks.data(), sizeof(BTask) * plan->tasks.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(plan->d_counters, 0, sizeof(uint32_t) * std::max<size_t>(1, cw));
    // Pageable uploads may still be in flight on the legacy stream when
    // cudaMemcpy returns; the plan's launches go to other streams.
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return e;
}

cudaError_t launch(cg3mBatchPlan* plan, cudaStream_t s)
{
    if (plan->tasks.empty()) {
        return cudaSuccess;
    }
    cudaError_t e = cudaMemsetAsync(plan->d_next, 0, sizeof(int), s);
    if (e != cudaSuccess) {
        return e;
    }
    const int grid = (int)std::min<size_t>(plan->tasks.size(), (size_t)plan->sm_count * plan->blocks_per_sm);
    batched_kernel<<<grid, kThreads, kSmemBytes, s>>>(plan->d_problems, plan->d_tasks, (int)plan->tasks.size(),
                                                      plan->d_next, plan->d_partials, plan->d_counters);
    return cudaGetLastError();
}

std::mutex g_tune_mutex;
std::map<std::string, Policy> g_tuned;  // batch signature -> chosen policy

std::string signature(int device, const std::vector<BProblem>& ps)
{
    std::string s = std::to_string(device) + ":";
    s.reserve(ps.size() * 24);
    char b[80];
    for (const auto& p : ps) {
        std::snprintf(b, sizeof b, "%d%d,%d,%d,%d,%d;", p.ta, p.tb, p.m, p.n, p.k, p.epi.beta_zero);
        s += b;
    }
    return s;
}

// Times every candidate policy (median of 3 launches after one warm-up) with
// the caller's A and B and a scratch C, and returns the fastest.  The
// caller's C is never written.
Policy autotune(cg3mBatchPlan* plan, cudaStream_t s)
{
    size_t celems = 0;
    for (const auto& p : plan->host) {
        celems += (size_t)p.ldc * p.n;
    }
    float2* scratch = nullptr;
    if (cudaMalloc(&scratch, sizeof(float2) * std::max<size_t>(1, celems)) != cudaSuccess) {
        cudaGetLastError();
        return kDefaultPolicy;
    }
    cudaMemsetAsync(scratch, 0, sizeof(float2) * std::max<size_t>(1, celems), s);
    std::vector<BProblem> trial = plan->host;
    size_t off = 0;
    for (auto& p : trial) {
        p.C = scratch + off;
        off += (size_t)p.ldc * p.n;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    Policy best = kDefaultPolicy;
    float best_ms = 1e30f;
    for (const Policy& pol : kPolicies) {
        if (materialise(plan, trial, pol) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        float times[3] = {0, 0, 0};
        bool ok = true;
        for (int r = 0; r < 4 && ok; ++r) {
            ok = cudaEventRecord(e0, s) == cudaSuccess && launch(plan, s) == cudaSuccess &&
                 cudaEventRecord(e1, s) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess;
            if (ok && r > 0) {
                cudaEventElapsedTime(&times[r - 1], e0, e1);
            }
        }
        if (!ok) {
            cudaGetLastError();
            continue;
        }
        std::sort(times, times + 3);
        if (times[1] < best_ms) {
            best_ms = times[1];
            best = pol;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamSynchronize(s);
    cudaFree(scratch);
    return best;
}

}  // namespace

namespace cg3m {

bool make_strided_plan(const Problem& p, int mode, int batch, int sm_count, StridedPlan* out)
{
    if (batch <= 0 || p.m <= 0 || p.n <= 0 || p.k <= 0 || (mode != kMode3M && mode != kMode4M)) {
        return false;
    }
    BProblem bp{};
    bp.m = p.m;
    bp.n = p.n;
    bp.k = p.k;
    const double one = choose_tile(bp, 8192, mode);
    choose_parts(bp, 4, one * batch / std::max(sm_count, 1));
    StridedPlan pl{};
    pl.tile = bp.tile;
    pl.tile_m = tile_bm(bp.tile);
    pl.tile_n = tile_bn(bp.tile);
    pl.parts = bp.parts;
    pl.span = bp.span;
    pl.tiles = bp.tiles_m * bp.tiles_n;
    pl.ppitch = (int)align_up((size_t)p.m, 32);
    pl.partial_stride = bp.parts > 1 ? (size_t)pl.ppitch * p.n * 2 * bp.parts : 0;
    pl.counters = 1 + (size_t)batch * pl.tiles;
    pl.partial_off = align_up(pl.counters * sizeof(uint32_t), 256);
    pl.bytes = pl.partial_off + (size_t)batch * pl.partial_stride * sizeof(float);
    *out = pl;
    return true;
}

int single_tile_bm(int tile) { return tile_bm(tile); }
int single_tile_bn(int tile) { return tile_bn(tile); }

// Time model of the one-launch kernel (three-product mode), in microseconds,
// fitted on B200 to 1100 timed (shape, tile, partitions) launches (median
// error 1.5 %).  Clusters of `parts` blocks run in waves of as many clusters
// as fit at once (cudaOccupancyMaxActiveClusters on a 148-SM B200, scaled for
// other SM counts); each wave costs the tile's fixed part (first copies,
// epilogue) plus span x its per-term time, and tiles that share an SM (64 x 32:
// two blocks, 32 x 32: three) add a per-term cost for every block on the
// busiest SM.  The cluster merge costs a little per partition.
namespace {
struct SingleCost {
    double fixed_us, term_ns, shared_term_ns;
};
constexpr SingleCost kSingleCost[kTileCount] = {{4.96, 183.8, 0.0},  {3.55, 129.2, 0.0}, {3.31, 176.6, 0.0},
                                                {3.29, 118.7, 0.0},  {2.99, 51.4, 59.7}, {2.26, 15.3, 43.7}};
constexpr int kSingleOcc[kTileCount] = {1, 1, 1, 1, 2, 3};
// Clusters resident at once on 148 SMs, by blocks per SM (1..3) and cluster size (1..8).
constexpr int kClusterCap[3][kMaxClusterParts] = {{148, 74, 45, 33, 26, 22, 15, 15},
                                                  {296, 148, 93, 71, 56, 45, 37, 33},
                                                  {444, 222, 142, 104, 82, 71, 56, 48}};
constexpr double kSingleMergePerPartUs = 0.146;
}  // namespace

double plan_single(int m, int n, int k, int mode, int sm_count, int forced_tile, int forced_parts, int* tile,
                   int* parts)
{
    sm_count = std::max(sm_count, 1);
    double best = 1e300;
    int bt = kTileCount - 1, bp = 1;
    for (int t = 0; t < kTileCount; ++t) {
        if ((forced_tile >= 0 && t != forced_tile) || (mode == kMode4M && t == 0)) {
            continue;
        }
        const long long tiles = (long long)ceil_div(m, tile_bm(t)) * ceil_div(n, tile_bn(t));
        for (int q = 1; q <= kMaxClusterParts; ++q) {
            if (forced_parts > 0 && q != forced_parts) {
                continue;
            }
            const int span = q == 1 ? k : span_for(k, q);
            if (q > 1 && (q - 1) * span >= k) {
                continue;
            }
            const long long cap =
                std::max<long long>(1, (long long)kClusterCap[kSingleOcc[t] - 1][q - 1] * sm_count / 148);
            const long long waves = (tiles + cap - 1) / cap;
            const long long load = (tiles * q + sm_count - 1) / sm_count;
            const SingleCost& c = kSingleCost[t];
            // Four-product mode: four FFMA per output and K term instead of
            // three (the per-term costs scaled by that ratio, not fitted).
            const double fma = mode == kMode4M ? 4.0 / 3.0 : 1.0;
            double us = (double)waves * c.fixed_us +
                        span * 1e-3 * fma * ((double)waves * c.term_ns + (double)load * c.shared_term_ns);
            if (q > 1) {
                us += kSingleMergePerPartUs * q;
            }
            if (us < best) {
                best = us;
                bt = t;
                bp = q;
            }
        }
    }
    if (tile != nullptr) {
        *tile = bt;
    }
    if (parts != nullptr) {
        *parts = bp;
    }
    return best;
}

cudaError_t launch_single(cudaStream_t s, const Problem& p, int mode, int repair, int tile, int parts)
{
    if (p.m <= 0 || p.n <= 0 || p.k <= 0 || parts < 1 || parts > kMaxClusterParts || tile < 0 ||
        tile >= kTileCount || (mode != kMode3M && mode != kMode4M) || (mode == kMode4M && tile == 0)) {
        return cudaErrorInvalidValue;
    }
    BProblem bp{};
    bp.ta = p.transa;
    bp.tb = p.transb;
    bp.m = p.m;
    bp.n = p.n;
    bp.k = p.k;
    const bool beta_zero = p.br == 0.0f && p.bi == 0.0f;
    const bool unit = p.ar == 1.0f && p.ai == 0.0f && beta_zero;
    bp.epi = EpiParams{p.ar, p.ai, p.br, p.bi, unit ? 1 : 0, beta_zero ? 1 : 0};
    bp.A = static_cast<const float2*>(p.A);
    bp.B = static_cast<const float2*>(p.B);
    bp.C = static_cast<float2*>(p.C);
    bp.lda = p.lda;
    bp.ldb = p.ldb;
    bp.ldc = p.ldc;
    bp.tile = tile;
    bp.repair = repair;
    bp.parts = parts;
    bp.span = span_for(p.k, parts);
    if ((parts - 1) * bp.span >= p.k) {
        return cudaErrorInvalidValue;  // the caller passes a partition count whose last part is non-empty
    }
    if (parts == 1) {
        bp.span = p.k;
    }
    bp.tiles_m = ceil_div(p.m, tile_bm(tile));
    bp.tiles_n = ceil_div(p.n, tile_bn(tile));
    const cudaError_t e =
        mode == kMode3M ? launch_single_tile<kMode3M>(s, bp, tile) : launch_single_tile<kMode4M>(s, bp, tile);
    return e != cudaSuccess ? e : cudaGetLastError();
}

cudaError_t launch_strided(cudaStream_t s, const Problem& p, int mode, int repair, long long sA, long long sB,
                           long long sC, int batch, const StridedPlan& plan, void* ws, int sm_count)
{
    BProblem proto{};
    proto.ta = p.transa;
    proto.tb = p.transb;
    proto.m = p.m;
    proto.n = p.n;
    proto.k = p.k;
    const bool beta_zero = p.br == 0.0f && p.bi == 0.0f;
    const bool unit = p.ar == 1.0f && p.ai == 0.0f && beta_zero;
    proto.epi = EpiParams{p.ar, p.ai, p.br, p.bi, unit ? 1 : 0, beta_zero ? 1 : 0};
    proto.A = static_cast<const float2*>(p.A);
    proto.B = static_cast<const float2*>(p.B);
    proto.C = static_cast<float2*>(p.C);
    proto.lda = p.lda;
    proto.ldb = p.ldb;
    proto.ldc = p.ldc;
    proto.tile = plan.tile;
    proto.repair = repair;
    proto.parts = plan.parts;
    proto.span = plan.span;
    proto.tiles_m = ceil_div(p.m, plan.tile_m);
    proto.tiles_n = ceil_div(p.n, plan.tile_n);
    proto.ppitch = plan.ppitch;
    uint32_t* counters = static_cast<uint32_t*>(ws);
    float* partials = reinterpret_cast<float*>(static_cast<char*>(ws) + plan.partial_off);
    cudaError_t e = cudaMemsetAsync(counters, 0, plan.counters * sizeof(uint32_t), s);
    if (e != cudaSuccess) {
        return e;
    }
    const long long ntasks = (long long)plan.tiles * plan.parts * batch;
    const int grid = (int)std::min<long long>(ntasks, (long long)std::max(sm_count, 1));
    if (mode == kMode3M) {
        e = cudaFuncSetAttribute(strided_kernel<kMode3M>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kSmemBytes);
        if (e == cudaSuccess) {
            strided_kernel<kMode3M><<<grid, kThreads, kSmemBytes, s>>>(proto, sA, sB, sC, batch, plan.partial_stride,
                                                                       partials, counters);
        }
    } else {
        e = cudaFuncSetAttribute(strided_kernel<kMode4M>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kSmemBytes);
        if (e == cudaSuccess) {
            strided_kernel<kMode4M><<<grid, kThreads, kSmemBytes, s>>>(proto, sA, sB, sC, batch, plan.partial_stride,
                                                                       partials, counters);
        }
    }
    return e != cudaSuccess ? e : cudaGetLastError();
}

}  // namespace cg3m

extern "C" {

cg3mStatus_t cg3mBatchPlanCreate(cg3mHandle_t handle, const cg3mProblem* problems, int count, int tune,
                                 cg3mBatchPlan_t* out, int* bad_index)
{
    if (handle == nullptr) {
        return CG3M_STATUS_HANDLE_IS_NULLPTR;
    }
    if (out == nullptr || count < 0 || (count > 0 && problems == nullptr)) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    *out = nullptr;
    std::vector<BProblem> ps;
    std::vector<int> index((size_t)count, -1);
    for (int i = 0; i < count; ++i) {
        const cg3mProblem& q = problems[i];
        int action = 0;
        const cg3mStatus_t st = validate(q.transa, q.transb, q.m, q.n, q.k, &q.alpha, q.A, q.lda, q.B, q.ldb, &q.beta,
                                         q.C, q.ldc, true, &action);
        if (st != CG3M_STATUS_SUCCESS) {
            if (bad_index != nullptr) {
                *bad_index = i;
            }
            return st;
        }
        if (action == 0) {
            continue;  // quick return: C unchanged
        }
        BProblem p{};
        p.ta = q.transa;
        p.tb = q.transb;
        p.m = q.m;
        p.n = q.n;
        p.k = action == 1 ? 0 : q.k;
        const bool beta_zero = q.beta.real == 0.0f && q.beta.imag == 0.0f;
        const bool unit = q.alpha.real == 1.0f && q.alpha.imag == 0.0f && beta_zero;
        p.epi = EpiParams{q.alpha.real, q.alpha.imag, q.beta.real, q.beta.imag, unit ? 1 : 0, beta_zero ? 1 : 0};
        p.A = reinterpret_cast<const float2*>(q.A);
        p.B = reinterpret_cast<const float2*>(q.B);
        p.C = reinterpret_cast<float2*>(q.C);
        p.lda = q.lda;
        p.ldb = q.ldb;
        p.ldc = q.ldc;
        index[(size_t)i] = (int)ps.size();
        ps.push_back(p);
    }
    cg3mBatchPlan* plan = new (std::nothrow) cg3mBatchPlan();
    if (plan == nullptr) {
        return CG3M_STATUS_ALLOC_FAILED;
    }
    plan->count = count;
    plan->index = std::move(index);
    plan->host = std::move(ps);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&plan->sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaFuncSetAttribute(batched_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&plan->blocks_per_sm, batched_kernel, kThreads, kSmemBytes) !=
            cudaSuccess) {
        cudaGetLastError();
        delete plan;
        return CG3M_STATUS_INTERNAL_ERROR;
    }
    plan->device = dev;
    plan->blocks_per_sm = std::max(1, plan->blocks_per_sm);
    Policy pol = kDefaultPolicy;
    const std::string sig = signature(dev, plan->host);
    bool cached = false;
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        auto it = g_tuned.find(sig);
        if (it != g_tuned.end()) {
            pol = it->second;
            cached = true;
        }
    }
    if (tune && !cached && !plan->host.empty()) {
        pol = autotune(plan, handle->stream);
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        g_tuned[sig] = pol;
    }
    if (materialise(plan, plan->host, pol) != cudaSuccess) {
        cudaGetLastError();
        delete plan;
        return CG3M_STATUS_ALLOC_FAILED;
    }
    *out = plan;
    return CG3M_STATUS_SUCCESS;
}

cg3mStatus_t cg3mBatchPlanExecute(cg3mHandle_t handle, cg3mBatchPlan_t plan, int use_graph)
{
    if (handle == nullptr) {
        return CG3M_STATUS_HANDLE_IS_NULLPTR;
    }
    if (plan == nullptr) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    if (!use_graph || plan->tasks.empty()) {
        return launch(plan, handle->stream) == cudaSuccess ? CG3M_STATUS_SUCCESS : CG3M_STATUS_EXECUTION_FAILED;
    }
    if (plan->exec == nullptr) {
        if (plan->capture_stream == nullptr &&
            cudaStreamCreateWithFlags(&plan->capture_stream, cudaStreamNonBlocking) != cudaSuccess) {
            return CG3M_STATUS_INTERNAL_ERROR;
        }
        if (cudaStreamBeginCapture(plan->capture_stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
            return CG3M_STATUS_EXECUTION_FAILED;
        }
        const cudaError_t le = launch(plan, plan->capture_stream);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(plan->capture_stream, &g);
        if (le != cudaSuccess || ce != cudaSuccess || g == nullptr) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return CG3M_STATUS_EXECUTION_FAILED;
        }
        plan->graph = g;
        if (cudaGraphInstantiate(&plan->exec, g, 0) != cudaSuccess) {
            cudaGetLastError();
            plan->exec = nullptr;
            return CG3M_STATUS_EXECUTION_FAILED;
        }
    }
    return cudaGraphLaunch(plan->exec, handle->stream) == cudaSuccess ? CG3M_STATUS_SUCCESS
                                                                      : CG3M_STATUS_EXECUTION_FAILED;
}

cg3mStatus_t cg3mBatchPlanDestroy(cg3mBatchPlan_t plan)
{
    if (plan == nullptr) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    // Work enqueued with the plan may still read its task list.
    if (plan->device >= 0) {
        int cur = 0;
        cudaGetDevice(&cur);
        cudaSetDevice(plan->device);
        cudaDeviceSynchronize();
        cudaSetDevice(cur);
    }
    delete plan;
    return CG3M_STATUS_SUCCESS;
}

cg3mStatus_t cg3mBatchPlanDescribe(cg3mBatchPlan_t plan, int* tile_m, int* tile_n, int* k_partitions)
{
    if (plan == nullptr) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    for (int i = 0; i < plan->count; ++i) {
        const int h = plan->index[(size_t)i];
        const BProblem* p = h >= 0 ? &plan->host[(size_t)h] : nullptr;
        if (tile_m) tile_m[i] = p ? tile_bm(p->tile) : 0;
        if (tile_n) tile_n[i] = p ? tile_bn(p->tile) : 0;
        if (k_partitions) k_partitions[i] = p ? (p->k > 0 ? p->parts : 0) : 0;
    }
    return CG3M_STATUS_SUCCESS;
}

}  // extern "C"
