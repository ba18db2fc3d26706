// ozaki.cu -- FP64-accurate recompute of the flagged outputs of dense tiles on
// the tensor cores: the rounding-correction pass of the tensor-core forms.
//
// The reference recomputes flagged outputs with its segmented FP32 replay
// (cgemm3m_rounding_kernel.cpp:192-404); the tensor-core forms of this library
// promise instead that every flagged output is within one FP32 rounding of the
// exact product.  Recomputing ~3/4 of a 4096^3 product in FP64 on the CUDA
// cores takes ~24 ms at this GPU's FP64 rate, so the exact products run on the
// int8 tensor cores as error-free slice products (the splitting scheme of
// Ozaki, Ogita, Oishi and Rump, "Error-free transformations of matrix
// multiplication by using fast routines of matrix multiplication and its
// applications", Numer. Algorithms 59 (2012), with int8 slices as in Ootomo,
// Ozaki and Yokota, "DGEMM on integer matrix multiplication unit", IJHPCA 2024):
//
//   1. ozaki_split_kernel: every op(A) row i and op(B) column j gets a power
//      of two 2^E > max |x| over the row (real and imaginary parts together),
//      and each part x * 2^-E in (-1, 1) is cut into S = 8 slices of 7 bits:
//      q_s = trunc(r_{s-1} * 2^7), r_s = r_{s-1} * 2^7 - q_s (exact steps), so
//      x = 2^E (sum_s q_s 2^-7s + rho), |rho| < 2^-7S, q_s in [-127, 127].
//   2. ozaki_pair_kernel: for each diagonal d = s + t (2 .. S+1) the int8
//      products sum_k q_s(A) q_t(B) of all pairs on the diagonal are exact in
//      the int32 TMEM accumulators (|sum| <= 2 * 8 * 4096 * 127^2 < 2^31):
//        Re_d = sum Ar_s Br_t + Ai_s (-Bi_t),  Im_d = sum Ar_s Bi_t + Ai_s Br_t;
//      after each diagonal the epilogue adds Re_d 2^-7d, Im_d 2^-7d to FP64
//      partial sums (global, L2-resident while the tile runs), and after the
//      last one scales by 2^(E_i + F_j).
//   3. The dropped terms (pairs with s + t > S + 1 and the remainders rho)
//      are bounded per real product and term by (S + 1) 2^-7S, so
//        |error| <= 2^(E_i + F_j) * 2n (S + 1) 2^-7S  per component.
//      An output is written only when both components exceed 2^25 times that
//      bound (so the result, rounded to FP32, is within one FP32 rounding of
//      the exact product); otherwise it is marked for the FP64 per-output
//      kernel, as are outputs whose row or column holds a non-finite value.
//
// B200 design: a cluster of two CTAs per 256 x 256 output tile
// (tcgen05.mma.cta_group::2.kind::i8, M = 256, N = 256, K = 32): CTA r stages
// rows [128r, 128r + 128) of the A slices and columns [128r, 128r + 128) of
// the B slices, 64-byte K rows with the 64-byte swizzle, 40 KB per stage
// (Ar_s, Ai_s | Br_t, Bi_t, -Bi_t) in a 5-stage ring; each CTA's TMEM holds
// its 128 rows x 256 columns of Re (columns 0..255) and Im (256..511).  Warp 0
// of both CTAs issues the TMA copies (completion on the even CTA's barrier),
// one thread of the even CTA issues every MMA, warps 2..9 of both CTAs drain
// the accumulators after each diagonal.  Every wait is bounded.
#include "cg3m_internal.h"
#include "ptx.cuh"

namespace cg3m {

namespace {

// Slices per operand part.  The row exponent is shared by the real and the
// imaginary part, so a part much smaller than the other spends its leading
// slices on zeros; with 7 slices ~6 % of the flagged outputs of the precision
// form's data (Im scaled by 2^e, |e| <= 8) could not be certified at n = 2048,
// with 8 slices the bound is 2^7 tighter.
constexpr int kOzS = 8;
constexpr int kOzLastDiag = kOzS + 1;        // diagonals d = s + t in [2, S + 1]
constexpr int OZ_TILE_M = kOzakiTile;        // output rows of a pair tile (M of the pair MMA)
constexpr int OZ_ROWS = 128;                 // A rows staged by one CTA
constexpr int OZ_BK = 64;                    // K bytes per staged row (64-byte swizzle)
constexpr int OZ_PLANE = OZ_ROWS * OZ_BK;    // 8 KB
constexpr int kOzEpiWarps = 8;
constexpr int kOzThreads = (2 + kOzEpiWarps) * 32;
constexpr int kOzNonFinite = 1 << 20;          // exponent marker: the row or column holds Inf/NaN
constexpr int kOzZero = -(1 << 20);            // exponent marker: the row or column is all zero

// A pair tile is 256 rows x TN columns (TN = N of the pair MMA): each CTA
// stages TN / 2 columns of the B slices; a stage holds Ar_s, Ai_s | Br_t,
// Bi_t, -Bi_t.
template <int TN>
struct OzGeom {
    static constexpr int BCOLS = TN / 2;
    static constexpr int B_PLANE = BCOLS * OZ_BK;
    static constexpr int STAGE = 2 * OZ_PLANE + 3 * B_PLANE;
    static constexpr int STAGES = (208 * 1024) / STAGE;
    static constexpr size_t SMEM = (size_t)STAGES * STAGE + 1024 + 256;
    static constexpr int GRAN_N = TN / 16;  // 16 x 16 count tiles across the pair tile
    static_assert(STAGE % 1024 == 0 && B_PLANE % 1024 == 0, "plane tiles start on 1024-byte boundaries");
    static_assert(kOzThreads >= 16 * GRAN_N, "one thread per count tile in the density check");
    static_assert(BCOLS % 16 == 0, "epilogue chunks of 16 columns");
};

struct OzParams {
    int n;
    int kblocks;             // 64-byte K blocks
    int tiles_m, tiles_n;    // pair tiles along the rows and the columns
    const int* E;            // op(A) row exponents
    const int* F;            // op(B) column exponents
    const uint32_t* flag_bits;
    const uint32_t* tile_count;
    uint32_t* stats;
    uint32_t* fallback_bits;
    double2* partial;        // n x n, column-major
    float2* C;
    double thresh;           // 2^25 (1 + 2^-20) * 2n (S + 1) 2^-7S
    int* status;
};

__device__ __forceinline__ bool flag_at(const uint32_t* bits, size_t idx)
{
    return (bits[idx >> 5] >> (idx & 31)) & 1u;
}

// ---- 1. slices ---------------------------------------------------------------------

// One block per op(A) row (blockIdx.x < n) or op(B) column.  Plane layout:
// [plane][row][kpitch] int8, A planes 2(s-1) + {0 re, 1 im}, B planes
// 3(t-1) + {0 re, 1 im, 2 -im}.
__global__ void __launch_bounds__(256) ozaki_split_kernel(int n, int pitch, const float2* __restrict__ rows_a,
                                                          const float2* __restrict__ rows_b, int8_t* __restrict__ pa,
                                                          int8_t* __restrict__ pb, int kpitch, size_t plane_bytes,
                                                          int* __restrict__ E, int* __restrict__ F)
{
    __shared__ float wmax[8];
    __shared__ int wbad[8];
    const int r = blockIdx.x;
    const bool is_a = r < n;
    const int row = is_a ? r : r - n;
    const float2* src = (is_a ? rows_a : rows_b) + (size_t)row * pitch;
    const int tid = threadIdx.x;
    float m = 0.0f;
    int bad = 0;
    for (int k = tid; k < n; k += 256) {
        const float2 x = src[k];
        bad |= !isfinite(x.x) || !isfinite(x.y);
        m = fmaxf(m, fmaxf(fabsf(x.x), fabsf(x.y)));
    }
#pragma unroll
    for (int off = 16; off >= 1; off /= 2) {
        m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
        bad |= __shfl_xor_sync(0xffffffffu, bad, off);
    }
    if ((tid & 31) == 0) {
        wmax[tid >> 5] = m;
        wbad[tid >> 5] = bad;
    }
    __syncthreads();
    float amax = 0.0f;
    int any_bad = 0;
    for (int w = 0; w < 8; ++w) {
        amax = fmaxf(amax, wmax[w]);
        any_bad |= wbad[w];
    }
    // 2^(e-1) <= amax < 2^e, so every part scaled by 2^-e lies in (-1, 1).
    const int e = any_bad ? kOzNonFinite : amax > 0.0f ? ilogbf(amax) + 1 : kOzZero;
    if (tid == 0) {
        (is_a ? E : F)[row] = e;
    }
    const bool usable = !any_bad && amax > 0.0f;
    const double scale = usable ? ldexp(1.0, -e) : 0.0;
    int8_t* dst = (is_a ? pa : pb) + (size_t)row * kpitch;
    const int planes_per_slice = is_a ? 2 : 3;
    // Four consecutive K terms per thread: 4-byte stores into every plane.
    for (int k0 = tid * 4; k0 < n; k0 += 256 * 4) {
        double xr[4], xi[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int k = k0 + u;
            const float2 x = (k < n && usable) ? src[k] : make_float2(0.0f, 0.0f);
            xr[u] = (double)x.x * scale;  // exact: a power-of-two scaling in FP64
            xi[u] = (double)x.y * scale;
        }
#pragma unroll
        for (int s = 0; s < kOzS; ++s) {
            signed char vr[4], vi[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const double yr = xr[u] * 128.0, yi = xi[u] * 128.0;  // exact
                const double tr = trunc(yr), ti = trunc(yi);         // |t| <= 127
                xr[u] = yr - tr;                                      // exact: the fraction of y
                xi[u] = yi - ti;
                vr[u] = (signed char)(int)tr;
                vi[u] = (signed char)(int)ti;
            }
            int8_t* base = dst + (size_t)(planes_per_slice * s) * plane_bytes;
            // K beyond n is never read (the tensor maps stop at n), so whole
            // 4-byte groups may be stored while k0 < n <= kpitch.
            *reinterpret_cast<char4*>(base + k0) = make_char4(vr[0], vr[1], vr[2], vr[3]);
            *reinterpret_cast<char4*>(base + plane_bytes + k0) = make_char4(vi[0], vi[1], vi[2], vi[3]);
            if (!is_a) {
                *reinterpret_cast<char4*>(base + 2 * plane_bytes + k0) =
                    make_char4((signed char)-vi[0], (signed char)-vi[1], (signed char)-vi[2], (signed char)-vi[3]);
            }
        }
    }
}

// ---- 2. slice products ----------------------------------------------------------------

// Shared-memory matrix descriptor: K-major, 64-byte swizzle (layout type 4),
// 8-row groups 8 x 64 = 512 bytes apart (SBO), leading offset unused (1),
// descriptor version 1.  Each plane tile starts on a 1024-byte boundary; the
// second 32-byte K step of a row advances the start address by 32 bytes.
__device__ __forceinline__ uint64_t oz_desc(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)((8 * OZ_BK) >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)4 << 61;
    return d;
}

__device__ __forceinline__ void umma_i8_pair(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                             uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, {%5, %5, %5, %5, %5, %5, %5, %5}, p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(0u)
        : "memory");
}

// Warp-wide 32 lanes x 16 consecutive 32-bit TMEM columns, two blocks, one wait.
__device__ __forceinline__ void tmem_ld16x2_s32(uint32_t ta, uint32_t tb, int* va, int* vb)
{
    float fa[16], fb[16];
    tmem_ld16x2(ta, tb, fa, fb);
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        va[i] = __float_as_int(fa[i]);
        vb[i] = __float_as_int(fb[i]);
    }
}

__device__ __forceinline__ int diag_lo(int d) { return d - kOzS > 1 ? d - kOzS : 1; }
__device__ __forceinline__ int diag_hi(int d) { return d - 1 < kOzS ? d - 1 : kOzS; }

template <int TN>
__global__ void __launch_bounds__(kOzThreads, 1)
    ozaki_pair_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                      const OzParams p)
{
    using G = OzGeom<TN>;
    constexpr int OZ_STAGES = G::STAGES;
    constexpr int OZ_STAGE = G::STAGE;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* ring = align_shared<1024>(smem_raw);
    uint64_t* full = reinterpret_cast<uint64_t*>(ring + OZ_STAGES * OZ_STAGE);
    uint64_t* empty = full + OZ_STAGES;
    uint64_t* acc_full = empty + OZ_STAGES;  // MMA -> epilogue: the diagonal's sums are in TMEM
    uint64_t* acc_free = acc_full + 1;       // epilogue -> MMA (even CTA): TMEM drained
    uint64_t* mma_done = acc_free + 1;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_done + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    __shared__ uint32_t flagged_here;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const uint32_t rank = cluster_ctarank() & 1u;
    const bool leader = rank == 0;
    const uint16_t pair_mask = 0x3u;
    // Pair tiles in groups of 8 tile rows, rows fastest: the ~74 tiles in
    // flight share a few A and B panels and walk K in step, so the slices they
    // stream come from L2.
    constexpr int GM = 8;
    const int pid = blockIdx.x >> 1;
    const int in_group = GM * p.tiles_n;
    const int first_m = (pid / in_group) * GM;
    const int gsz = min(p.tiles_m - first_m, GM);
    const int tm = first_m + (pid % in_group) % gsz;
    const int tn = (pid % in_group) / gsz;
    const int m0 = tm * OZ_TILE_M + (int)rank * OZ_ROWS;  // this CTA's rows
    const int n0 = tn * TN;                               // the pair's columns
    const int n = p.n;

    // A tile runs here only when one of its 16 x 16 count tiles is dense; both
    // CTAs of the pair read the same counts and leave together, before any
    // barrier or TMEM is touched.
    uint32_t here = 0;
    bool dense = false;
    if (tid == 0) {
        flagged_here = 0;
    }
    {
        const int g16 = (n + 15) / 16;
        if (tid < 16 * G::GRAN_N) {
            const int gi = tm * 16 + tid % 16;
            const int gj = tn * G::GRAN_N + tid / 16;
            if (gi < g16 && gj < g16) {
                const uint32_t c = p.tile_count[(size_t)gj * g16 + gi];
                dense = c > kSparseMax;
                if (gi * 16 >= m0 && gi * 16 < m0 + OZ_ROWS) {
                    here = c;  // flagged outputs in this CTA's 128 rows
                }
            }
        }
    }
    if (!__syncthreads_or(dense)) {
        return;
    }
    if (here != 0) {
        atomicAdd(&flagged_here, here);
    }
    __syncthreads();
    if (tid == 0) {
        if (flagged_here != 0) {
            atomicAdd(&p.stats[kStatDenseOutputs], flagged_here);
        }
        if (leader) {
            atomicAdd(&p.stats[kStatExactTiles], 1u);
            // output positions of the tile inside the matrix (the roofline's work)
            const int rows = min(OZ_TILE_M, n - tm * OZ_TILE_M), cols = min(TN, n - n0);
            atomicAdd(&p.stats[kStatExactOutputs], (uint32_t)(rows * cols));
        }
        for (int s = 0; s < OZ_STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(acc_full, 1);
        mbar_init(acc_free, 2 * kOzEpiWarps);
        mbar_init(mma_done, 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 1) {
        tmem_alloc_pair(tmem_slot, 512);
        tmem_relinquish_pair();
    }
    tc_fence_before();
    cluster_sync();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        // ---------------- TMA producer (both CTAs) ----------------
        if (lane == 0) {
            tma_prefetch_desc(&tmA);
            tma_prefetch_desc(&tmB);
            int it = 0;
            bool stop = false;
            for (int d = 2; d <= kOzLastDiag && !stop; ++d) {
                for (int kb = 0; kb < p.kblocks && !stop; ++kb) {
                    for (int s = diag_lo(d); s <= diag_hi(d); ++s, ++it) {
                        const int slot = it % OZ_STAGES;
                        if ((it >= OZ_STAGES && !mbar_wait(&empty[slot], ((it / OZ_STAGES) - 1) & 1, p.status)) ||
                            *abort_flag) {
                            *abort_flag = 1;
                            stop = true;
                            break;
                        }
                        uint8_t* st = ring + slot * OZ_STAGE;
                        const uint32_t bar = mapa_shared(smem_u32(&full[slot]), 0);
                        if (leader) {
                            mbar_arrive_expect_tx(&full[slot], 2 * OZ_STAGE);
                        }
                        const int t = d - s;
                        tma_load_3d_pair(st, &tmA, bar, kb * OZ_BK, m0, 2 * (s - 1));
                        tma_load_3d_pair(st + 2 * OZ_PLANE, &tmB, bar, kb * OZ_BK, n0 + (int)rank * G::BCOLS,
                                         3 * (t - 1));
                    }
                }
            }
            if (leader) {
                for (int j = it > OZ_STAGES ? it - OZ_STAGES : 0; j < it; ++j) {
                    mbar_wait(&full[j % OZ_STAGES], (j / OZ_STAGES) & 1, p.status);
                }
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer (even CTA) ----------------
        if (leader && lane == 0) {
            // S32 accumulate, signed 8-bit A and B, both K-major, N = 256, M = 256.
            const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) |
                                   ((uint32_t)(OZ_TILE_M >> 4) << 24);
            const uint32_t d_re = tmem, d_im = tmem + (uint32_t)TN;
            int it = 0;
            bool stop = false;
            for (int d = 2; d <= kOzLastDiag && !stop; ++d) {
                if (d > 2) {
                    if (!mbar_wait_cluster(acc_free, (d - 3) & 1, p.status)) {
                        *abort_flag = 1;
                        break;
                    }
                    tc_fence_after();
                }
                bool first = true;
                for (int kb = 0; kb < p.kblocks && !stop; ++kb) {
                    for (int s = diag_lo(d); s <= diag_hi(d); ++s, ++it) {
                        const int slot = it % OZ_STAGES;
                        if (!mbar_wait(&full[slot], (it / OZ_STAGES) & 1, p.status)) {
                            *abort_flag = 1;
                            stop = true;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t ar = smem_u32(ring + slot * OZ_STAGE);
                        const uint32_t ai = ar + OZ_PLANE, br = ar + 2 * OZ_PLANE, bi = br + G::B_PLANE,
                                       nbi = br + 2 * G::B_PLANE;
#pragma unroll
                        for (int kk = 0; kk < OZ_BK / 32; ++kk) {
                            const uint32_t o = (uint32_t)(kk * 32);
                            const uint32_t acc = (first && kk == 0) ? 0u : 1u;
                            umma_i8_pair(d_re, oz_desc(ar + o), oz_desc(br + o), idesc, acc);
                            umma_i8_pair(d_re, oz_desc(ai + o), oz_desc(nbi + o), idesc, 1u);
                            umma_i8_pair(d_im, oz_desc(ar + o), oz_desc(bi + o), idesc, acc);
                            umma_i8_pair(d_im, oz_desc(ai + o), oz_desc(br + o), idesc, 1u);
                        }
                        first = false;
                        umma_commit_pair(&empty[slot], pair_mask);
                    }
                }
                if (!stop) {
                    umma_commit_pair(acc_full, pair_mask);
                }
            }
            umma_commit_pair(mma_done, pair_mask);
            mbar_wait(mma_done, 0, p.status);  // nothing may still write TMEM when it is freed
        }
    } else {
        // ---------------- epilogue warps 2..9 (both CTAs) ----------------
        // TMEM lane quadrant = warp % 4 (the warp's 32 rows); warps 2-5 take
        // the first TN / 2 columns of the tile, warps 6-9 the rest.
        const int quad = warp & 3;
        const int half = (warp - 2) >> 2;
        const int row = m0 + quad * 32 + lane;
        const uint32_t lane_addr = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(half * G::BCOLS);
        const uint32_t free_addr = mapa_shared(smem_u32(acc_free), 0);
        const int ei = row < n ? p.E[row] : 0;
        uint32_t fallbacks = 0;
        for (int d = 2; d <= kOzLastDiag; ++d) {
            const bool ready = mbar_wait(acc_full, (d - 2) & 1, p.status);
            tc_fence_after();
            if (!__all_sync(0xffffffffu, ready && !*abort_flag)) {
                break;
            }
            const double w = ldexp(1.0, -7 * d);
#pragma unroll 1
            for (int cb = 0; cb < G::BCOLS; cb += 16) {
                int vr[16], vi[16];
                tmem_ld16x2_s32(lane_addr + (uint32_t)cb, lane_addr + (uint32_t)(TN + cb), vr, vi);
                if (row >= n) {
                    continue;
                }
                // The chunk's 16 partial sums are loaded before any is used
                // (independent loads in flight together): the MMAs wait for
                // this drain, so its memory latency must overlap.
                double2 prev[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int col = n0 + half * G::BCOLS + cb + j;
                    prev[j] = (d == 2 || col >= n) ? make_double2(0.0, 0.0)
                                                   : __ldcg(&p.partial[(size_t)col * n + row]);
                }
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int col = n0 + half * G::BCOLS + cb + j;
                    if (col >= n) {
                        break;
                    }
                    const size_t idx = (size_t)col * n + row;
                    double2 v = prev[j];
                    v.x = fma((double)vr[j], w, v.x);
                    v.y = fma((double)vi[j], w, v.y);
                    if (d < kOzLastDiag) {
                        __stcg(&p.partial[idx], v);
                        continue;
                    }
                    if (!flag_at(p.flag_bits, idx)) {
                        continue;  // not flagged: the GEMM's value stands
                    }
                    const int fj = p.F[col];
                    bool ok = ei != kOzNonFinite && fj != kOzNonFinite;
                    float2 out = make_float2(0.0f, 0.0f);
                    if (ok && ei != kOzZero && fj != kOzZero) {
                        const int sh = ei + fj;
                        const double zr = ldexp(v.x, sh), zi = ldexp(v.y, sh);
                        const double lim = ldexp(p.thresh, sh);
                        ok = fabs(zr) >= lim && fabs(zi) >= lim;
                        out = make_float2((float)zr, (float)zi);
                    }
                    if (ok) {
                        p.C[idx] = out;
                    } else {
                        atomicOr(&p.fallback_bits[idx >> 5], 1u << (idx & 31));
                        ++fallbacks;
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive_cluster(free_addr);
            }
        }
        fallbacks = __reduce_add_sync(0xffffffffu, fallbacks);
        if (lane == 0 && fallbacks != 0) {
            atomicAdd(&p.stats[kStatFallback], fallbacks);
        }
    }
    tc_fence_before();
    __syncthreads();
    cluster_sync();  // the even CTA's MMAs are complete; neither CTA's memory is used any more
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc_pair(tmem, 512);
    }
}

}  // namespace

OzLayout oz_layout(int n, uint8_t* base, std::vector<size_t>* guards)
{
    OzLayout L;
    L.kpitch = (n + 63) / 64 * 64;
    L.plane_bytes = (size_t)n * L.kpitch;
    size_t off = 0;
    const size_t e_off = off;
    off = next_region(off, (size_t)n * 4, guards);
    const size_t f_off = off;
    off = next_region(off, (size_t)n * 4, guards);
    const size_t a_off = off;
    off = next_region(off, 2 * kOzS * L.plane_bytes, guards);
    const size_t b_off = off;
    off = next_region(off, 3 * kOzS * L.plane_bytes, guards);
    const size_t p_off = off;
    off = next_region(off, (size_t)n * n * sizeof(double2), guards);
    L.bytes = off;
    if (base != nullptr) {
        L.E = reinterpret_cast<int*>(base + e_off);
        L.F = reinterpret_cast<int*>(base + f_off);
        L.planes_a = reinterpret_cast<int8_t*>(base + a_off);
        L.planes_b = reinterpret_cast<int8_t*>(base + b_off);
        L.partial = reinterpret_cast<double2*>(base + p_off);
    }
    return L;
}

// Tile width of the exact recompute.  256 x 192 tiles fill the waves of 74
// clusters better at n = 4096 (4.76 waves instead of 3.46) but measured no
// faster (7.15 against 7.03 ms: the narrower MMA and the partial last column
// cost what the fuller waves save), so every order uses 256 x 256.
int ozaki_tile_n(int n)
{
    (void)n;
    return 256;
}

template <int TN>
static cudaError_t launch_pair_tn(cudaStream_t s, int n, const OzLayout& L, OzParams p)
{
    using G = OzGeom<TN>;
    CUtensorMap ta, tb;
    const uint64_t dims_a[3] = {(uint64_t)n, (uint64_t)n, (uint64_t)(2 * kOzS)};
    const uint64_t dims_b[3] = {(uint64_t)n, (uint64_t)n, (uint64_t)(3 * kOzS)};
    const uint64_t strides[2] = {(uint64_t)L.kpitch, (uint64_t)L.plane_bytes};
    const uint32_t box_a[3] = {(uint32_t)OZ_BK, (uint32_t)OZ_ROWS, 2u};
    const uint32_t box_b[3] = {(uint32_t)OZ_BK, (uint32_t)G::BCOLS, 3u};
    if (!encode_tensor_map(&ta, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, dims_a, strides, box_a, CU_TENSOR_MAP_SWIZZLE_64B,
                           L.planes_a) ||
        !encode_tensor_map(&tb, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, dims_b, strides, box_b, CU_TENSOR_MAP_SWIZZLE_64B,
                           L.planes_b)) {
        return cudaErrorInvalidValue;
    }
    p.tiles_m = (n + OZ_TILE_M - 1) / OZ_TILE_M;
    p.tiles_n = (n + TN - 1) / TN;
    auto kernel = ozaki_pair_kernel<TN>;
    cudaError_t err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::SMEM);
    if (err != cudaSuccess) {
        return err;
    }
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)(2 * p.tiles_m * p.tiles_n));
    cfg.blockDim = dim3(kOzThreads);
    cfg.dynamicSmemBytes = G::SMEM;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    err = cudaLaunchKernelEx(&cfg, kernel, ta, tb, p);
    return err != cudaSuccess ? err : cudaGetLastError();
}

cudaError_t launch_ozaki(cudaStream_t s, int n, int pitch, const float2* rows_a, const float2* rows_b,
                         const OzLayout& L, const uint32_t* flag_bits, const uint32_t* tile_count, uint32_t* stats,
                         uint32_t* fallback_bits, float2* C, int* status, int* launched,
                         const std::function<void(int)>& mark)
{
    int count = 0;
    ozaki_split_kernel<<<2 * n, 256, 0, s>>>(n, pitch, rows_a, rows_b, L.planes_a, L.planes_b, L.kpitch,
                                              L.plane_bytes, L.E, L.F);
    cudaError_t err = cudaGetLastError();
    mark(++count);
    if (err == cudaSuccess) {
        OzParams p{};
        p.n = n;
        p.kblocks = (n + OZ_BK - 1) / OZ_BK;
        p.E = L.E;
        p.F = L.F;
        p.flag_bits = flag_bits;
        p.tile_count = tile_count;
        p.stats = stats;
        p.fallback_bits = fallback_bits;
        p.partial = L.partial;
        p.C = C;
        p.thresh = ldexp(1.0 + ldexp(1.0, -20), 25) * (2.0 * n * (kOzS + 1)) * ldexp(1.0, -7 * kOzS);
        p.status = status;
        err = launch_pair_tn<256>(s, n, L, p);
        mark(++count);
    }
    if (launched != nullptr) {
        *launched = count;
    }
    return err;
}

}  // namespace cg3m
