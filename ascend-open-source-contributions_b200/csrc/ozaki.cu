// ozaki.cu -- FP64-accurate recompute of the flagged outputs of dense tiles on
// the tensor cores: the rounding-correction pass of the tensor-core forms.
//
// The reference recomputes flagged outputs with its segmented FP32 replay
// (cgemm3m_rounding_kernel.cpp:192-404); the tensor-core forms of this library
// promise instead that every flagged output is within one FP32 rounding of the
// exact product.  Recomputing ~3/4 of a 4096^3 product in FP64 on the CUDA
// cores takes ~24 ms at this GPU's FP64 rate, so the products run on the int8
// tensor cores as exact integer products modulo small coprime moduli, put
// back together by the Chinese remainder theorem (the modular form of the
// Ozaki scheme: Ozaki, Uchino and Imamura, "Ozaki Scheme II: A GEMM-oriented
// emulation of floating-point matrix multiplication using an integer modular
// technique", 2025):
//
//   1. ozaki_split_kernel: every op(A) row i and op(B) column j gets a power
//      of two 2^E > max |x| over the row (real and imaginary parts together);
//      each part becomes the integer a = rn(x 2^(beta - E)), |a| <= 2^beta,
//      beta = 47, and the row counts its parts for which a != x 2^(beta - E)
//      (cA_i; cB_j for the columns).  The planes hold a mod p_m for the
//      kOzMods = 14 moduli p_m <= 256 (pairwise coprime, product M ~ 2^110.2)
//      as int8 in [-(p-1)/2, (p-1)/2] ([-128, 127] for 256).
//   2. ozaki_pair_kernel: for each modulus the int8 products
//        Re_m = sum Ar Br + Ai (-Bi),  Im_m = sum Ar Bi + Ai Br
//      are exact in the int32 TMEM accumulators (|sum| <= 2 * 4096 * 128^2
//      < 2^31); the epilogue stores y_m = sum mod p_m in [0, p_m) as one byte
//      per output and part: y_m = x mod p_m, x the exact integer product of
//      the rounded parts.
//   3. ozaki_crt_kernel: x = sum_m y_m w_m - k M with w_m = u_m (M / p_m)
//      mod M, u_m = (M / p_m)^-1 mod p_m (so w_m = 1 mod p_m, 0 mod the other
//      moduli), and k the nearest integer to sum_m y_m w_m / M (from the
//      exact limb sums)
//      (|x| <= 2 n 2^(2 beta) <= 2^107 < M / 8, so k is never in doubt),
//      evaluated exactly in three 40-bit limbs of FP64.  The factor u_m lives
//      in the constants w_m, so the residue kernel does no multiplication.  Rounding a part moves each real product by at most 2^(beta - 1),
//      so
//        |error| <= (cA_i + cB_j) 2^(beta - 1)   (units of 2^(E_i + F_j - 2 beta)),
//      zero for rows and columns that scaled exactly.  Every output of a tile
//      that ran is written (flagged or not: the form's own products skip
//      these tiles) when the bound is zero or both parts exceed 2^25 times it
//      (so the result, rounded to FP32, is within one FP32 rounding of the
//      exact product); otherwise it is marked for the FP64 per-output kernel,
//      as are outputs whose row or column holds a non-finite value.
//
// B200 design: a cluster of two CTAs per 256 x 256 output tile
// (tcgen05.mma.cta_group::2.kind::i8, M = 256, N = 256, K = 32): CTA r stages
// rows [128r, 128r + 128) of the op(A) residues and columns [128r, 128r + 128)
// of the op(B) residues, 64-byte K rows with the 64-byte swizzle, 40 KB per
// stage (Ar, Ai | Br, Bi, -Bi) in a 5-stage ring; each CTA's TMEM holds its
// 128 rows x 256 columns of Re (columns 0..255) and Im (256..511).  Warp 0 of
// both CTAs issues the TMA copies (completion on the even CTA's barrier), one
// thread of the even CTA issues every MMA, warps 2..9 of both CTAs drain the
// accumulators after each modulus.  Every wait is bounded.
#include "cg3m_internal.h"
#include "ptx.cuh"

namespace cg3m {

namespace {

constexpr int kOzMods = 14;                    // moduli (planes per operand part)
constexpr int kOzBeta = 47;                    // bits of the scaled integer parts
constexpr int kOzMaxN = 4096;                  // 2 n 2^(2 beta) <= M / 8 up to this order
constexpr int OZ_TILE_M = kOzakiTile;          // output rows of a pair tile (M of the pair MMA)
constexpr int OZ_TN = kOzakiTile;              // output columns of a pair tile (N of the pair MMA)
constexpr int OZ_ROWS = 128;                   // A rows staged by one CTA
constexpr int OZ_BCOLS = OZ_TN / 2;            // B columns staged by one CTA
constexpr int OZ_BK = 64;                      // K bytes per staged row (64-byte swizzle)
constexpr int OZ_PLANE = OZ_ROWS * OZ_BK;      // 8 KB
constexpr int OZ_B_PLANE = OZ_BCOLS * OZ_BK;   // 8 KB
constexpr int OZ_STAGE = 2 * OZ_PLANE + 3 * OZ_B_PLANE;
constexpr int OZ_STAGES = (208 * 1024) / OZ_STAGE;
constexpr size_t OZ_SMEM = (size_t)OZ_STAGES * OZ_STAGE + 1024 + 256;
constexpr int OZ_GRAN_N = OZ_TN / 16;          // 16 x 16 count tiles across the pair tile
constexpr int kOzEpiWarps = 8;
constexpr int kOzThreads = (2 + kOzEpiWarps) * 32;
constexpr int kOzNonFinite = 1 << 20;          // exponent marker: the row or column holds Inf/NaN
constexpr int kOzZero = -(1 << 20);            // exponent marker: the row or column is all zero
constexpr double kMagic = 6755399441055744.0;  // 1.5 * 2^52: x + kMagic rounds x to an integer
constexpr float kMagicF = 12582912.0f;         // 1.5 * 2^23
static_assert(OZ_STAGE % 1024 == 0 && OZ_B_PLANE % 1024 == 0, "plane tiles start on 1024-byte boundaries");
static_assert(kOzThreads >= 16 * OZ_GRAN_N, "one thread per count tile in the density check");
static_assert(OZ_BCOLS % 16 == 0, "epilogue chunks of 16 columns");

// Moduli, largest first: 256 and 13 odd numbers, pairwise coprime
// (255 = 3 5 17, 253 = 11 23, 247 = 13 19, 217 = 7 31, the rest prime).
constexpr int kOzModuli[kOzMods] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199};

// Constants of the moduli (host-computed once, passed by value).
struct OzCrt {
    int p[kOzMods];
    int c16[kOzMods];        // 2^16 mod p
    float pf[kOzMods];
    float inv_pf[kOzMods];   // rn(1 / p)
    double pd[kOzMods];
    double inv_pd[kOzMods];  // rn(1 / p)
    double w[kOzMods][3];    // w = u (M / p) mod M, u = (M / p)^-1 mod p, in 40-bit limbs, low first
    double m[3];             // M in 40-bit limbs, low first
    double k2, k1;           // rn(2^80 / M), rn(2^40 / M): k from the limb sums
};

struct OzParams {
    int n;
    int kblocks;             // 64-byte K blocks
    int tiles_m, tiles_n;    // pair tiles along the rows and the columns
    const uint32_t* tile_count;
    uint32_t* stats;
    uint8_t* tile_ran;       // per pair tile (tn * tiles_m + tm): 1 when it ran here
    uint8_t* residues;       // [2 * kOzMods][y_pad / 16][y_pad][16]
    int y_pad;
    size_t y_plane;
    OzCrt crt;
    int* status;
};

struct OzFinish {
    int n;
    int tiles_m;
    const int* E;            // op(A) row exponents
    const int* F;            // op(B) column exponents
    const int* CA;           // rounded parts per op(A) row
    const int* CB;           // rounded parts per op(B) column
    const uint8_t* tile_ran;
    const uint8_t* residues;
    int y_pad;
    size_t y_plane;
    uint32_t* stats;
    uint32_t* fallback_bits;
    float2* C;
    OzCrt crt;
};

// t mod p in [-(p-1)/2, (p-1)/2] for odd p and an integer-valued t, |t| <= 2^47,
// given tm = t + 1.5 * 2^52 (exact): the nearest integer q to t * rn(1/p) is
// the nearest integer to t / p (their distance, <= 2^-13.6, is below that of
// t / p to a half-integer, >= 1 / 2p), and tm - q p = 1.5 * 2^52 + (t - q p)
// is exact, its low word the residue.
__device__ __forceinline__ int mod_odd_d(double t, double tm, double pd, double inv_pd)
{
    const double q = __dsub_rn(__fma_rn(t, inv_pd, kMagic), kMagic);
    return __double2loint(__fma_rn(-q, pd, tm));
}

// ---- 1. residues -------------------------------------------------------------------

// One block per op(A) row (blockIdx.x < n) or op(B) column.  Plane layout:
// [plane][row][kpitch] int8, A planes 2m + {0 re, 1 im}, B planes
// 3m + {0 re, 1 im, 2 -im}.
__global__ void __launch_bounds__(256, 4)
    ozaki_split_kernel(int n, int pitch, const float2* __restrict__ rows_a, const float2* __restrict__ rows_b,
                       int8_t* __restrict__ pa, int8_t* __restrict__ pb, int kpitch, size_t plane_bytes,
                       int* __restrict__ E, int* __restrict__ F, int* __restrict__ CA, int* __restrict__ CB,
                       const __grid_constant__ OzCrt crt)
{
    __shared__ float wmax[8];
    __shared__ int wbad[8];
    __shared__ int wcnt[8];
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
    // 2^(e-1) <= amax < 2^e, so every part scaled by 2^(beta - e) lies in (-2^beta, 2^beta).
    const int e = any_bad ? kOzNonFinite : amax > 0.0f ? ilogbf(amax) + 1 : kOzZero;
    const bool usable = !any_bad && amax > 0.0f;
    const double scale = usable ? ldexp(1.0, kOzBeta - e) : 0.0;
    int8_t* dst = (is_a ? pa : pb) + (size_t)row * kpitch;
    const int planes_per_mod = is_a ? 2 : 3;
    int rounded = 0;
    // Four consecutive K terms per thread: 4-byte stores into every plane.
#pragma unroll 1
    for (int k0 = tid * 4; k0 < n; k0 += 256 * 4) {
        // The real parts, then the imaginary parts, of four consecutive terms.
#pragma unroll 1
        for (int part = 0; part < 2; ++part) {
            double t[4], tm[4];  // tm = t + 1.5 * 2^52
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int k = k0 + u;
                const float2 x = (k < n && usable) ? src[k] : make_float2(0.0f, 0.0f);
                const double sx = __dmul_rn((double)(part == 0 ? x.x : x.y), scale);  // exact: a power of two
                tm[u] = __dadd_rn(sx, kMagic);    // rounds to an integer: |sx| < 2^51
                t[u] = __dsub_rn(tm[u], kMagic);  // nearest integer, |t| <= 2^beta
                rounded += t[u] != sx;
            }
#pragma unroll
            for (int mi = 0; mi < kOzMods; ++mi) {
                int v[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (mi == 0) {
                        // mod 256: the low byte of the two's complement integer
                        v[q] = (int)(signed char)(__double2loint(tm[q]) & 0xFF);
                    } else {
                        v[q] = mod_odd_d(t[q], tm[q], crt.pd[mi], crt.inv_pd[mi]);
                    }
                }
                int8_t* plane = dst + (size_t)(planes_per_mod * mi + part) * plane_bytes;
                // K beyond n is never read (the tensor maps stop at n), so whole
                // 4-byte groups may be stored while k0 < n <= kpitch.
                *reinterpret_cast<char4*>(plane + k0) =
                    make_char4((signed char)v[0], (signed char)v[1], (signed char)v[2], (signed char)v[3]);
                if (!is_a && part == 1) {
                    // -(-128) wraps to -128: the same residue mod 256
                    *reinterpret_cast<char4*>(plane + plane_bytes + k0) =
                        make_char4((signed char)-v[0], (signed char)-v[1], (signed char)-v[2], (signed char)-v[3]);
                }
            }
        }
    }
    rounded = __reduce_add_sync(0xffffffffu, rounded);
    if ((tid & 31) == 0) {
        wcnt[tid >> 5] = rounded;
    }
    __syncthreads();
    if (tid == 0) {
        int total = 0;
        for (int w = 0; w < 8; ++w) {
            total += wcnt[w];
        }
        (is_a ? E : F)[row] = e;
        (is_a ? CA : CB)[row] = total;
    }
}

// ---- 2. residue products --------------------------------------------------------------

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

// x mod p in [0, p) for odd p and |x| < 2^27: t = (x >> 16) c16 + (x & 0xFFFF)
// is congruent to x with |t| < 2^20, exact in FP32, and t * rn(1/p) is off
// t / p by < 2^-12 (the distance of t / p to a half-integer is >= 1 / 2p).
__device__ __forceinline__ uint32_t residue_byte(int x, int c16, float pf, float inv_pf)
{
    const int t = (x >> 16) * c16 + (x & 0xFFFF);
    const float tf = __fsub_rn(__int_as_float(0x4B400000 + t), kMagicF);
    const float q = __fsub_rn(__fmaf_rn(tf, inv_pf, kMagicF), kMagicF);
    float r = __fmaf_rn(-q, pf, tf);
    r = r < 0.0f ? __fadd_rn(r, pf) : r;
    return (uint32_t)__float_as_int(__fadd_rn(r, kMagicF)) & 0xFFu;
}

// 16 accumulator values (int32 bits) -> 16 residue bytes; x mod 256 is the low byte.
__device__ __forceinline__ uint4 residue_bytes16(const float* v, bool pow2, int c16, float pf, float inv_pf)
{
    uint32_t w[4];
#pragma unroll
    for (int g = 0; g < 4; ++g) {
        uint32_t word = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int x = __float_as_int(v[4 * g + b]);
            const uint32_t y = pow2 ? ((uint32_t)x & 0xFFu) : residue_byte(x, c16, pf, inv_pf);
            word |= y << (8 * b);
        }
        w[g] = word;
    }
    return make_uint4(w[0], w[1], w[2], w[3]);
}

__global__ void __launch_bounds__(kOzThreads, 1)
    ozaki_pair_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                      const __grid_constant__ OzParams p)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t* ring = align_shared<1024>(smem_raw);
    uint64_t* full = reinterpret_cast<uint64_t*>(ring + OZ_STAGES * OZ_STAGE);
    uint64_t* empty = full + OZ_STAGES;
    uint64_t* acc_full = empty + OZ_STAGES;  // MMA -> epilogue: the modulus's sums are in TMEM
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
    // flight share a few A and B panels and walk K in step, so the residues
    // they stream come from L2.
    constexpr int GM = 8;
    const int pid = blockIdx.x >> 1;
    const int in_group = GM * p.tiles_n;
    const int first_m = (pid / in_group) * GM;
    const int gsz = min(p.tiles_m - first_m, GM);
    const int tm = first_m + (pid % in_group) % gsz;
    const int tn = (pid % in_group) / gsz;
    const int m0 = tm * OZ_TILE_M + (int)rank * OZ_ROWS;  // this CTA's rows
    const int n0 = tn * OZ_TN;                            // the pair's columns
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
        if (tid < 16 * OZ_GRAN_N) {
            const int gi = tm * 16 + tid % 16;
            const int gj = tn * OZ_GRAN_N + tid / 16;
            if (gi < g16 && gj < g16) {
                const uint32_t c = p.tile_count[(size_t)gj * g16 + gi];
                dense = c > kSparseMax;
                if (gi * 16 >= m0 && gi * 16 < m0 + OZ_ROWS) {
                    here = c;  // flagged outputs in this CTA's 128 rows
                }
            }
        }
    }
    const bool run = __syncthreads_or(dense);
    if (tid == 0 && leader) {
        p.tile_ran[(size_t)tn * p.tiles_m + tm] = run ? 1 : 0;  // read by the reconstruction
    }
    if (!run) {
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
            const int rows = min(OZ_TILE_M, n - tm * OZ_TILE_M), cols = min(OZ_TN, n - n0);
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
            for (int mi = 0; mi < kOzMods && !stop; ++mi) {
                for (int kb = 0; kb < p.kblocks; ++kb, ++it) {
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
                    tma_load_3d_pair(st, &tmA, bar, kb * OZ_BK, m0, 2 * mi);
                    tma_load_3d_pair(st + 2 * OZ_PLANE, &tmB, bar, kb * OZ_BK, n0 + (int)rank * OZ_BCOLS, 3 * mi);
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
            const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(OZ_TN >> 3) << 17) |
                                   ((uint32_t)(OZ_TILE_M >> 4) << 24);
            const uint32_t d_re = tmem, d_im = tmem + (uint32_t)OZ_TN;
            int it = 0;
            bool stop = false;
            for (int mi = 0; mi < kOzMods && !stop; ++mi) {
                if (mi > 0) {
                    if (!mbar_wait_cluster(acc_free, (mi - 1) & 1, p.status)) {
                        *abort_flag = 1;
                        break;
                    }
                    tc_fence_after();
                }
                for (int kb = 0; kb < p.kblocks; ++kb, ++it) {
                    const int slot = it % OZ_STAGES;
                    if (!mbar_wait(&full[slot], (it / OZ_STAGES) & 1, p.status)) {
                        *abort_flag = 1;
                        stop = true;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t ar = smem_u32(ring + slot * OZ_STAGE);
                    const uint32_t ai = ar + OZ_PLANE, br = ar + 2 * OZ_PLANE, bi = br + OZ_B_PLANE,
                                   nbi = br + 2 * OZ_B_PLANE;
#pragma unroll
                    for (int kk = 0; kk < OZ_BK / 32; ++kk) {
                        const uint32_t o = (uint32_t)(kk * 32);
                        const uint32_t acc = (kb == 0 && kk == 0) ? 0u : 1u;
                        umma_i8_pair(d_re, oz_desc(ar + o), oz_desc(br + o), idesc, acc);
                        umma_i8_pair(d_re, oz_desc(ai + o), oz_desc(nbi + o), idesc, 1u);
                        umma_i8_pair(d_im, oz_desc(ar + o), oz_desc(bi + o), idesc, acc);
                        umma_i8_pair(d_im, oz_desc(ai + o), oz_desc(br + o), idesc, 1u);
                    }
                    umma_commit_pair(&empty[slot], pair_mask);
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
        // the first 128 columns of the tile, warps 6-9 the rest.  Every row
        // and column of the tile lies inside the padded residue planes, so
        // the stores need no bounds (rows and columns past n hold zeros).
        const int quad = warp & 3;
        const int half = (warp - 2) >> 2;
        const int row = m0 + quad * 32 + lane;
        const uint32_t lane_addr = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(half * OZ_BCOLS);
        const uint32_t free_addr = mapa_shared(smem_u32(acc_free), 0);
        const size_t strip = (size_t)p.y_pad * 16;  // bytes of one 16-column strip of a plane
        uint8_t* const out0 = p.residues + (size_t)((n0 + half * OZ_BCOLS) >> 4) * strip + (size_t)row * 16;
        for (int mi = 0; mi < kOzMods; ++mi) {
            const bool ready = mbar_wait(acc_full, mi & 1, p.status);
            tc_fence_after();
            if (!__all_sync(0xffffffffu, ready && !*abort_flag)) {
                break;
            }
            const bool pow2 = mi == 0;
            const int c16 = p.crt.c16[mi];
            const float pf = p.crt.pf[mi], inv_pf = p.crt.inv_pf[mi];
            uint8_t* const re_out = out0 + (size_t)(2 * mi) * p.y_plane;
            uint8_t* const im_out = re_out + p.y_plane;
#pragma unroll 1
            for (int cb = 0; cb < OZ_BCOLS; cb += 16) {
                float vr[16], vi[16];
                tmem_ld16x2(lane_addr + (uint32_t)cb, lane_addr + (uint32_t)(OZ_TN + cb), vr, vi);
                const size_t o = (size_t)(cb >> 4) * strip;
                __stcg(reinterpret_cast<uint4*>(re_out + o), residue_bytes16(vr, pow2, c16, pf, inv_pf));
                __stcg(reinterpret_cast<uint4*>(im_out + o), residue_bytes16(vi, pow2, c16, pf, inv_pf));
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive_cluster(free_addr);
            }
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

// ---- 3. reconstruction ---------------------------------------------------------------

// 2^e as a double for -1022 <= e <= 1023.
__device__ __forceinline__ double pow2d(int e)
{
    return __hiloint2double((e + 1023) << 20, 0);
}

// The exact integer products of one part for outputs c0 and c0 + 1 of the
// four whose residue bytes the words hold (word mi: byte c for modulus mi).
__device__ __forceinline__ void crt_part2(const OzCrt& crt, const uint32_t* words, int c0, double* x)
{
    double s[2][3];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        s[c][0] = s[c][1] = s[c][2] = 0.0;
    }
#pragma unroll
    for (int mi = 0; mi < kOzMods; ++mi) {
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            // byte c0 + c of the word as the low byte of 2^52 + y
            const int lo = (int)__byte_perm(words[mi], 0u, 0x4440u + (unsigned)(c0 + c));
            const double yd = __dsub_rn(__hiloint2double(0x43300000, lo), 4503599627370496.0);  // exact
            // every product and partial sum stays below 2^52: exact
            s[c][0] = __fma_rn(yd, crt.w[mi][0], s[c][0]);
            s[c][1] = __fma_rn(yd, crt.w[mi][1], s[c][1]);
            s[c][2] = __fma_rn(yd, crt.w[mi][2], s[c][2]);
        }
    }
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        // S / M = k + x / M with |x / M| < 1/8, S = (s2 2^40 + s1) 2^40 + s0;
        // s2 rn(2^80 / M) + s1 rn(2^40 / M) is off S / M by < 2^-40 (S / M < 3570)
        const double k = rint(__fma_rn(s[c][2], crt.k2, __dmul_rn(s[c][1], crt.k1)));
        const double d0 = __fma_rn(-k, crt.m[0], s[c][0]);  // exact integers below 2^53
        const double d1 = __fma_rn(-k, crt.m[1], s[c][1]);
        const double d2 = __fma_rn(-k, crt.m[2], s[c][2]);
        // x = (d2 2^40 + d1) 2^40 + d0: two roundings, relative error < 2^-52
        x[c0 + c] = __fma_rn(__fma_rn(d2, 1099511627776.0, d1), 1099511627776.0, d0);
    }
}

// One thread per op(A) row and two consecutive op(B) columns; a block holds 32
// rows x 16 columns inside one exact tile, and a warp (4 rows x 8 column
// pairs) reads 64 consecutive residue bytes per plane and writes whole 32-byte
// sectors of C.  Two outputs per thread keep it near 64 registers, for twice
// the resident warps of four.  Writes every output of the tile whose bound
// certifies it and marks the rest in fallback_bits.
constexpr int kCrtRows = 32;

__global__ void __launch_bounds__(256, 4) ozaki_crt_kernel(const __grid_constant__ OzFinish f)
{
    const int pair = threadIdx.x & 7;
    const int row = blockIdx.y * kCrtRows + (threadIdx.x >> 3);
    const int col0 = blockIdx.x * 16 + pair * 2;
    const int n = f.n;
    const int tm = (blockIdx.y * kCrtRows) / OZ_TILE_M, tn = (blockIdx.x * 16) / OZ_TN;
    if (!f.tile_ran[(size_t)tn * f.tiles_m + tm] || row >= n || col0 >= n) {
        return;
    }
    // Every output of a tile that ran is written here, flagged or not: the
    // form's own products skipped these tiles.
    const uint8_t* src = f.residues + ((size_t)blockIdx.x * f.y_pad + row) * 16 + pair * 2;
    double xr[2], xi[2];
    {
        uint32_t words[kOzMods];
#pragma unroll
        for (int mi = 0; mi < kOzMods; ++mi) {
            words[mi] = __ldcs(reinterpret_cast<const unsigned short*>(src + (size_t)(2 * mi) * f.y_plane));
        }
        crt_part2(f.crt, words, 0, xr);
#pragma unroll
        for (int mi = 0; mi < kOzMods; ++mi) {
            words[mi] = __ldcs(reinterpret_cast<const unsigned short*>(src + (size_t)(2 * mi + 1) * f.y_plane));
        }
        crt_part2(f.crt, words, 0, xi);
    }
    const int ei = f.E[row];
    const int ca = f.CA[row];
    uint32_t fallbacks = 0;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        const int col = col0 + c;
        if (col >= n) {
            break;
        }
        const size_t idx = (size_t)col * n + row;
        const int fj = f.F[col];
        bool ok = ei != kOzNonFinite && fj != kOzNonFinite;
        float2 out = make_float2(0.0f, 0.0f);  // a zero row or column: the exact product is zero
        if (ok && ei != kOzZero && fj != kOzZero) {
            const int cnt = ca + f.CB[col];
            if (cnt != 0) {
                // |error| <= cnt 2^(beta - 1): both parts must exceed 2^25 (1 + 2^-20) times that
                const double lim = (double)cnt * 0x1.00001p+71;
                ok = fabs(xr[c]) >= lim && fabs(xi[c]) >= lim;
            }
            const double sc = pow2d(ei + fj - 2 * kOzBeta);  // exact: x is an integer, |x| >= 1 or x = 0
            out = make_float2((float)(xr[c] * sc), (float)(xi[c] * sc));
        }
        if (ok) {
            f.C[idx] = out;
        } else {
            atomicOr(&f.fallback_bits[idx >> 5], 1u << (idx & 31));
            ++fallbacks;
        }
    }
    if (fallbacks != 0) {
        atomicAdd(&f.stats[kStatFallback], fallbacks);
    }
}

// The constants of the moduli, exact in 128-bit integers.
OzCrt make_crt()
{
    OzCrt c{};
    unsigned __int128 M = 1;
    for (int mi = 0; mi < kOzMods; ++mi) {
        M *= (unsigned)kOzModuli[mi];
    }
    const unsigned __int128 mask40 = ((unsigned __int128)1 << 40) - 1;
    auto limbs = [&](unsigned __int128 v, double* out) {
        for (int l = 0; l < 3; ++l) {
            out[l] = (double)(uint64_t)((v >> (40 * l)) & mask40);
        }
    };
    for (int mi = 0; mi < kOzMods; ++mi) {
        const int p = kOzModuli[mi];
        const unsigned __int128 W = M / (unsigned)p;
        const int wm = (int)(W % (unsigned)p);
        int u = 0;
        for (int v = 1; v < p; ++v) {
            if ((wm * v) % p == 1) {
                u = v;
                break;
            }
        }
        const unsigned __int128 w = (W * (unsigned)u) % M;  // W u < M p < 2^119: no overflow
        c.p[mi] = p;
        c.c16[mi] = (1 << 16) % p;
        c.pf[mi] = (float)p;
        c.inv_pf[mi] = 1.0f / (float)p;
        c.pd[mi] = (double)p;
        c.inv_pd[mi] = 1.0 / (double)p;
        limbs(w, c.w[mi]);
    }
    limbs(M, c.m);
    c.k2 = (double)((long double)((unsigned __int128)1 << 80) / (long double)M);
    c.k1 = (double)((long double)((unsigned __int128)1 << 40) / (long double)M);
    return c;
}

// Whether every exact product of order <= kOzMaxN lies within M / 8 (the
// reconstruction's margin).
bool crt_range_ok()
{
    unsigned __int128 M = 1;
    for (int mi = 0; mi < kOzMods; ++mi) {
        M *= (unsigned)kOzModuli[mi];
    }
    const unsigned __int128 bound = (unsigned __int128)(2 * kOzMaxN) << (2 * kOzBeta);
    return bound <= M / 8;
}

}  // namespace

OzLayout oz_layout(int n, uint8_t* base, std::vector<size_t>* guards)
{
    OzLayout L;
    L.kpitch = (n + 63) / 64 * 64;
    L.plane_bytes = (size_t)n * L.kpitch;
    L.y_pad = (n + kOzakiTile - 1) / kOzakiTile * kOzakiTile;
    L.y_plane = (size_t)L.y_pad * L.y_pad;
    const int tiles = L.y_pad / kOzakiTile;
    size_t off = 0;
    const size_t e_off = off;
    off = next_region(off, (size_t)n * 4, guards);
    const size_t f_off = off;
    off = next_region(off, (size_t)n * 4, guards);
    const size_t ca_off = off;
    off = next_region(off, (size_t)n * 4, guards);
    const size_t cb_off = off;
    off = next_region(off, (size_t)n * 4, guards);
    const size_t t_off = off;
    off = next_region(off, (size_t)tiles * tiles, guards);
    const size_t a_off = off;
    off = next_region(off, 2 * kOzMods * L.plane_bytes, guards);
    const size_t b_off = off;
    off = next_region(off, 3 * kOzMods * L.plane_bytes, guards);
    const size_t y_off = off;
    off = next_region(off, 2 * kOzMods * L.y_plane, guards);
    L.bytes = off;
    if (base != nullptr) {
        L.E = reinterpret_cast<int*>(base + e_off);
        L.F = reinterpret_cast<int*>(base + f_off);
        L.CA = reinterpret_cast<int*>(base + ca_off);
        L.CB = reinterpret_cast<int*>(base + cb_off);
        L.tile_ran = base + t_off;
        L.planes_a = reinterpret_cast<int8_t*>(base + a_off);
        L.planes_b = reinterpret_cast<int8_t*>(base + b_off);
        L.residues = base + y_off;
    }
    return L;
}

int ozaki_tile_n(int n)
{
    (void)n;
    return OZ_TN;
}

static const OzCrt& crt_constants()
{
    static const OzCrt crt = make_crt();
    return crt;
}

cudaError_t launch_ozaki_split(cudaStream_t s, int n, int pitch, const float2* rows_a, const float2* rows_b,
                               const OzLayout& L)
{
    static const bool range_ok = crt_range_ok();
    if (n > kOzMaxN || !range_ok) {
        return cudaErrorInvalidValue;  // the moduli cover the exact products up to order kOzMaxN
    }
    ozaki_split_kernel<<<2 * n, 256, 0, s>>>(n, pitch, rows_a, rows_b, L.planes_a, L.planes_b, L.kpitch,
                                              L.plane_bytes, L.E, L.F, L.CA, L.CB, crt_constants());
    return cudaGetLastError();
}

cudaError_t launch_ozaki_tiles(cudaStream_t s, int n, const OzLayout& L, const uint32_t* tile_count, uint32_t* stats, uint32_t* fallback_bits, float2* C,
                               int* status, int* launched, const std::function<void(int)>& mark)
{
    const OzCrt& crt = crt_constants();
    int count = 0;
    if (launched != nullptr) {
        *launched = 0;
    }
    if (n > kOzMaxN) {
        return cudaErrorInvalidValue;
    }
    cudaError_t err = cudaSuccess;
    const int tiles = L.y_pad / kOzakiTile;
    {
        CUtensorMap ta, tb;
        const uint64_t dims_a[3] = {(uint64_t)n, (uint64_t)n, (uint64_t)(2 * kOzMods)};
        const uint64_t dims_b[3] = {(uint64_t)n, (uint64_t)n, (uint64_t)(3 * kOzMods)};
        const uint64_t strides[2] = {(uint64_t)L.kpitch, (uint64_t)L.plane_bytes};
        const uint32_t box_a[3] = {(uint32_t)OZ_BK, (uint32_t)OZ_ROWS, 2u};
        const uint32_t box_b[3] = {(uint32_t)OZ_BK, (uint32_t)OZ_BCOLS, 3u};
        if (!encode_tensor_map(&ta, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, dims_a, strides, box_a,
                               CU_TENSOR_MAP_SWIZZLE_64B, L.planes_a) ||
            !encode_tensor_map(&tb, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, dims_b, strides, box_b,
                               CU_TENSOR_MAP_SWIZZLE_64B, L.planes_b)) {
            err = cudaErrorInvalidValue;
        }
        OzParams p{};
        p.n = n;
        p.kblocks = (n + OZ_BK - 1) / OZ_BK;
        p.tiles_m = tiles;
        p.tiles_n = tiles;
        p.tile_count = tile_count;
        p.stats = stats;
        p.tile_ran = L.tile_ran;
        p.residues = L.residues;
        p.y_pad = L.y_pad;
        p.y_plane = L.y_plane;
        p.crt = crt;
        p.status = status;
        if (err == cudaSuccess) {
            err = cudaFuncSetAttribute(ozaki_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)OZ_SMEM);
        }
        if (err == cudaSuccess) {
            cudaLaunchConfig_t cfg{};
            cfg.gridDim = dim3((unsigned)(2 * tiles * tiles));
            cfg.blockDim = dim3(kOzThreads);
            cfg.dynamicSmemBytes = OZ_SMEM;
            cfg.stream = s;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = 2;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            err = cudaLaunchKernelEx(&cfg, ozaki_pair_kernel, ta, tb, p);
            if (err == cudaSuccess) {
                err = cudaGetLastError();
            }
        }
        mark(++count);
    }
    if (err == cudaSuccess) {
        OzFinish f{};
        f.n = n;
        f.tiles_m = tiles;
        f.E = L.E;
        f.F = L.F;
        f.CA = L.CA;
        f.CB = L.CB;
        f.tile_ran = L.tile_ran;
        f.residues = L.residues;
        f.y_pad = L.y_pad;
        f.y_plane = L.y_plane;
        f.stats = stats;
        f.fallback_bits = fallback_bits;
        f.C = C;
        f.crt = crt;
        ozaki_crt_kernel<<<dim3((unsigned)(L.y_pad / 16), (unsigned)(L.y_pad / kCrtRows)), 256, 0, s>>>(f);
        err = cudaGetLastError();
        mark(++count);
    }
    if (launched != nullptr) {
        *launched = count;
    }
    return err;
}

}  // namespace cg3m
