// planner.cpp -- argument validation and path / tile / K-split selection.
//
// Reference: ValidateCgemmParams and ValidateCgemmPointers
// (blas/gemm/arch35/cgemm_host.cpp:589-634,687-699), LaunchComplexGemm
// (:701-730), CalculateCgemmWorkspaceSizes (:228-285) with
// SelectCgemmAccumulationTile (:130), EstimateCgemmCoreWork (:145),
// SelectCgemmProductTile (:157), SelectCgemm3mDecomposition (:174) and the
// rounding gate (:234-238), AllocateCgemmWorkspace (:326-360).
//
// The validation order, statuses and quick returns are the reference's.  The
// tile/K-split policy keeps the reference's structure -- a joint search over
// output tile x K partitions that minimises the busiest core's work times
// (span + 16), with a forced deeper split for narrow long-K outputs -- but its
// capacities are the B200's: the "cores" are SM slots (148 SMs x resident CTAs
// of the tile), the tiles are this kernel's, and the partition bound scales
// with how few tiles there are, since a 148-SM part needs far more
// independent tasks than a 1-4-way split of a handful of tiles provides.
#include <algorithm>
#include <cstring>
#include <limits>

#include <vector>

#include "cg3m_internal.h"

namespace cg3m {

static bool is_op(int op, bool allow_conj_only)
{
    return op == CG3M_OP_N || op == CG3M_OP_T || op == CG3M_OP_C || (allow_conj_only && op == CG3M_OP_R);
}

cg3mStatus_t validate(int transa, int transb, int m, int n, int k, const cg3mComplex* alpha, const void* A, int lda,
                      const void* B, int ldb, const cg3mComplex* beta, const void* C, int ldc, bool allow_conj_only,
                      int* action)
{
    *action = 0;
    // Enum errors are reported as INVALID_VALUE by the 3m entry (cgemm_host.cpp:713).
    if (!is_op(transa, allow_conj_only) || !is_op(transb, allow_conj_only)) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    if (m < 0 || n < 0 || k < 0) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    const bool normal_a = transa == CG3M_OP_N || transa == CG3M_OP_R;
    const bool normal_b = transb == CG3M_OP_N || transb == CG3M_OP_R;
    if (lda < std::max(1, normal_a ? m : k)) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    if (ldb < std::max(1, normal_b ? k : n)) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    if (ldc < std::max(1, m)) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    if (alpha == nullptr || beta == nullptr) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    if (m == 0 || n == 0) {
        return CG3M_STATUS_SUCCESS;  // quick return after validation (cgemm_host.cpp:715)
    }
    const bool alpha_zero = alpha->real == 0.0f && alpha->imag == 0.0f;
    if (C == nullptr) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    if (!alpha_zero && k > 0 && (A == nullptr || B == nullptr)) {
        return CG3M_STATUS_INVALID_VALUE;
    }
    if (k == 0 || alpha_zero) {
        const bool beta_one = beta->real == 1.0f && beta->imag == 0.0f;
        *action = beta_one ? 0 : 1;  // cgemm_host.cpp:639
        return CG3M_STATUS_SUCCESS;
    }
    *action = 2;
    return CG3M_STATUS_SUCCESS;
}

namespace {

struct TileChoice {
    int bm, bn;
    int slots_per_sm;  // resident CTAs per SM of this tile's kernel
};

// FP32 FFMA kernel tile (gemm_fp32.cu).  The kernel also instantiates 64 x 64,
// 64 x 32 and 32 x 32 tiles, but measured on B200 they run at about a third of
// the 128 x 64 tile's per-SM FFMA rate (short pipelines, few warps), so the
// planner splits K over 128 x 64 tiles instead (512^3: 64 x 32 x 3 parts
// 62.9 us, 128 x 64 x 4 parts 38.8 us; 1024^3: 306 vs 174 us).
const TileChoice kFp32Tiles[] = {{128, 64, 1}};
// Cost of one wave of 128 x 64 FP32 tiles in K terms of that tile (0.133 us
// per term): a fixed part of about 38 terms (pipeline fill, epilogue, wave
// launch; fitted on 512^3 .. 2048^3) plus the span; the split-K merge costs
// about 30 terms plus the partial planes it reads.
constexpr uint64_t kFp32WaveFixed = 38;
constexpr uint64_t kMergeFixed = 30;
constexpr uint64_t kMergeFloatsPerTerm = 41500;
// With 2..8 partitions the partitions of a tile form one thread-block cluster
// and merge through distributed shared memory inside the GEMM (no merge
// kernel, no partial planes): waves then hold as many clusters as fit at once
// (cudaOccupancyMaxActiveClusters for one block per SM on 148 SMs), and the
// merge costs about one K term per partition.
constexpr int kClusterMergeMax = 8;
constexpr uint64_t kClusterCapOneBlock[kClusterMergeMax] = {148, 74, 45, 33, 26, 22, 15, 15};

uint64_t fp32_waves(uint64_t tiles, int parts, int sm_count)
{
    if (parts > 1 && parts <= kClusterMergeMax) {
        const uint64_t cap = std::max<uint64_t>(1, kClusterCapOneBlock[parts - 1] * (uint64_t)sm_count / 148);
        return (tiles + cap - 1) / cap;
    }
    return (tiles * parts + sm_count - 1) / sm_count;
}
// The same costs in microseconds for the whole packed call (pack kernel over
// op(A) and op(B) -- 8 bytes read, 12 written per element -- GEMM waves, merge
// kernel), fitted on B200 to 28 timed shapes (median error 3.3 %).
constexpr double kPackedFixedUs = 1.64;
constexpr double kPackedUsPerMB = 0.199;
constexpr double kPackedUsPerTerm = 0.1205;
constexpr double kMergeLaunchUs = 3.53;
constexpr double kMergeUsPerTerm = 0.0;
// Tensor-core kernel tile (gemm_tc.cu): 128 x 128, one CTA per SM (TMEM).
const TileChoice kTcTiles[] = {{128, 128, 1}};

// Busiest-SM work for `tiles` output tiles split into `parts` K partitions
// (EstimateCgemmCoreWork, cgemm_host.cpp:145-156, with SM slots as cores).
uint64_t core_work(const TileChoice& t, int m, int n, int parts, int sm_count)
{
    const uint64_t tiles = (uint64_t)ceil_div(m, t.bm) * ceil_div(n, t.bn);
    const uint64_t slots = (uint64_t)sm_count * t.slots_per_sm;
    const uint64_t waves = (tiles * parts + slots - 1) / slots;
    // Work per wave: one tile's multiply-adds per K term, scaled by how many of
    // the SM's slots share its FP32 pipe.
    const uint64_t rows = std::min(m, t.bm), cols = std::min(n, t.bn);
    return waves * rows * cols * (uint64_t)t.slots_per_sm;
}

// kSpan = ceil(ceil(k/g)/parts)*g (cgemm_host.cpp:274-275 with g = 16).  The
// granule g is the GEMM kernel's K-tile so that only the last partition has a
// ragged tail: 16 for the FP32 kernel, 64 elements (one 128-byte row of the
// widest split plane) for the tensor-core kernel.
int k_span(int k, int parts, int g = 16)
{
    return ceil_div(ceil_div(k, g), parts) * g;
}

double packed_time_us(const Problem& p, int parts, int span, uint64_t tiles, int sm_count)
{
    const uint64_t waves = fp32_waves(tiles, parts, sm_count);
    const double bytes = ((double)p.m * p.k + (double)p.k * p.n) * 20.0;
    double us = kPackedFixedUs + kPackedUsPerMB * bytes * 1e-6 + kPackedUsPerTerm * (double)waves * (span + kFp32WaveFixed);
    if (parts > kClusterMergeMax) {
        us += kMergeLaunchUs + kMergeUsPerTerm * (kMergeFixed + (double)(2 * parts + 2) * p.m * p.n / kMergeFloatsPerTerm);
    } else if (parts > 1) {
        us += kPackedUsPerTerm * parts;
    }
    return us;
}

// Tensor-core call in microseconds (pack of the split planes, waves of CTA-pair
// tiles, merge), fitted on B200 to the 200 performance shapes (graph replay;
// median error 13-19 %, hence the margin where it is compared).
double tc_time_us(const Problem& p, int form, int parts, int span, int sm_count)
{
    const uint64_t tiles = p.m > 128 ? (uint64_t)ceil_div(p.m, 256) * ceil_div(p.n, 128)
                                     : (uint64_t)ceil_div(p.n, 128);
    const double waves = (double)((tiles * parts + sm_count - 1) / sm_count);
    const double elems = (double)p.m * p.k + (double)p.k * p.n;
    if (form == CG3M_FORM_TF32X3) {
        return 11.80 + 0.1374 * elems * 32e-6 + 0.11003 * waves * span + (parts > 1 ? 1.25 : 0.0);
    }
    const double terms = form == CG3M_FORM_BF16X9 ? 1.5 : 1.0;  // nine products instead of six
    return 13.27 + 0.1055 * elems * 44e-6 + 0.08315 * terms * waves * span;
}

}  // namespace

bool make_plan(const Problem& p, const cg3mOptions& opts, int sm_count, Plan* plan)
{
    Plan out{};
    out.action = 2;
    out.form = opts.form;
    out.unit = p.ar == 1.0f && p.ai == 0.0f && p.br == 0.0f && p.bi == 0.0f;
    // Tensor-core forms restart their TMEM accumulators every `tc_segment` K
    // terms and merge segments with round-to-nearest FP32 adds.  The truncation
    // error of one segment grows with its length, while the plain FP32 form's
    // error grows with sqrt(K); these lengths keep the tensor-core error at or
    // below the plain form's (measured on data with a 2^16 dynamic range in the
    // imaginary parts), at the cost of more merges for short K.
    out.tc_segment = opts.tc_segment > 0 ? opts.tc_segment : (p.k >= 2048 ? 128 : p.k > 1024 ? 64 : 32);
    out.beta_zero = p.br == 0.0f && p.bi == 0.0f;
    if (sm_count <= 0) {
        sm_count = 148;
    }
    const bool tc = opts.form != CG3M_FORM_FP32;
    if (opts.engine < 0 || opts.engine > 2 || opts.onchip_tile < 0 || opts.onchip_tile > 6) {
        return false;
    }

    // Rounding-correction gate (cgemm_host.cpp:234-238).
    out.rounding = opts.rounding == CG3M_ROUNDING_AUTO && out.unit && p.m == p.n && p.n == p.k && p.k >= 2048 &&
                   p.k <= 4096 && p.lda == p.m && p.ldb == p.m && p.ldc == p.m;

    // ---- engine 2: one launch, K partitions merged in a cluster -----------------
    if (opts.engine == 2) {
        if (tc || out.rounding || opts.k_partitions > 8) {
            return false;
        }
        int parts = opts.k_partitions;
        while (parts > 1 && (parts - 1) * k_span(p.k, parts) >= p.k) {
            --parts;
        }
        int tile = 0;
        out.est_us = plan_single(p.m, p.n, p.k, 0, sm_count, opts.onchip_tile - 1, parts, &tile, &parts);
        out.engine = 2;
        out.onchip_tile = tile;
        out.tile_m = single_tile_bm(tile);
        out.tile_n = single_tile_bn(tile);
        out.parts = parts;
        out.span = parts > 1 ? k_span(p.k, parts) : p.k;
        out.total = 0;
        *plan = out;
        return true;
    }

    // ---- tile x K-partition search -------------------------------------------
    const TileChoice* tiles = tc ? kTcTiles : kFp32Tiles;
    const int granule = tc ? 64 : 16;
    const int ntiles = 1;
    const uint64_t default_tiles = (uint64_t)ceil_div(p.m, tiles[0].bm) * ceil_div(p.n, tiles[0].bn);
    TileChoice best_tile = tiles[0];
    int best_parts = 1;
    if (opts.k_partitions > 0) {
        best_parts = std::min(opts.k_partitions, 64);
    } else if (!tc && !out.rounding) {
        // FP32: waves of 128 x 64 tiles at (span + fixed) each, plus the merge
        // (EstimateCgemmCoreWork's busiest-core work with measured B200 costs).
        uint64_t best = std::numeric_limits<uint64_t>::max();
        for (int parts = 1; parts <= 32; ++parts) {
            const int span = k_span(p.k, parts, granule);
            if ((parts - 1) * span >= p.k || (parts > 1 && span < 64)) {
                continue;
            }
            const uint64_t waves = fp32_waves(default_tiles, parts, sm_count);
            const uint64_t gemm = waves * ((uint64_t)span + kFp32WaveFixed);
            const uint64_t merge =
                parts > kClusterMergeMax ? kMergeFixed + (uint64_t)(2 * parts + 2) * p.m * p.n / kMergeFloatsPerTerm
                : parts > 1              ? (uint64_t)parts
                                         : 0;
            if (gemm + merge < best) {
                best = gemm + merge;
                best_parts = parts;
            }
        }
    } else if (default_tiles < (uint64_t)sm_count * tiles[0].slots_per_sm && !out.rounding) {
        // Few tiles: search jointly (SelectCgemm3mDecomposition, :174-200).
        // Partitions are bounded by what can still fill the machine: at most
        // 4-way as in the reference when tiles are plentiful, deeper only while
        // tiles x parts stays within two waves of SM slots and every partition
        // keeps >= 256 K terms.
        uint64_t best = std::numeric_limits<uint64_t>::max();
        for (int t = 0; t < ntiles; ++t) {
            const uint64_t nt = (uint64_t)ceil_div(p.m, tiles[t].bm) * ceil_div(p.n, tiles[t].bn);
            const uint64_t slots = (uint64_t)sm_count * tiles[t].slots_per_sm;
            int max_parts = (int)std::max<uint64_t>(4, (2 * slots) / std::max<uint64_t>(nt, 1));
            max_parts = std::min(max_parts, 64);
            for (int parts = 1; parts <= max_parts; ++parts) {
                const int span = k_span(p.k, parts, granule);
                if ((parts - 1) * span >= p.k) {
                    continue;
                }
                if (parts > 4 && span < 256) {
                    continue;
                }
                const uint64_t work = core_work(tiles[t], p.m, p.n, parts, sm_count) * (uint64_t)(span + 16);
                // Charge the partial-output traffic of the merge: 2 planes per part.
                const uint64_t merge = parts > 1 ? (uint64_t)parts * p.m * p.n / sm_count : 0;
                if (work + merge < best) {
                    best = work + merge;
                    best_tile = tiles[t];
                    best_parts = parts;
                }
            }
        }
    }
    // Narrow long-K outputs force >= 8 partitions (cgemm_host.cpp:269-273).
    if (opts.k_partitions <= 0 && !tc && p.k >= 1024 && std::min(p.m, p.n) <= 16 && std::max(p.m, p.n) <= 32) {
        best_parts = std::max(best_parts, 8);
    }
    // The tensor-core forms' rounding pass runs its products over the whole K:
    // the risk plane needs the whole chain and the form's products on the
    // tiles the exact recompute does not take run unsplit.
    if (tc && out.rounding) {
        best_parts = 1;
    }
    out.tile_m = best_tile.bm;
    out.tile_n = best_tile.bn;
    out.parts = best_parts;
    out.span = k_span(p.k, best_parts, granule);
    while (out.parts > 1 && (out.parts - 1) * out.span >= p.k) {
        --out.parts;
        out.span = k_span(p.k, out.parts, granule);
    }
    if (out.parts == 1) {
        out.span = p.k;
    }

    // ---- engine (FP32 form without the rounding pass) ---------------------------
    // The one-launch engine skips the pack kernel and the merge kernel; it
    // wins on small and latency-bound shapes, the packed engine's faster FFMA
    // tile on large ones.  Both time models are fitted on B200.
    if (!tc && !out.rounding && opts.engine == 0 && (opts.k_partitions <= 0 || out.parts <= 8)) {
        const bool narrow = p.k >= 1024 && std::min(p.m, p.n) <= 16 && std::max(p.m, p.n) <= 32;
        const int forced = opts.k_partitions > 0 ? out.parts : narrow ? 8 : 0;
        int tile = 0, parts = 0;
        const double single = plan_single(p.m, p.n, p.k, 0, sm_count, -1, forced, &tile, &parts);
        out.est_us = packed_time_us(p, out.parts, out.span, default_tiles, sm_count);
        if (single < out.est_us) {
            out.est_us = single;
            out.engine = 2;
            out.onchip_tile = tile;
            out.tile_m = single_tile_bm(tile);
            out.tile_n = single_tile_bn(tile);
            out.parts = parts;
            out.span = parts > 1 ? k_span(p.k, parts) : p.k;
            out.total = 0;
            *plan = out;
            return true;
        }
    }

    // ---- tensor-core forms on small shapes ---------------------------------------
    // A tensor-core call carries a fixed cost of 12-13 us (pack, TMEM set-up,
    // pipeline fill) that the FP32 engines do not.  Where the FP32 planner's
    // own plan is clearly faster (a 1.1x margin over the rougher tensor-core
    // model), the call runs that plan in plain FP32 -- its error is the plain
    // form's, which every form promises not to exceed -- and reports form
    // FP32.  engine 1 (or a forced K split) keeps the tensor-core path.
    if (tc && !out.rounding && opts.engine == 0 && opts.k_partitions <= 0) {
        cg3mOptions fo = opts;
        fo.form = CG3M_FORM_FP32;
        fo.rounding = CG3M_ROUNDING_OFF;
        Plan fp;
        if (make_plan(p, fo, sm_count, &fp) && fp.est_us * 1.1 < tc_time_us(p, opts.form, out.parts, out.span,
                                                                              sm_count)) {
            *plan = fp;
            return true;
        }
    }

    // ---- workspace layout -----------------------------------------------------
    const bool kmajor = tc;
    int splits = 1;
    size_t elem = 4;
    if (opts.form == CG3M_FORM_TF32X3) {
        splits = 2;
    } else if (opts.form == CG3M_FORM_BF16X6 || opts.form == CG3M_FORM_BF16X9) {
        splits = 3;
        elem = 2;
    }
    out.planes = 3 * splits;
    if (kmajor) {
        // [mn][k] planes: K padded so every row starts on a 128-byte boundary.
        const int kp = (int)align_up((size_t)p.k, 128 / elem);
        out.pitch_a = kp;
        out.pitch_b = kp;
        out.plane_a_elems = (size_t)p.m * kp;
        out.plane_b_elems = (size_t)p.n * kp;
    } else {
        out.pitch_a = (int)align_up((size_t)p.m, 32);
        out.pitch_b = (int)align_up((size_t)p.n, 32);
        out.plane_a_elems = (size_t)out.pitch_a * p.k;
        out.plane_b_elems = (size_t)out.pitch_b * p.k;
    }
    size_t off = 0;
    std::vector<size_t> guards;
    out.planes_a_off = off;
    off = next_region(off, out.plane_a_elems * elem * out.planes, &guards);
    out.planes_b_off = off;
    off = next_region(off, out.plane_b_elems * elem * out.planes, &guards);
    out.partial_pitch = (int)align_up((size_t)p.m, 32);
    out.partial_plane_elems = (size_t)out.partial_pitch * p.n;
    // K splits merged on chip through the tile's cluster: the FP32 GEMM (up to 8
    // partitions) and the tensor-core CTA-pair kernel (used for m > 128; up to 4
    // partitions, two CTAs each).  The pair kernel merges on chip only when all
    // of its clusters of 2 x parts CTAs are resident at once: a grid that one
    // wave holds as loose CTAs but not as clusters runs a second wave, which
    // costs more than the merge launch it saves (1.3-1.6x on 128..144-CTA grids).
    bool tc_merge = false;
    if (tc && p.m > 128 && out.parts <= 4) {
        const uint64_t pair_tiles = (uint64_t)ceil_div(p.m, 256) * ceil_div(p.n, 128);
        const uint64_t cap =
            std::max<uint64_t>(1, kClusterCapOneBlock[2 * out.parts - 1] * (uint64_t)sm_count / 148);
        tc_merge = pair_tiles <= cap;
    }
    out.cluster_merge = !out.rounding && out.parts > 1 &&
                        (tc ? tc_merge
                            : (out.parts <= kClusterMergeMax && out.tile_m == 128 && out.tile_n == 64));
    out.partial_off = off;
    if (out.parts > 1 && !out.cluster_merge) {
        off = next_region(off, out.partial_plane_elems * 4 * 2 * out.parts, &guards);
    }
    out.round_off = off;
    if (out.rounding) {
        std::vector<size_t> inner;
        off = next_region(off, rounding_bytes(p.n, out.form, &inner), &guards);  // layout in rounding.cu
        for (size_t g : inner) {
            guards.push_back(out.round_off + g);
        }
    }
    out.total = off;
    if (guards.size() > (size_t)Plan::kMaxGuards) {
        return false;
    }
    out.guards = (int)guards.size();
    for (size_t i = 0; i < guards.size(); ++i) {
        out.guard_off[i] = guards[i];
    }
    *plan = out;
    return true;
}

}  // namespace cg3m
