// pack.cu -- deinterleave / pack kernel.
//
// Reference: gemm_cgemm_deinterleave_kernel, blas/gemm/arch35/cgemm_kernel.cpp
// :137-157 and DeinterleaveElement, cgemm_deinterleave_common.h:18-52.  The
// reference splits interleaved complex A and B into FP32 planes Ar, Ai, Ar+Ai
// (and the B counterparts) for the standard 3M products, applying the
// conjugation of op 'C' to the imaginary part, and keeps the stored shape.
//
// B200 design: one launch packs both operands (blockIdx.z selects A or B).
// Unlike the reference, op() is resolved here: each plane is written in the
// one layout its GEMM consumes, so every GEMM kernel has a single layout.
//   MN-major (FP32 FFMA GEMM):  A plane [k][pitch] holds op(A)(i,p) at p*pitch+i,
//                               B plane [k][pitch] holds op(B)(p,j) at p*pitch+j.
//   K-major  (tensor-core GEMM): A plane [m][pitch] holds op(A)(i,p) at i*pitch+p,
//                               B plane [n][pitch] holds op(B)(p,j) at j*pitch+p.
// Each plane element is written once; 32x32 complex tiles are staged through
// shared memory when the source's contiguous dimension is not the plane's.
// Components: re, im (conjugated), sum = fl(re + im).  Tensor-core forms split
// every component into TF32 hi/lo or three BF16 terms after the sum is formed
// in FP32, so the split never changes the 3M identity.
#include <cuda_bf16.h>

#include "cg3m_internal.h"

namespace cg3m {
namespace {

struct PackSide {
    const float2* src;  // stored matrix, column-major
    int rows, cols, ld; // stored shape
    int trans;          // 1: plane rows follow source rows (transpose through smem)
    float conj;         // -1 for op C / R, else +1
    void* out;          // plane 0; plane q at out + q*plane_elems elements
    int pitch;
    size_t plane_elems;
    // Packed rows with the leading planes (tensor-core forms' rounding pass):
    // the form's planes, of which the leading split term of re and im is written.
    void* lead;
    int lead_pitch;
    size_t lead_plane_elems;
    // The rest of the planes (same pass): per 256-row band of the plane rows,
    // nonzero when a 256 x 256 tile of that band is left to the form's products.
    const uint8_t* band_need;
};

__device__ __forceinline__ float tf32_rna(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// Writes the planes of one component value v (component c in 0..2).  REST:
// all but the leading split term of re and im (written with the packed rows).
template <int FORM, bool REST = false>
__device__ __forceinline__ void put(const PackSide& s, int c, size_t idx, float v)
{
    if constexpr (FORM == CG3M_FORM_FP32) {
        static_cast<float*>(s.out)[c * s.plane_elems + idx] = v;
    } else if constexpr (FORM == CG3M_FORM_TF32X3) {
        const float hi = tf32_rna(v);
        const float lo = tf32_rna(v - hi);
        float* o = static_cast<float*>(s.out);
        if (!REST || c == 2) {
            o[(2 * c) * s.plane_elems + idx] = hi;
        }
        o[(2 * c + 1) * s.plane_elems + idx] = lo;
    } else {
        const __nv_bfloat16 b0 = __float2bfloat16_rn(v);
        const float r1 = v - __bfloat162float(b0);
        const __nv_bfloat16 b1 = __float2bfloat16_rn(r1);
        const float r2 = r1 - __bfloat162float(b1);
        const __nv_bfloat16 b2 = __float2bfloat16_rn(r2);
        __nv_bfloat16* o = static_cast<__nv_bfloat16*>(s.out);
        if (!REST || c == 2) {
            o[(3 * c) * s.plane_elems + idx] = b0;
        }
        o[(3 * c + 1) * s.plane_elems + idx] = b1;
        o[(3 * c + 2) * s.plane_elems + idx] = b2;
    }
}

// Interleaved complex rows of op(X) (conjugation applied) for the rounding-
// correction pass: the reference's cgemm3m_pack_kernel transpose
// (cgemm3m_rounding_kernel.cpp:148-190), so that every output's K vectors are
// contiguous.
// kFormRowsTf32 / kFormRowsBf16 also write the leading split term of re and
// im into the form's planes (the risk-plane GEMM of the tensor-core forms'
// pass reads those alone), with the values the full pack would write.
constexpr int kFormRows = 100;
constexpr int kFormRowsTf32 = 101;
constexpr int kFormRowsBf16 = 102;

// One element of op(X) at plane row prow, plane column pcol.
template <int FORM, bool REST = false>
__device__ __forceinline__ void put_all(const PackSide& s, int prow, int pcol, float2 v)
{
    const float re = v.x;
    const float im = v.y * s.conj;
    if constexpr (FORM == kFormRows || FORM == kFormRowsTf32 || FORM == kFormRowsBf16) {
        static_cast<float2*>(s.out)[(size_t)prow * s.pitch + pcol] = make_float2(re, im);
        const size_t li = (size_t)prow * s.lead_pitch + pcol;
        if constexpr (FORM == kFormRowsTf32) {
            float* o = static_cast<float*>(s.lead);
            o[li] = tf32_rna(re);
            o[2 * s.lead_plane_elems + li] = tf32_rna(im);
        } else if constexpr (FORM == kFormRowsBf16) {
            __nv_bfloat16* o = static_cast<__nv_bfloat16*>(s.lead);
            o[li] = __float2bfloat16_rn(re);
            o[3 * s.lead_plane_elems + li] = __float2bfloat16_rn(im);
        }
        return;
    }
    const size_t idx = (size_t)prow * s.pitch + pcol;
    put<FORM, REST>(s, 0, idx, re);
    put<FORM, REST>(s, 1, idx, im);
    put<FORM, REST>(s, 2, idx, __fadd_rn(re, im));
}

constexpr int TILE = 32;
constexpr int ROWS = 8;

template <int FORM, bool REST = false>
__global__ void __launch_bounds__(TILE* ROWS) pack_kernel(PackSide a, PackSide b)
{
    __shared__ float2 tile[TILE][TILE + 1];
    // Block x of side z covers tiles x, x + gridDim.x, ... of that side's own
    // tile grid (tile t at (t mod tiles_r, t / tiles_r)), so a long-K shape
    // launches no blocks over the other side's extent.  The full packs launch
    // one block per tile; the rest of the planes in the rounding pass uses a
    // smaller grid, as most of its tiles may lie in bands it skips.
    const PackSide& s = blockIdx.z == 0 ? a : b;
    const int tiles_r = (s.rows + TILE - 1) / TILE;
    const long long tiles = (long long)tiles_r * ((s.cols + TILE - 1) / TILE);
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (long long t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int r0 = (int)(t % tiles_r) * TILE;
        const int c0 = (int)(t / tiles_r) * TILE;
        if constexpr (REST) {
            // plane rows r0.. (transposed) or c0.. lie in one 256-row band
            if (!s.band_need[(s.trans ? r0 : c0) / 256]) {
                continue;
            }
        }
        if (!s.trans) {
            // Plane row = source column, plane column = source row: both contiguous.
            const int r = r0 + tx;
            if (r < s.rows) {
#pragma unroll
                for (int q = 0; q < TILE / ROWS; ++q) {
                    const int c = c0 + ty + q * ROWS;
                    if (c < s.cols) {
                        const float2 v = __ldg(&s.src[(size_t)c * s.ld + r]);
                        put_all<FORM, REST>(s, c, r, v);
                    }
                }
            }
            continue;
        }
        // Plane row = source row, plane column = source column: transpose the tile.
        {
            const int r = r0 + tx;
#pragma unroll
            for (int q = 0; q < TILE / ROWS; ++q) {
                const int c = c0 + ty + q * ROWS;
                if (r < s.rows && c < s.cols) {
                    tile[ty + q * ROWS][tx] = __ldg(&s.src[(size_t)c * s.ld + r]);
                }
            }
        }
        __syncthreads();
        const int c = c0 + tx;
        if (c < s.cols) {
#pragma unroll
            for (int q = 0; q < TILE / ROWS; ++q) {
                const int r = r0 + ty + q * ROWS;
                if (r < s.rows) {
                    put_all<FORM, REST>(s, r, c, tile[tx][ty + q * ROWS]);
                }
            }
        }
        __syncthreads();  // the tile is rewritten by the next iteration
    }
}

// Blocks per side: the larger of the two sides' 32 x 32 tile counts.
unsigned pack_blocks(const PackSide& a, const PackSide& b)
{
    const long long ta = (long long)ceil_div(a.rows, TILE) * ceil_div(a.cols, TILE);
    const long long tb = (long long)ceil_div(b.rows, TILE) * ceil_div(b.cols, TILE);
    return (unsigned)(ta > tb ? ta : tb);
}

}  // namespace

cudaError_t launch_pack_rows(cudaStream_t stream, const Problem& p, void* rows_a, void* rows_b, int pitch,
                             const Plan* lead_plan, void* ws)
{
    auto side = [&](bool isA) {
        PackSide s{};
        const int op = isA ? p.transa : p.transb;
        const bool normal = op == CG3M_OP_N || op == CG3M_OP_R;
        const int opr = isA ? p.m : p.k;
        const int opc = isA ? p.k : p.n;
        s.src = static_cast<const float2*>(isA ? p.A : p.B);
        s.rows = normal ? opr : opc;
        s.cols = normal ? opc : opr;
        s.ld = isA ? p.lda : p.ldb;
        s.conj = (op == CG3M_OP_C || op == CG3M_OP_R) ? -1.0f : 1.0f;
        // K-major rows: A row i holds op(A)(i, :), B row j holds op(B)(:, j).
        s.trans = isA ? (normal ? 1 : 0) : (normal ? 0 : 1);
        s.out = isA ? rows_a : rows_b;
        s.pitch = pitch;  // row stride in complex elements (>= k)
        s.plane_elems = 0;
        if (lead_plan != nullptr) {
            // the K-major planes follow op(X) rows like the packed rows, so the
            // tile walk (s.trans) is the same
            s.lead = static_cast<uint8_t*>(ws) + (isA ? lead_plan->planes_a_off : lead_plan->planes_b_off);
            s.lead_pitch = isA ? lead_plan->pitch_a : lead_plan->pitch_b;
            s.lead_plane_elems = isA ? lead_plan->plane_a_elems : lead_plan->plane_b_elems;
        }
        return s;
    };
    const PackSide a = side(true), b = side(false);
    const dim3 grid(pack_blocks(a, b), 1, 2), block(TILE, ROWS);
    if (lead_plan == nullptr || lead_plan->form == CG3M_FORM_FP32) {
        pack_kernel<kFormRows><<<grid, block, 0, stream>>>(a, b);
    } else if (lead_plan->form == CG3M_FORM_TF32X3) {
        pack_kernel<kFormRowsTf32><<<grid, block, 0, stream>>>(a, b);
    } else {
        pack_kernel<kFormRowsBf16><<<grid, block, 0, stream>>>(a, b);
    }
    return cudaGetLastError();
}

cudaError_t launch_pack(cudaStream_t stream, const Problem& p, const Plan& plan, void* ws, const uint8_t* band_a,
                        const uint8_t* band_b)
{
    const bool kmajor = plan.form != CG3M_FORM_FP32;
    auto side = [&](bool isA) {
        PackSide s{};
        const int op = isA ? p.transa : p.transb;
        const bool normal = op == CG3M_OP_N || op == CG3M_OP_R;
        const int opr = isA ? p.m : p.k;  // rows of op(X)
        const int opc = isA ? p.k : p.n;  // cols of op(X)
        s.src = static_cast<const float2*>(isA ? p.A : p.B);
        s.rows = normal ? opr : opc;
        s.cols = normal ? opc : opr;
        s.ld = isA ? p.lda : p.ldb;
        s.conj = (op == CG3M_OP_C || op == CG3M_OP_R) ? -1.0f : 1.0f;
        // MN-major planes are indexed [k][mn]: A wants source rows on the plane's
        // columns when op(A) is N (no transpose); B when op(B) is T/C.
        // K-major planes are indexed [mn][k]: the opposite.
        const bool plane_cols_are_src_rows = isA ? (normal != kmajor) : (normal == kmajor);
        s.trans = plane_cols_are_src_rows ? 0 : 1;
        s.out = static_cast<uint8_t*>(ws) + (isA ? plan.planes_a_off : plan.planes_b_off);
        s.pitch = isA ? plan.pitch_a : plan.pitch_b;
        s.plane_elems = isA ? plan.plane_a_elems : plan.plane_b_elems;
        s.band_need = isA ? band_a : band_b;
        return s;
    };
    const PackSide a = side(true), b = side(false);
    const dim3 grid(pack_blocks(a, b), 1, 2), block(TILE, ROWS);
    if (band_a != nullptr) {
        // the rest of the tensor-core planes, for the bands the form's products read
        const dim3 rest_grid(grid.x < 148u * 8u ? grid.x : 148u * 8u, 1, 2);
        switch (plan.form) {
            case CG3M_FORM_TF32X3: pack_kernel<CG3M_FORM_TF32X3, true><<<rest_grid, block, 0, stream>>>(a, b); break;
            case CG3M_FORM_FP32: return cudaErrorInvalidValue;
            default: pack_kernel<CG3M_FORM_BF16X6, true><<<rest_grid, block, 0, stream>>>(a, b); break;
        }
        return cudaGetLastError();
    }
    switch (plan.form) {
        case CG3M_FORM_FP32: pack_kernel<CG3M_FORM_FP32><<<grid, block, 0, stream>>>(a, b); break;
        case CG3M_FORM_TF32X3: pack_kernel<CG3M_FORM_TF32X3><<<grid, block, 0, stream>>>(a, b); break;
        default: pack_kernel<CG3M_FORM_BF16X6><<<grid, block, 0, stream>>>(a, b); break;
    }
    return cudaGetLastError();
}

}  // namespace cg3m
