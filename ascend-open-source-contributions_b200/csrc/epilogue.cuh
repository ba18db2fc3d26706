// epilogue.cuh -- the complex alpha/beta epilogue shared by every GEMM kernel.
//
// Reference: CgemmEpilogueVf, blas/gemm/arch35/cgemm_epilogue_kernel.cpp:247-279
// (resultReal = alphaReal*productReal - alphaImag*productImag, ... then
// += beta*C when beta != 0).  Every operation is rounded separately (no
// contraction) so the result is a fixed function of (re, im, alpha, beta, C).
#pragma once

#include <cuda_runtime.h>

#include "../../include/cg3m.h"

namespace cg3m {

struct EpiParams {
    float ar, ai, br, bi;
    int unit, beta_zero;
    // Non-finite repair (cg3mCgemm with alpha = 1, beta = 0): an output whose
    // three-product value is not finite is recomputed from the caller's A and
    // B (ops ta, tb, leading dimensions lda, ldb, depth k) before it is stored.
    int repair;
    int ta, tb, k, lda, ldb;
    const float2* A;
    const float2* B;
};

// Non-finite repair (RepairNonFiniteOutput, cgemm_compute_kernel.cpp:672-706):
// the product op(A)(row, :) . op(B)(:, col) recomputed over the whole K in
// increasing order with each FP32 product materialised (rr, ii, ri, ir) and
// re += rr - ii, im += ri + ir, one rounding per operation.  A 3M product that
// overflowed before cancelling gets the four-product value scalar BLAS gives.
__device__ __forceinline__ float2 repair_four_product(const float2* A, int lda, int ta, const float2* B, int ldb,
                                                      int tb, int k, int row, int col)
{
    const bool na = ta == CG3M_OP_N || ta == CG3M_OP_R;
    const bool nb = tb == CG3M_OP_N || tb == CG3M_OP_R;
    const float ca = (ta == CG3M_OP_C || ta == CG3M_OP_R) ? -1.0f : 1.0f;
    const float cb = (tb == CG3M_OP_C || tb == CG3M_OP_R) ? -1.0f : 1.0f;
    float re = 0.0f, im = 0.0f;
    for (int kk = 0; kk < k; ++kk) {
        const float2 a = A[na ? (size_t)row + (size_t)kk * lda : (size_t)kk + (size_t)row * lda];
        const float2 b = B[nb ? (size_t)kk + (size_t)col * ldb : (size_t)col + (size_t)kk * ldb];
        const float av = a.y * ca, bv = b.y * cb;
        const float rr = __fmul_rn(a.x, b.x), ii = __fmul_rn(av, bv);
        const float ri = __fmul_rn(a.x, bv), ir = __fmul_rn(av, b.x);
        re = __fadd_rn(re, __fsub_rn(rr, ii));
        im = __fadd_rn(im, __fadd_rn(ri, ir));
    }
    return make_float2(re, im);
}

// alpha == 1 and beta == 0 store (re, im) unchanged (the reference's fused
// path writes the merged products directly); beta == 0 never reads C.
__device__ __forceinline__ float2 epilogue_value(float re, float im, const EpiParams& e, const float2* cptr)
{
    if (e.unit) {
        return make_float2(re, im);
    }
    float xr = __fsub_rn(__fmul_rn(e.ar, re), __fmul_rn(e.ai, im));
    float xi = __fadd_rn(__fmul_rn(e.ar, im), __fmul_rn(e.ai, re));
    if (!e.beta_zero) {
        const float2 c = *cptr;
        xr = __fadd_rn(xr, __fsub_rn(__fmul_rn(e.br, c.x), __fmul_rn(e.bi, c.y)));
        xi = __fadd_rn(xi, __fadd_rn(__fmul_rn(e.br, c.y), __fmul_rn(e.bi, c.x)));
    }
    return make_float2(xr, xi);
}

// The epilogue of output (row, col) with the non-finite repair applied first
// when the call asks for it.
__device__ __forceinline__ float2 epilogue_at(float re, float im, const EpiParams& e, const float2* cptr, int row,
                                              int col)
{
    if (e.repair && !(isfinite(re) && isfinite(im))) {
        const float2 v = repair_four_product(e.A, e.lda, e.ta, e.B, e.ldb, e.tb, e.k, row, col);
        re = v.x;
        im = v.y;
    }
    return epilogue_value(re, im, e, cptr);
}

}  // namespace cg3m
