// epilogue.cuh -- the complex alpha/beta epilogue shared by every GEMM kernel.
//
// Reference: CgemmEpilogueVf, blas/gemm/arch35/cgemm_epilogue_kernel.cpp:247-279
// (resultReal = alphaReal*productReal - alphaImag*productImag, ... then
// += beta*C when beta != 0).  Every operation is rounded separately (no
// contraction) so the result is a fixed function of (re, im, alpha, beta, C).
#pragma once

#include <cuda_runtime.h>

namespace cg3m {

struct EpiParams {
    float ar, ai, br, bi;
    int unit, beta_zero;
};

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

}  // namespace cg3m
