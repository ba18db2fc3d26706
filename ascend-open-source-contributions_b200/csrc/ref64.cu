// ref64.cu -- FP64 reference product and error report (diagnostics only).
//
// Every result can report its normwise and worst
// componentwise errors (real and imaginary parts separately) against an FP64
// zgemm.  For full-size problems that reference is computed here, on the
// device, in complex128 with a plain 32x32 shared-memory tiling; it is never
// used to produce a cgemm3m result.
#include "cg3m_internal.h"

namespace cg3m {
namespace {

struct Ref64 {
    int ta, tb, m, n, k;
    double ar, ai, br, bi;
    const float2* A;
    int lda;
    const float2* B;
    int ldb;
    const float2* C;
    int ldc;
    double2* out;
};

__device__ __forceinline__ double2 load_op(const float2* x, int ld, int op, int r, int c)
{
    const bool normal = op == CG3M_OP_N || op == CG3M_OP_R;
    const float2 v = normal ? x[(size_t)c * ld + r] : x[(size_t)r * ld + c];
    const bool conj = op == CG3M_OP_C || op == CG3M_OP_R;
    return make_double2((double)v.x, conj ? -(double)v.y : (double)v.y);
}

constexpr int T = 32;

__global__ void zgemm_ref_kernel(Ref64 p)
{
    __shared__ double2 sa[T][T + 1];
    __shared__ double2 sb[T][T + 1];
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    const int i0 = blockIdx.x * T, j0 = blockIdx.y * T;
    double accr[4] = {0, 0, 0, 0}, acci[4] = {0, 0, 0, 0};
    for (int l0 = 0; l0 < p.k; l0 += T) {
        for (int q = ty; q < T; q += 8) {
            const int r = i0 + tx, c = l0 + q;
            sa[q][tx] = (r < p.m && c < p.k) ? load_op(p.A, p.lda, p.ta, r, c) : make_double2(0, 0);
            const int rb = l0 + tx, cb = j0 + q;
            sb[q][tx] = (rb < p.k && cb < p.n) ? load_op(p.B, p.ldb, p.tb, rb, cb) : make_double2(0, 0);
        }
        __syncthreads();
        for (int l = 0; l < T; ++l) {
            const double2 a = sa[l][tx];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double2 b = sb[ty + 8 * q][l];
                accr[q] = fma(a.x, b.x, fma(-a.y, b.y, accr[q]));
                acci[q] = fma(a.x, b.y, fma(a.y, b.x, acci[q]));
            }
        }
        __syncthreads();
    }
    const int i = i0 + tx;
    if (i >= p.m) {
        return;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = j0 + ty + 8 * q;
        if (j >= p.n) {
            continue;
        }
        double r = p.ar * accr[q] - p.ai * acci[q];
        double im = p.ar * acci[q] + p.ai * accr[q];
        if (p.br != 0.0 || p.bi != 0.0) {
            const float2 c = p.C[(size_t)j * p.ldc + i];
            r += p.br * c.x - p.bi * c.y;
            im += p.br * c.y + p.bi * c.x;
        }
        p.out[(size_t)j * p.m + i] = make_double2(r, im);
    }
}

__device__ __forceinline__ unsigned long long ord(double v)
{
    // Non-negative doubles order like their bit patterns; NaN counts as +inf.
    if (!(v == v)) {
        v = __longlong_as_double(0x7ff0000000000000ll);
    }
    return (unsigned long long)__double_as_longlong(v);
}

__global__ void error_kernel(int m, int n, const float2* C, int ldc, const double2* ref, double* rep)
{
    double s_d = 0, s_x = 0, rel_r = 0, rel_i = 0, abs_r = 0, abs_i = 0;
    const size_t total = (size_t)m * n;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(idx / m), i = (int)(idx - (size_t)j * m);
        const float2 c = C[(size_t)j * ldc + i];
        const double2 x = ref[idx];
        const double dr = fabs((double)c.x - x.x), di = fabs((double)c.y - x.y);
        s_d += dr * dr + di * di;
        s_x += x.x * x.x + x.y * x.y;
        abs_r = fmax(abs_r, dr);
        abs_i = fmax(abs_i, di);
        if (!(dr == dr)) abs_r = rel_r = INFINITY;
        if (!(di == di)) abs_i = rel_i = INFINITY;
        if (x.x != 0) rel_r = fmax(rel_r, dr / fabs(x.x));
        if (x.y != 0) rel_i = fmax(rel_i, di / fabs(x.y));
    }
    for (int off = 16; off > 0; off >>= 1) {
        s_d += __shfl_xor_sync(0xffffffffu, s_d, off);
        s_x += __shfl_xor_sync(0xffffffffu, s_x, off);
        rel_r = fmax(rel_r, __shfl_xor_sync(0xffffffffu, rel_r, off));
        rel_i = fmax(rel_i, __shfl_xor_sync(0xffffffffu, rel_i, off));
        abs_r = fmax(abs_r, __shfl_xor_sync(0xffffffffu, abs_r, off));
        abs_i = fmax(abs_i, __shfl_xor_sync(0xffffffffu, abs_i, off));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&rep[0], s_d);
        atomicAdd(&rep[1], s_x);
        atomicMax(reinterpret_cast<unsigned long long*>(&rep[2]), ord(rel_r));
        atomicMax(reinterpret_cast<unsigned long long*>(&rep[3]), ord(rel_i));
        atomicMax(reinterpret_cast<unsigned long long*>(&rep[4]), ord(abs_r));
        atomicMax(reinterpret_cast<unsigned long long*>(&rep[5]), ord(abs_i));
    }
}

}  // namespace

cudaError_t launch_zgemm_ref(cudaStream_t s, const Problem& p, const void* Cin, void* out64)
{
    Ref64 r{p.transa, p.transb, p.m, p.n, p.k, p.ar, p.ai, p.br, p.bi, static_cast<const float2*>(p.A), p.lda,
            static_cast<const float2*>(p.B), p.ldb, static_cast<const float2*>(Cin), p.ldc,
            static_cast<double2*>(out64)};
    const dim3 grid(ceil_div(p.m, T), ceil_div(p.n, T)), block(T, 8);
    zgemm_ref_kernel<<<grid, block, 0, s>>>(r);
    return cudaGetLastError();
}

cudaError_t launch_error_report(cudaStream_t s, int m, int n, const void* C, int ldc, const void* out64,
                                double* dev_report)
{
    cudaError_t e = cudaMemsetAsync(dev_report, 0, 8 * sizeof(double), s);
    if (e != cudaSuccess) {
        return e;
    }
    const size_t total = (size_t)m * n;
    int blocks = (int)((total + 255) / 256);
    blocks = blocks > 148 * 8 ? 148 * 8 : blocks;
    error_kernel<<<blocks, 256, 0, s>>>(m, n, static_cast<const float2*>(C), ldc, static_cast<const double2*>(out64),
                                        dev_report);
    return cudaGetLastError();
}

}  // namespace cg3m
