// rounding.cu -- the rounding-correction pass (north-star item (d)).
//
// Reference: gemm_cgemm3m_rounding_do, blas/gemm/arch35/cgemm3m_rounding_kernel.cpp
// :474-497, run after the path-tracking GEMM when the call is a contiguous
// square unit-output product of order 2048..4096 (cgemm_host.cpp:234-238):
//   1. pack (:148-190)      op(A) rows and op(B) columns as contiguous complex
//                           K vectors (conjugation applied);
//   2. permute (:406-472)   per-row energies sum |x|^2, accumulated per lane of
//                           a 64-lane segment layout (lane l holds k in
//                           [l*span, (l+1)*span), span = ceil(n/64) | 1) and
//                           reduced across lanes;
//   3. select (:43-130)     flag output (i,j) when max(|Re|,|Im|) or
//                           var = 2^-48 (path + E_i E_j bridge) is not finite,
//                           or 3.75^2 var >= 1e-4; flagged indices are
//                           compacted into a list;
//   4. recompute (:192-404) each flagged output again, in a fixed order.
// B200 design: one CTA of 64 threads per row for the energies (the row is
// staged in shared memory; span is odd so the strided lane reads are
// conflict-free); a grid-stride select with an atomic append (the list order
// does not matter: each flagged output is recomputed independently, so the
// result bits do not depend on it); one warp per flagged output for the
// recompute.  FP32 form: the reference's segmented replay -- the 64 lanes are
// held two per thread, the lane reductions and the inclusive lane scan follow
// a fixed pairwise order.  Tensor-core forms: the flagged outputs are
// recomputed as an FP64 dot product (32 contiguous K chunks, one per thread,
// summed in a fixed tree) and rounded once to FP32.
#include <cstring>
#include <functional>

#include "cg3m_internal.h"

namespace cg3m {

cudaError_t launch_pack_rows(cudaStream_t stream, const Problem& p, void* rows_a, void* rows_b);
cudaError_t launch_gemm_fp32_path(cudaStream_t stream, const Problem& pr, const Plan& plan, void* ws, float* path,
                                  int* status);
cudaError_t launch_gemm_tc_path(cudaStream_t stream, const Problem& pr, const Plan& plan, void* ws, float* path,
                                int* status);

namespace {

constexpr int kLanes = 64;
constexpr float kConfidence = 3.75f;  // CGEMM_ROUNDING_CONFIDENCE, cgemm_host.cpp:37

// ---- 2. energies ----------------------------------------------------------------

__global__ void __launch_bounds__(kLanes) energy_kernel(const float2* __restrict__ rows_a,
                                                        const float2* __restrict__ rows_b, int n, int span,
                                                        float* __restrict__ energy)
{
    extern __shared__ float2 row[];
    __shared__ float lanes[kLanes];
    const int r = blockIdx.x;
    const float2* src = r < n ? rows_a + (size_t)r * n : rows_b + (size_t)(r - n) * n;
    for (int k = threadIdx.x; k < n; k += kLanes) {
        row[k] = src[k];
    }
    __syncthreads();
    const int l = threadIdx.x;
    float e = 0.0f;
    for (int s = 0; s < span; ++s) {
        const int k = l * span + s;
        if (k >= n) {
            break;
        }
        const float2 x = row[k];
        e = __fmaf_rn(x.x, x.x, e);
        e = __fmaf_rn(x.y, x.y, e);
    }
    lanes[l] = e;
    __syncthreads();
    for (int stride = kLanes / 2; stride >= 1; stride /= 2) {
        if (l < stride) {
            lanes[l] = __fadd_rn(lanes[l], lanes[l + stride]);
        }
        __syncthreads();
    }
    if (l == 0) {
        energy[r] = lanes[0];
    }
}

// ---- 3. selection -----------------------------------------------------------------

__global__ void select_kernel(int n, const float2* __restrict__ C, const float* __restrict__ energy,
                              const float* __restrict__ path, float bridge, uint32_t* __restrict__ list,
                              uint32_t* __restrict__ count)
{
    const size_t total = (size_t)n * n;
    const float conf2 = __fmul_rn(kConfidence, kConfidence);
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(idx / n), i = (int)(idx - (size_t)j * n);
        const float2 c = C[idx];
        const float re = fabsf(c.x), im = fabsf(c.y);
        const float magnitude = re > im ? re : im;
        const float variance =
            __fmul_rn(0x1p-48f, __fadd_rn(path[idx], __fmul_rn(__fmul_rn(energy[i], energy[n + j]), bridge)));
        const bool sel = !isfinite(magnitude) || !isfinite(variance) || __fmul_rn(conf2, variance) >= 0.0001f;
        if (sel) {
            const uint32_t pos = atomicAdd(count, 1u);
            list[pos] = (uint32_t)idx;
        }
    }
}

// ---- 4a. FP32 segmented replay (FastSegmentDot) ---------------------------------------

struct Cf {
    float r, i;
};

// One 3M term with the fused identity (ThreeProductTerms, :192-208).
__device__ __forceinline__ Cf term(float2 x, float2 y)
{
    const float p = __fmul_rn(__fadd_rn(x.x, x.y), y.x);
    const float q = __fmul_rn(x.x, __fsub_rn(y.y, y.x));
    const float rr = __fmul_rn(x.y, __fadd_rn(y.x, y.y));
    return Cf{__fsub_rn(p, rr), __fadd_rn(p, q)};
}

// Sum over 64 lanes held as (a = lane t, b = lane t+32) in a warp, in the
// pairwise order v[l] += v[l+stride] for stride 32, 16, ..., 1.
__device__ __forceinline__ float lane_reduce(float a, float b)
{
    float v = __fadd_rn(a, b);  // stride 32
#pragma unroll
    for (int stride = 16; stride >= 1; stride /= 2) {
        const float o = __shfl_down_sync(0xffffffffu, v, stride);
        if ((int)(threadIdx.x & 31) < stride) {
            v = __fadd_rn(v, o);
        }
    }
    return __shfl_sync(0xffffffffu, v, 0);
}

__device__ __forceinline__ float lane_max(float a, float b)
{
    float v = fmaxf(a, b);
#pragma unroll
    for (int stride = 16; stride >= 1; stride /= 2) {
        v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, stride));
    }
    return v;
}

// Inclusive Hillis-Steele scan over 64 lanes (a = lane t, b = lane t+32):
// new[l] = l >= d ? s[l] + s[l-d] : s[l], d = 1, 2, ..., 32.
__device__ __forceinline__ void lane_scan(float& a, float& b)
{
    const int t = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d *= 2) {
        const float a_up = __shfl_up_sync(0xffffffffu, a, d);        // lane t-d (t >= d)
        const float b_up = __shfl_up_sync(0xffffffffu, b, d);        // lane t+32-d (t >= d)
        const float a_wrap = __shfl_sync(0xffffffffu, a, (t + 32 - d) & 31);  // lane t+32-d (t < d)
        const float na = t >= d ? __fadd_rn(a, a_up) : a;
        const float nb = __fadd_rn(b, t >= d ? b_up : a_wrap);
        a = na;
        b = nb;
    }
    b = __fadd_rn(b, a);  // d = 32: lane t+32 adds lane t
}

__global__ void recompute_fp32_kernel(int n, int span, const float2* __restrict__ rows_a,
                                      const float2* __restrict__ rows_b, const uint32_t* __restrict__ list,
                                      const uint32_t* __restrict__ count, float2* __restrict__ C)
{
    const uint32_t total = *count;
    const int t = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < total; w += warps) {
        const uint32_t idx = list[w];
        const int j = (int)(idx / (uint32_t)n), i = (int)(idx - (uint32_t)j * n);
        const float2* x = rows_a + (size_t)i * n;
        const float2* y = rows_b + (size_t)j * n;
        Cf s[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int l = t + 32 * h;
            Cf acc{0.0f, 0.0f};
            for (int q = 0; q < span; ++q) {
                const int k = l * span + q;
                if (k >= n) {
                    break;
                }
                const Cf tv = term(x[k], y[k]);
                acc.r = __fadd_rn(acc.r, tv.r);
                acc.i = __fadd_rn(acc.i, tv.i);
            }
            s[h] = acc;
        }
        const float direct_r = lane_reduce(s[0].r, s[1].r);
        const float direct_i = lane_reduce(s[0].i, s[1].i);
        float pr0 = s[0].r, pr1 = s[1].r, pi0 = s[0].i, pi1 = s[1].i;
        lane_scan(pr0, pr1);
        lane_scan(pi0, pi1);
        // exclusive prefix: lane l gets the inclusive value of lane l-1
        const float prev_r0 = __shfl_up_sync(0xffffffffu, pr0, 1), prev_i0 = __shfl_up_sync(0xffffffffu, pi0, 1);
        const float prev_r1 = __shfl_up_sync(0xffffffffu, pr1, 1), prev_i1 = __shfl_up_sync(0xffffffffu, pi1, 1);
        const float last_r0 = __shfl_sync(0xffffffffu, pr0, 31), last_i0 = __shfl_sync(0xffffffffu, pi0, 31);
        Cf init[2];
        init[0] = t >= 1 ? Cf{prev_r0, prev_i0} : Cf{0.0f, 0.0f};
        init[1] = t >= 1 ? Cf{prev_r1, prev_i1} : Cf{last_r0, last_i0};
        Cf fin[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int l = t + 32 * h;
            float r = __fadd_rn(init[h].r, 0.0f), im = __fadd_rn(init[h].i, 0.0f);
            for (int q = 0; q < span; ++q) {
                const int k = l * span + q;
                if (k >= n) {
                    break;
                }
                const Cf tv = term(x[k], y[k]);
                r = __fadd_rn(r, tv.r);
                im = __fadd_rn(im, tv.i);
            }
            fin[h] = Cf{__fsub_rn(r, init[h].r), __fsub_rn(im, init[h].i)};
        }
        float bridged_r = lane_reduce(fin[0].r, fin[1].r);
        float bridged_i = lane_reduce(fin[0].i, fin[1].i);
        const float max_r = lane_max(fabsf(pr0), fabsf(pr1));
        const float max_i = lane_max(fabsf(pi0), fabsf(pi1));
        // SelectStableSegmentSum (:243-262): keep the direct sum when the
        // prefixes are at least 32x the result.
        if (max_r >= __fmul_rn(fabsf(direct_r), 32.0f)) {
            bridged_r = direct_r;
        }
        if (max_i >= __fmul_rn(fabsf(direct_i), 32.0f)) {
            bridged_i = direct_i;
        }
        if (t == 0) {
            C[idx] = make_float2(bridged_r, bridged_i);
        }
    }
}

// ---- 4b. FP64 recompute (tensor-core forms) -----------------------------------------

__global__ void recompute_fp64_kernel(int n, const float2* __restrict__ rows_a, const float2* __restrict__ rows_b,
                                      const uint32_t* __restrict__ list, const uint32_t* __restrict__ count,
                                      float2* __restrict__ C)
{
    const uint32_t total = *count;
    const int t = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const int chunk = (n + 31) / 32;
    for (uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < total; w += warps) {
        const uint32_t idx = list[w];
        const int j = (int)(idx / (uint32_t)n), i = (int)(idx - (uint32_t)j * n);
        const float2* x = rows_a + (size_t)i * n;
        const float2* y = rows_b + (size_t)j * n;
        double sr = 0.0, si = 0.0;
        const int k1 = min(n, (t + 1) * chunk);
        for (int k = t * chunk; k < k1; ++k) {
            const float2 a = x[k], b = y[k];
            sr = fma((double)a.x, (double)b.x, fma(-(double)a.y, (double)b.y, sr));
            si = fma((double)a.x, (double)b.y, fma((double)a.y, (double)b.x, si));
        }
#pragma unroll
        for (int stride = 16; stride >= 1; stride /= 2) {
            const double or_ = __shfl_down_sync(0xffffffffu, sr, stride);
            const double oi = __shfl_down_sync(0xffffffffu, si, stride);
            if (t < stride) {
                sr += or_;
                si += oi;
            }
        }
        if (t == 0) {
            C[idx] = make_float2((float)sr, (float)si);
        }
    }
}

}  // namespace

// bridge = (floor(n/128)*128^2 + (n mod 128)^2) / (18 n^2), in FP32 as the
// reference forms it (cgemm3m_rounding_kernel.cpp:96-100).
static float bridge_term(int n)
{
    const int tail = n % 128;
    volatile float a = (float)(n / 128) * (float)(128 * 128);
    volatile float b = a + (float)(tail * tail);
    volatile float d = 18.0f * (float)n;
    volatile float e = d * (float)n;
    return b / e;
}

// Layout of the rounding region (Plan::round_off): path n^2 floats | rows of
// op(A) n^2 complex | columns of op(B) n^2 complex | energies 2n floats |
// flagged list n^2 u32 | counter.
struct RoundLayout {
    float* path;
    float2* rows_a;
    float2* rows_b;
    float* energy;
    uint32_t* list;
    uint32_t* count;
};

static RoundLayout round_layout(const Plan& plan, void* ws, int n)
{
    uint8_t* b = static_cast<uint8_t*>(ws) + plan.round_off;
    const size_t nn = (size_t)n * n;
    RoundLayout L;
    size_t off = 0;
    L.path = reinterpret_cast<float*>(b + off);
    off = align_up(off + nn * 4, kRegionAlign);
    L.rows_a = reinterpret_cast<float2*>(b + off);
    off = align_up(off + nn * 8, kRegionAlign);
    L.rows_b = reinterpret_cast<float2*>(b + off);
    off = align_up(off + nn * 8, kRegionAlign);
    L.energy = reinterpret_cast<float*>(b + off);
    off = align_up(off + (size_t)2 * n * 4, kRegionAlign);
    L.list = reinterpret_cast<uint32_t*>(b + off);
    off = align_up(off + nn * 4, kRegionAlign);
    L.count = reinterpret_cast<uint32_t*>(b + off);
    return L;
}

size_t rounding_bytes(int n)
{
    const size_t nn = (size_t)n * n;
    size_t off = 0;
    off = align_up(off + nn * 4, kRegionAlign);
    off = align_up(off + nn * 8, kRegionAlign);
    off = align_up(off + nn * 8, kRegionAlign);
    off = align_up(off + (size_t)2 * n * 4, kRegionAlign);
    off = align_up(off + nn * 4, kRegionAlign);
    off = align_up(off + 256, kRegionAlign);
    return off;
}

cudaError_t launch_gemm_with_path(cudaStream_t s, const Problem& p, const Plan& plan, void* ws, int* status)
{
    const RoundLayout L = round_layout(plan, ws, p.n);
    return plan.form == CG3M_FORM_FP32 ? launch_gemm_fp32_path(s, p, plan, ws, L.path, status)
                                       : launch_gemm_tc_path(s, p, plan, ws, L.path, status);
}

cudaError_t launch_rounding(cudaStream_t s, const Problem& p, const Plan& plan, void* ws, int*, int* launched,
                            const std::function<void(int)>& mark)
{
    const int n = p.n;
    const RoundLayout L = round_layout(plan, ws, n);
    const int span = ((n + kLanes - 1) / kLanes) | 1;
    int count = 0;
    cudaError_t err = launch_pack_rows(s, p, L.rows_a, L.rows_b);
    mark(++count);
    if (err == cudaSuccess) {
        energy_kernel<<<2 * n, kLanes, (size_t)n * sizeof(float2), s>>>(L.rows_a, L.rows_b, n, span, L.energy);
        err = cudaGetLastError();
        mark(++count);
    }
    if (err == cudaSuccess) {
        err = cudaMemsetAsync(L.count, 0, sizeof(uint32_t), s);
    }
    if (err == cudaSuccess) {
        select_kernel<<<148 * 8, 256, 0, s>>>(n, static_cast<const float2*>(p.C), L.energy, L.path, bridge_term(n),
                                              L.list, L.count);
        err = cudaGetLastError();
        mark(++count);
    }
    if (err == cudaSuccess) {
        if (plan.form == CG3M_FORM_FP32) {
            recompute_fp32_kernel<<<148 * 16, 128, 0, s>>>(n, span, L.rows_a, L.rows_b, L.list, L.count,
                                                          static_cast<float2*>(p.C));
        } else {
            recompute_fp64_kernel<<<148 * 16, 128, 0, s>>>(n, L.rows_a, L.rows_b, L.list, L.count,
                                                          static_cast<float2*>(p.C));
        }
        err = cudaGetLastError();
        mark(++count);
    }
    if (launched != nullptr) {
        *launched = count;
    }
    return err;
}

}  // namespace cg3m
