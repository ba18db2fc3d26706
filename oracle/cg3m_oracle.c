/*
 * cg3m_oracle.c -- CPU restatement of the reference's cgemm3m algorithm.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library links, loads or
 * calls this file; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it, and only as the checker.
 *
 * Build: cc -O2 -ffp-contract=off -fno-fast-math -shared -fPIC (see build.py).
 * Every floating-point operation below is written out one rounding at a time;
 * fmaf() appears only where the modelled GPU kernel issues an FFMA.
 *
 * Contents (reference citations are paths inside ops-blas/):
 *   1. oracle_cgemm      -- reference-BLAS cgemm in FP32, loop order of Netlib
 *                           3.10.0 as the reference pins it: golden call at
 *                           test/gemm/cgemm3m/cgemm3m_golden.h:20-49 and the
 *                           ordered restatement CorrectOrderedOutput,
 *                           blas/gemm/arch35/cgemm_epilogue_kernel.cpp:130-168.
 *   2. oracle_zgemm      -- the same product in FP64 (error norms).
 *   3. oracle_cgemm3m_fp32 -- bit-exact model of this project's plain FP32 3M
 *                           path: standard 3M planes (cgemm_deinterleave_common.h
 *                           :35-46), per-partition sequential FFMA products,
 *                           fixed-order partition merge and alpha/beta epilogue
 *                           (cgemm_epilogue_kernel.cpp:247-279).
 *   3b. oracle_cgemm_modes_fp32 -- bit-exact model of the on-chip product
 *                           family (3M or four products, optional non-finite
 *                           repair, cgemm_compute_kernel.cpp:672-706).
 *   4. rounding-correction restatement: risk integral (cgemm_compute_kernel.cpp
 *      :432-474), row/column energies (cgemm3m_rounding_kernel.cpp:406-435),
 *      selection (:43-100) and segmented prefix recompute (:192-309).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OP_N 0
#define OP_T 1
#define OP_C 2
#define OP_R 3 /* conjugate without transpose (internal, autograd) */

typedef struct {
    float re, im;
} c32;
typedef struct {
    double re, im;
} c64;

#ifdef ORACLE_TIMING_BUILD
/* Timing build (the CPU baseline): the same operations in the same order.
 * -ffp-contract=off and the absence of fast-math already forbid contraction
 * and reassociation, so the compiler may only vectorise across independent
 * outputs; tests check this build's bytes against the checker's. */
static inline float fmul(float a, float b) { return a * b; }
static inline float fadd(float a, float b) { return a + b; }
static inline float fsub(float a, float b) { return a - b; }
#else
static inline float fmul(float a, float b) { volatile float r = a * b; return r; }
static inline float fadd(float a, float b) { volatile float r = a + b; return r; }
static inline float fsub(float a, float b) { volatile float r = a - b; return r; }
#endif

/* Element of op(X) at (row, col) for a column-major stored X. */
static inline c32 op_elem(const c32* x, int ld, int op, int row, int col)
{
    c32 v;
    if (op == OP_N || op == OP_R) {
        v = x[(size_t)col * ld + row];
    } else {
        v = x[(size_t)row * ld + col];
    }
    if (op == OP_C || op == OP_R) {
        v.im = -v.im;
    }
    return v;
}

/* (a.re*b.re - a.im*b.im, a.re*b.im + a.im*b.re), one rounding per operation. */
static inline c32 cmul(c32 a, c32 b)
{
    c32 r;
    r.re = fsub(fmul(a.re, b.re), fmul(a.im, b.im));
    r.im = fadd(fmul(a.re, b.im), fmul(a.im, b.re));
    return r;
}

/*
 * 1. Reference-BLAS cgemm, FP32, no contraction.
 *
 * op(A)=N (and the internal R): column j of C is first scaled by beta (zeroed
 * when beta==0, untouched when beta==1), then for each l: temp = alpha*op(B)(l,j)
 * and C(:,j) += temp*A(:,l) -- the order of CorrectOrderedOutput's normalA
 * branch (cgemm_epilogue_kernel.cpp:141-157) and of Netlib's N,x loops.
 * op(A)=T/C: temp = sum_l op(A)(i,l)*op(B)(l,j) from zero, then
 * C = alpha*temp (+ beta*C when beta != 0) -- the !normalA branch (:158-167).
 * alpha==0 or k==0 follows GoldenCgemm3m's shortcut (cgemm3m_golden.h:29-45).
 */
void oracle_cgemm(int transa, int transb, int m, int n, int k, const float* alpha2, const c32* a, int lda,
                  const c32* b, int ldb, const float* beta2, c32* c, int ldc)
{
    const c32 alpha = {alpha2[0], alpha2[1]};
    const c32 beta = {beta2[0], beta2[1]};
    const int beta_zero = beta.re == 0.0f && beta.im == 0.0f;
    const int beta_one = beta.re == 1.0f && beta.im == 0.0f;
    if (m == 0 || n == 0) {
        return;
    }
    if (k == 0 || (alpha.re == 0.0f && alpha.im == 0.0f)) {
        if (beta_one) {
            return;
        }
        for (int j = 0; j < n; ++j) {
            for (int i = 0; i < m; ++i) {
                c32* v = &c[(size_t)j * ldc + i];
                if (beta_zero) {
                    v->re = 0.0f;
                    v->im = 0.0f;
                } else {
                    *v = cmul(beta, *v);
                }
            }
        }
        return;
    }
    const int normal_a = transa == OP_N || transa == OP_R;
    if (normal_a) {
        for (int j = 0; j < n; ++j) {
            for (int i = 0; i < m; ++i) {
                c32* v = &c[(size_t)j * ldc + i];
                if (beta_zero) {
                    v->re = 0.0f;
                    v->im = 0.0f;
                } else if (!beta_one) {
                    *v = cmul(beta, *v);
                }
            }
            for (int l = 0; l < k; ++l) {
                const c32 temp = cmul(alpha, op_elem(b, ldb, transb, l, j));
                for (int i = 0; i < m; ++i) {
                    c32* v = &c[(size_t)j * ldc + i];
                    const c32 p = cmul(temp, op_elem(a, lda, transa, i, l));
                    v->re = fadd(v->re, p.re);
                    v->im = fadd(v->im, p.im);
                }
            }
        }
        return;
    }
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < m; ++i) {
            c32 temp = {0.0f, 0.0f};
            for (int l = 0; l < k; ++l) {
                const c32 p = cmul(op_elem(a, lda, transa, i, l), op_elem(b, ldb, transb, l, j));
                temp.re = fadd(temp.re, p.re);
                temp.im = fadd(temp.im, p.im);
            }
            c32* v = &c[(size_t)j * ldc + i];
            c32 out = cmul(alpha, temp);
            if (!beta_zero) {
                const c32 old = cmul(beta, *v);
                out.re = fadd(out.re, old.re);
                out.im = fadd(out.im, old.im);
            }
            *v = out;
        }
    }
}

/* 2. The same product in FP64 (inputs widened exactly), C written as FP64. */
void oracle_zgemm(int transa, int transb, int m, int n, int k, const double* alpha2, const c32* a, int lda,
                  const c32* b, int ldb, const double* beta2, const c32* c_in, int ldc, c64* c_out)
{
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < m; ++i) {
            double sr = 0.0, si = 0.0;
            for (int l = 0; l < k; ++l) {
                const c32 x = op_elem(a, lda, transa, i, l);
                const c32 y = op_elem(b, ldb, transb, l, j);
                sr += (double)x.re * y.re - (double)x.im * y.im;
                si += (double)x.re * y.im + (double)x.im * y.re;
            }
            double outr = alpha2[0] * sr - alpha2[1] * si;
            double outi = alpha2[0] * si + alpha2[1] * sr;
            if (beta2[0] != 0.0 || beta2[1] != 0.0) {
                const c32 old = c_in[(size_t)j * ldc + i];
                outr += beta2[0] * old.re - beta2[1] * old.im;
                outi += beta2[0] * old.im + beta2[1] * old.re;
            }
            c_out[(size_t)j * m + i].re = outr;
            c_out[(size_t)j * m + i].im = outi;
        }
    }
}

/*
 * 3. Bit-exact model of the plain FP32 3M path of this project.
 *
 * Planes (standard 3M, cgemm_deinterleave_common.h:35-46): ar, ai (conjugation
 * applied), sa = fl(ar+ai); likewise br, bi, sb.  Partition p covers
 * k in [p*span, min(k,(p+1)*span)); within it the three products accumulate
 * sequentially with one FFMA per term.  Per partition: re_p = P0-P1,
 * im_p = (P2-P0)-P1; partitions are summed in increasing order
 * (cgemm_epilogue_kernel.cpp:255-268).  Epilogue: alpha==1+0i and beta==0
 * store (re, im) directly (the fused-path output); otherwise
 * x = alpha*(re,im) [+ beta*C when beta != 0], one rounding per operation.
 * A k==0 / alpha==0 call is handled by the caller exactly as oracle_cgemm.
 */
void oracle_cgemm3m_fp32(int transa, int transb, int m, int n, int k, const float* alpha2, const c32* a, int lda,
                         const c32* b, int ldb, const float* beta2, c32* c, int ldc, int span)
{
    const float ar_ = alpha2[0], ai_ = alpha2[1], br_ = beta2[0], bi_ = beta2[1];
    const int unit = ar_ == 1.0f && ai_ == 0.0f && br_ == 0.0f && bi_ == 0.0f;
    const int beta_zero = br_ == 0.0f && bi_ == 0.0f;
    if (span <= 0 || span > k) {
        span = k;
    }
    /* op(A) as contiguous column-major planes (conjugation applied); the loop
     * order below only changes memory access, not any output's operation order. */
    float* xr = (float*)malloc(sizeof(float) * (size_t)m * k);
    float* xi = (float*)malloc(sizeof(float) * (size_t)m * k);
    float* xs = (float*)malloc(sizeof(float) * (size_t)m * k);
    float* p0 = (float*)malloc(sizeof(float) * (size_t)m);
    float* p1 = (float*)malloc(sizeof(float) * (size_t)m);
    float* p2 = (float*)malloc(sizeof(float) * (size_t)m);
    float* re = (float*)malloc(sizeof(float) * (size_t)m);
    float* im = (float*)malloc(sizeof(float) * (size_t)m);
    for (int l = 0; l < k; ++l) {
        for (int i = 0; i < m; ++i) {
            const c32 x = op_elem(a, lda, transa, i, l);
            xr[(size_t)l * m + i] = x.re;
            xi[(size_t)l * m + i] = x.im;
            xs[(size_t)l * m + i] = fadd(x.re, x.im);
        }
    }
    for (int j = 0; j < n; ++j) {
        for (int k0 = 0, part = 0; k0 < k; k0 += span, ++part) {
            const int k1 = k0 + span < k ? k0 + span : k;
            for (int i = 0; i < m; ++i) {
                p0[i] = 0.0f;
                p1[i] = 0.0f;
                p2[i] = 0.0f;
            }
            for (int l = k0; l < k1; ++l) {
                const c32 y = op_elem(b, ldb, transb, l, j);
                const float sb = fadd(y.re, y.im);
                const float* cr = xr + (size_t)l * m;
                const float* ci = xi + (size_t)l * m;
                const float* cs = xs + (size_t)l * m;
                for (int i = 0; i < m; ++i) {
                    p0[i] = fmaf(cr[i], y.re, p0[i]);
                    p1[i] = fmaf(ci[i], y.im, p1[i]);
                    p2[i] = fmaf(cs[i], sb, p2[i]);
                }
            }
            for (int i = 0; i < m; ++i) {
                const float rp = fsub(p0[i], p1[i]);
                const float ip = fsub(fsub(p2[i], p0[i]), p1[i]);
                if (part == 0) {
                    re[i] = rp;
                    im[i] = ip;
                } else {
                    re[i] = fadd(re[i], rp);
                    im[i] = fadd(im[i], ip);
                }
            }
        }
        for (int i = 0; i < m; ++i) {
            c32* v = &c[(size_t)j * ldc + i];
            if (unit) {
                v->re = re[i];
                v->im = im[i];
                continue;
            }
            float zr = fsub(fmul(ar_, re[i]), fmul(ai_, im[i]));
            float zi = fadd(fmul(ar_, im[i]), fmul(ai_, re[i]));
            if (!beta_zero) {
                const float cr = v->re, ci = v->im;
                zr = fadd(zr, fsub(fmul(br_, cr), fmul(bi_, ci)));
                zi = fadd(zi, fadd(fmul(br_, ci), fmul(bi_, cr)));
            }
            v->re = zr;
            v->im = zi;
        }
    }
    free(xr);
    free(xi);
    free(xs);
    free(p0);
    free(p1);
    free(p2);
    free(re);
    free(im);
}

/*
 * 3b. Bit-exact model of the on-chip product family (strided batches,
 * cgemm): mode 0 = the standard 3M identity as in 3., mode 1 = four real
 * products P0 = Ar.Br, P1 = Ai.Bi, P2 = Ar.Bi, P3 = Ai.Br accumulated with one
 * FFMA per term, re_p = P0-P1, im_p = P2+P3.  Partitions of `span` K terms
 * are merged in increasing order.  With repair != 0 a merged product with a
 * non-finite component is replaced by the explicit four-product sum of
 * RepairNonFiniteOutput (blas/gemm/arch35/cgemm_compute_kernel.cpp:672-706):
 * over the whole K, rr, ii, ri, ir rounded separately, re += rr - ii,
 * im += ri + ir.  Then the alpha/beta epilogue of 3.  Caller handles
 * k == 0 / alpha == 0 as oracle_cgemm.
 */
void oracle_cgemm_modes_fp32(int mode, int repair, int transa, int transb, int m, int n, int k, const float* alpha2,
                             const c32* a, int lda, const c32* b, int ldb, const float* beta2, c32* c, int ldc,
                             int span)
{
    const float ar_ = alpha2[0], ai_ = alpha2[1], br_ = beta2[0], bi_ = beta2[1];
    const int unit = ar_ == 1.0f && ai_ == 0.0f && br_ == 0.0f && bi_ == 0.0f;
    const int beta_zero = br_ == 0.0f && bi_ == 0.0f;
    if (span <= 0 || span > k) {
        span = k;
    }
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < m; ++i) {
            float re = 0.0f, im = 0.0f;
            for (int k0 = 0, part = 0; k0 < k; k0 += span, ++part) {
                const int k1 = k0 + span < k ? k0 + span : k;
                float q0 = 0.0f, q1 = 0.0f, q2 = 0.0f, q3 = 0.0f;
                for (int l = k0; l < k1; ++l) {
                    const c32 x = op_elem(a, lda, transa, i, l);
                    const c32 y = op_elem(b, ldb, transb, l, j);
                    if (mode == 0) {
                        q0 = fmaf(x.re, y.re, q0);
                        q1 = fmaf(x.im, y.im, q1);
                        q2 = fmaf(fadd(x.re, x.im), fadd(y.re, y.im), q2);
                    } else {
                        q0 = fmaf(x.re, y.re, q0);
                        q1 = fmaf(x.im, y.im, q1);
                        q2 = fmaf(x.re, y.im, q2);
                        q3 = fmaf(x.im, y.re, q3);
                    }
                }
                const float rp = fsub(q0, q1);
                const float ip = mode == 0 ? fsub(fsub(q2, q0), q1) : fadd(q2, q3);
                if (part == 0) {
                    re = rp;
                    im = ip;
                } else {
                    re = fadd(re, rp);
                    im = fadd(im, ip);
                }
            }
            if (repair && !(isfinite(re) && isfinite(im))) {
                re = 0.0f;
                im = 0.0f;
                for (int l = 0; l < k; ++l) {
                    const c32 x = op_elem(a, lda, transa, i, l);
                    const c32 y = op_elem(b, ldb, transb, l, j);
                    const float rr = fmul(x.re, y.re), ii = fmul(x.im, y.im);
                    const float ri = fmul(x.re, y.im), ir = fmul(x.im, y.re);
                    re = fadd(re, fsub(rr, ii));
                    im = fadd(im, fadd(ri, ir));
                }
            }
            c32* v = &c[(size_t)j * ldc + i];
            if (unit) {
                v->re = re;
                v->im = im;
                continue;
            }
            float zr = fsub(fmul(ar_, re), fmul(ai_, im));
            float zi = fadd(fmul(ar_, im), fmul(ai_, re));
            if (!beta_zero) {
                const float cr = v->re, ci = v->im;
                zr = fadd(zr, fsub(fmul(br_, cr), fmul(bi_, ci)));
                zi = fadd(zi, fadd(fmul(br_, ci), fmul(bi_, cr)));
            }
            v->re = zr;
            v->im = zi;
        }
    }
}

/* ------------------------------------------------------------------------- */
/* 4. Rounding-correction restatement.                                        */
/* ------------------------------------------------------------------------- */

/* Segment length of the risk integral: the fused kernel's K partitions at the
 * 128 tile are ceil(k / (panelDepth/2)) with panelDepth = 256, i.e. 128-term
 * segments (cgemm_host.cpp:257-260; test/gemm/cgemm3m/README.md:18). */
#define RISK_SEGMENT 128
#define LANES 64

/*
 * Risk integral per output (MergeProductsWithPath, cgemm_compute_kernel.cpp
 * :432-474).  The running complex partial sum s is sampled after each
 * RISK_SEGMENT-term segment; each segment of depth d adds
 * d/9*(s_old^2 + s_old*s_new + s_new^2) to the real and imaginary integrals,
 * and path = max(I_re, I_im).  The partial sums here are the ones the plain
 * FP32 3M model produces: per-segment products with sequential FFMA,
 * re_seg = P0-P1, im_seg = (P2-P0)-P1, running sum s += seg in FP32.
 * The multiplier d/9 is formed in FP32 as the reference does (Muls by
 * static_cast<float>(depth)/9.0f).  Output is column-major n x n (ld = n),
 * together with the unit-output C the same model yields.  This is also the
 * bit-exact model of the FP32 form's path-tracking GEMM, which accumulates
 * each 128-term segment from zero and merges segments in order exactly as
 * the reference's fused kernel does when it splits K into 128-term parts.
 */
void oracle_risk_path(int n, int transa, int transb, const c32* a, const c32* b, float* path, c32* c)
{
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < n; ++i) {
            float sr = 0.0f, si = 0.0f, ir = 0.0f, ii = 0.0f;
            for (int k0 = 0; k0 < n; k0 += RISK_SEGMENT) {
                const int k1 = k0 + RISK_SEGMENT < n ? k0 + RISK_SEGMENT : n;
                float p0 = 0.0f, p1 = 0.0f, p2 = 0.0f;
                for (int l = k0; l < k1; ++l) {
                    const c32 x = op_elem(a, n, transa, i, l);
                    const c32 y = op_elem(b, n, transb, l, j);
                    p0 = fmaf(x.re, y.re, p0);
                    p1 = fmaf(x.im, y.im, p1);
                    p2 = fmaf(fadd(x.re, x.im), fadd(y.re, y.im), p2);
                }
                const float nr = fadd(sr, fsub(p0, p1));
                const float ni = fadd(si, fsub(fsub(p2, p0), p1));
                const float w = (float)(k1 - k0) / 9.0f;
                float t = fmul(sr, sr);
                t = fmaf(sr, nr, t);
                t = fmaf(nr, nr, t);
                ir = fadd(ir, fmul(t, w));
                t = fmul(si, si);
                t = fmaf(si, ni, t);
                t = fmaf(ni, ni, t);
                ii = fadd(ii, fmul(t, w));
                sr = nr;
                si = ni;
            }
            path[(size_t)j * n + i] = ir > ii ? ir : ii;
            c[(size_t)j * n + i].re = sr;
            c[(size_t)j * n + i].im = si;
        }
    }
}

/* The same trajectory for an m x n block of outputs with full K (tests
 * compare a sub-block of a large problem): op(A) is m x k, op(B) is k x n. */
void oracle_risk_path_rect(int m, int n, int k, int transa, int transb, const c32* a, int lda, const c32* b, int ldb,
                           float* path, c32* c)
{
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < m; ++i) {
            float sr = 0.0f, si = 0.0f, ir = 0.0f, ii = 0.0f;
            for (int k0 = 0; k0 < k; k0 += RISK_SEGMENT) {
                const int k1 = k0 + RISK_SEGMENT < k ? k0 + RISK_SEGMENT : k;
                float p0 = 0.0f, p1 = 0.0f, p2 = 0.0f;
                for (int l = k0; l < k1; ++l) {
                    const c32 x = op_elem(a, lda, transa, i, l);
                    const c32 y = op_elem(b, ldb, transb, l, j);
                    p0 = fmaf(x.re, y.re, p0);
                    p1 = fmaf(x.im, y.im, p1);
                    p2 = fmaf(fadd(x.re, x.im), fadd(y.re, y.im), p2);
                }
                const float nr = fadd(sr, fsub(p0, p1));
                const float ni = fadd(si, fsub(fsub(p2, p0), p1));
                const float w = (float)(k1 - k0) / 9.0f;
                float t = fmul(sr, sr);
                t = fmaf(sr, nr, t);
                t = fmaf(nr, nr, t);
                ir = fadd(ir, fmul(t, w));
                t = fmul(si, si);
                t = fmaf(si, ni, t);
                t = fmaf(ni, ni, t);
                ii = fadd(ii, fmul(t, w));
                sr = nr;
                si = ni;
            }
            path[(size_t)j * m + i] = ir > ii ? ir : ii;
            c[(size_t)j * m + i].re = sr;
            c[(size_t)j * m + i].im = si;
        }
    }
}

/*
 * Row energies of op(A) and column energies of op(B), energy[0..n) for the rows
 * of op(A) and energy[n..2n) for the columns of op(B): sum |x|^2 over k
 * (PermuteSegments, cgemm3m_rounding_kernel.cpp:406-435).  Accumulated per lane
 * of the 64-lane segment layout (lane l holds k in [l*span, (l+1)*span)) with
 * FFMA, then the 64 lane sums are reduced pairwise (see lane_reduce).
 */
static float lane_reduce(float* v)
{
    /* Fixed pairwise tree over 64 lanes: stride 32, 16, ..., 1. */
    for (int stride = LANES / 2; stride >= 1; stride /= 2) {
        for (int l = 0; l < stride; ++l) {
            v[l] = fadd(v[l], v[l + stride]);
        }
    }
    return v[0];
}

static int segment_span(int n)
{
    return ((n + LANES - 1) / LANES) | 1; /* cgemm3m_rounding_kernel.cpp:266,488 */
}

void oracle_energy(int n, int transa, int transb, const c32* a, int lda, const c32* b, int ldb, float* energy)
{
    const int span = segment_span(n);
    float lanes[LANES];
    for (int side = 0; side < 2; ++side) {
        for (int r = 0; r < n; ++r) {
            for (int l = 0; l < LANES; ++l) {
                float e = 0.0f;
                for (int s = 0; s < span; ++s) {
                    const int kk = l * span + s;
                    if (kk >= n) {
                        break;
                    }
                    const c32 x = side == 0 ? op_elem(a, lda, transa, r, kk) : op_elem(b, ldb, transb, kk, r);
                    e = fmaf(x.re, x.re, e);
                    e = fmaf(x.im, x.im, e);
                }
                lanes[l] = e;
            }
            energy[side * n + r] = lane_reduce(lanes);
        }
    }
}

/*
 * Selection (SelectVf, cgemm3m_rounding_kernel.cpp:43-100): output (i,j) is
 * flagged when max(|Re C|,|Im C|) or the variance estimate is not finite, or
 * confidence^2 * var >= 1e-4, with
 *   var = 2^-48 * (path + E_row(i) * E_col(j) * bridge),
 *   bridge = (floor(n/128)*128^2 + (n mod 128)^2) / (18 n^2)   (:96-100).
 * Writes flags[j*n+i] in {0,1}; returns the count.
 */
static float bridge_term(int n)
{
    const int tail = n % 128;
    return ((float)(n / 128) * (float)(128 * 128) + (float)(tail * tail)) / (18.0f * (float)n * (float)n);
}

long oracle_select(int n, const c32* c, const float* energy, const float* path, float confidence, uint8_t* flags)
{
    const float bridge = bridge_term(n);
    const float scale = 0x1p-48f;
    long count = 0;
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < n; ++i) {
            const size_t idx = (size_t)j * n + i;
            const float re = fabsf(c[idx].re), im = fabsf(c[idx].im);
            const float magnitude = re > im ? re : im;
            const float variance = fmul(scale, fadd(path[idx], fmul(fmul(energy[i], energy[n + j]), bridge)));
            const int sel = !isfinite(magnitude) || !isfinite(variance) ||
                            fmul(fmul(confidence, confidence), variance) >= 0.0001f;
            flags[idx] = (uint8_t)sel;
            count += sel;
        }
    }
    return count;
}

/*
 * Segmented prefix recompute of one output (FastSegmentDot,
 * cgemm3m_rounding_kernel.cpp:264-309, with ThreeProductTerms :192-208,
 * SegmentExclusivePrefix :210-241, SelectStableSegmentSum :243-262).
 * Lane l holds k in [l*span, (l+1)*span) (zero beyond n).  Each term uses the
 * fused identity: x=ar+ai, p=x*br, q=ar*(bi-br), r=ai*(br+bi), re=p-r, im=p+q.
 * Per lane: direct sum of its terms; the lane sums are scanned (Hillis-Steele,
 * distances 1..32) to give each lane an exclusive prefix; each lane replays
 * its terms starting from that prefix and subtracts it afterwards; the 64
 * replayed lane values are reduced.  If max|inclusive prefix| >= 32*|direct|
 * the direct reduction is kept instead.  Lane reductions use lane_reduce's
 * fixed pairwise order.
 */
static void recompute_one(int n, const c32* arow, const c32* bcol, float* out_re, float* out_im)
{
    const int span = segment_span(n);
    float sum_r[LANES], sum_i[LANES], tr[LANES], ti[LANES];
    for (int l = 0; l < LANES; ++l) {
        float r = 0.0f, im = 0.0f;
        for (int s = 0; s < span; ++s) {
            const int kk = l * span + s;
            if (kk >= n) {
                break;
            }
            const c32 x = arow[kk], y = bcol[kk];
            const float p = fmul(fadd(x.re, x.im), y.re);
            const float q = fmul(x.re, fsub(y.im, y.re));
            const float rr = fmul(x.im, fadd(y.re, y.im));
            r = fadd(r, fsub(p, rr));
            im = fadd(im, fadd(p, q));
        }
        sum_r[l] = r;
        sum_i[l] = im;
    }
    memcpy(tr, sum_r, sizeof tr);
    memcpy(ti, sum_i, sizeof ti);
    const float direct_r = lane_reduce(tr);
    const float direct_i = lane_reduce(ti);
    /* Inclusive Hillis-Steele scan in place (every step reads the previous step). */
    for (int d = 1; d < LANES; d *= 2) {
        float nr[LANES], ni[LANES];
        for (int l = 0; l < LANES; ++l) {
            nr[l] = l >= d ? fadd(sum_r[l], sum_r[l - d]) : sum_r[l];
            ni[l] = l >= d ? fadd(sum_i[l], sum_i[l - d]) : sum_i[l];
        }
        memcpy(sum_r, nr, sizeof nr);
        memcpy(sum_i, ni, sizeof ni);
    }
    float fr[LANES], fi[LANES];
    float max_r = 0.0f, max_i = 0.0f;
    for (int l = 0; l < LANES; ++l) {
        const float init_r = l >= 1 ? sum_r[l - 1] : 0.0f;
        const float init_i = l >= 1 ? sum_i[l - 1] : 0.0f;
        float r = fadd(init_r, 0.0f), im = fadd(init_i, 0.0f);
        for (int s = 0; s < span; ++s) {
            const int kk = l * span + s;
            if (kk >= n) {
                break;
            }
            const c32 x = arow[kk], y = bcol[kk];
            const float p = fmul(fadd(x.re, x.im), y.re);
            const float q = fmul(x.re, fsub(y.im, y.re));
            const float rr = fmul(x.im, fadd(y.re, y.im));
            r = fadd(r, fsub(p, rr));
            im = fadd(im, fadd(p, q));
        }
        fr[l] = fsub(r, init_r);
        fi[l] = fsub(im, init_i);
        const float ar = fabsf(sum_r[l]), ai = fabsf(sum_i[l]);
        max_r = ar > max_r ? ar : max_r;
        max_i = ai > max_i ? ai : max_i;
    }
    float bridged_r = lane_reduce(fr);
    float bridged_i = lane_reduce(fi);
    if (max_r >= fmul(fabsf(direct_r), 32.0f)) {
        bridged_r = direct_r;
    }
    if (max_i >= fmul(fabsf(direct_i), 32.0f)) {
        bridged_i = direct_i;
    }
    *out_re = bridged_r;
    *out_im = bridged_i;
}

/*
 * Recompute every flagged output of a square unit-output problem in place.
 * op(A) rows and op(B) columns are gathered contiguously first (the
 * reference's pack/permute kernels, cgemm3m_rounding_kernel.cpp:148-190,437-472).
 */
void oracle_recompute(int n, int transa, int transb, const c32* a, int lda, const c32* b, int ldb,
                      const uint8_t* flags, c32* c)
{
    c32* arow = (c32*)malloc(sizeof(c32) * (size_t)n);
    c32* bcol = (c32*)malloc(sizeof(c32) * (size_t)n);
    int cached_i = -1;
    for (int j = 0; j < n; ++j) {
        for (int kk = 0; kk < n; ++kk) {
            bcol[kk] = op_elem(b, ldb, transb, kk, j);
        }
        for (int i = 0; i < n; ++i) {
            const size_t idx = (size_t)j * n + i;
            if (!flags[idx]) {
                continue;
            }
            if (cached_i != i) {
                for (int kk = 0; kk < n; ++kk) {
                    arow[kk] = op_elem(a, lda, transa, i, kk);
                }
                cached_i = i;
            }
            recompute_one(n, arow, bcol, &c[idx].re, &c[idx].im);
        }
        cached_i = -1;
    }
    free(arow);
    free(bcol);
}

/* Single-output recompute on explicit op(A) row / op(B) column vectors (tests). */
void oracle_recompute_dot(int n, const c32* arow, const c32* bcol, float* out2)
{
    recompute_one(n, arow, bcol, &out2[0], &out2[1]);
}

float oracle_bridge(int n) { return bridge_term(n); }
int oracle_segment_span(int n) { return segment_span(n); }
