/*
 * cg3m_aclblas.h -- the reference's aclblas* names for the cgemm3m call
 * surface, bound to this library.
 *
 * A program written against the reference's ops-blas header for
 * aclblasCgemm3m (ops-blas/include/cann_ops_blas.h:22-110,497-500,652) can
 * include this header instead and link libcg3m.so: the types are aliases of
 * the cg3m ones and the functions below are exported by the library as thin
 * wrappers of their cg3m counterparts.  The stream type becomes a CUDA stream
 * (passed as void*).  Status and op() values are this library's (the
 * reference does not ship their numeric values).
 */
#ifndef CG3M_ACLBLAS_H_
#define CG3M_ACLBLAS_H_

#include "cg3m.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef cg3mStatus_t aclblasStatus_t;
typedef cg3mOperation_t aclblasOperation_t;
typedef cg3mComplex aclblasComplex;
typedef cg3mHandle_t aclblasHandle_t;
typedef void* aclrtStream;

#define ACLBLAS_STATUS_SUCCESS CG3M_STATUS_SUCCESS
#define ACLBLAS_STATUS_HANDLE_IS_NULLPTR CG3M_STATUS_HANDLE_IS_NULLPTR
#define ACLBLAS_STATUS_INVALID_VALUE CG3M_STATUS_INVALID_VALUE
#define ACLBLAS_STATUS_INVALID_ENUM CG3M_STATUS_INVALID_ENUM
#define ACLBLAS_STATUS_ALLOC_FAILED CG3M_STATUS_ALLOC_FAILED
#define ACLBLAS_STATUS_INTERNAL_ERROR CG3M_STATUS_INTERNAL_ERROR
#define ACLBLAS_STATUS_EXECUTION_FAILED CG3M_STATUS_EXECUTION_FAILED
#define ACLBLAS_OP_N CG3M_OP_N
#define ACLBLAS_OP_T CG3M_OP_T
#define ACLBLAS_OP_C CG3M_OP_C

/* aclblasCreate, cann_ops_blas.h:46 */
aclblasStatus_t aclblasCreate(aclblasHandle_t* handle);
/* aclblasDestroy, cann_ops_blas.h:59 */
aclblasStatus_t aclblasDestroy(aclblasHandle_t handle);
/* aclblasSetStream, cann_ops_blas.h:71 */
aclblasStatus_t aclblasSetStream(aclblasHandle_t handle, aclrtStream stream);
/* aclblasGetStream, cann_ops_blas.h:81 */
aclblasStatus_t aclblasGetStream(aclblasHandle_t handle, aclrtStream* stream);
/* aclblasSetWorkspace, cann_ops_blas.h:98 */
aclblasStatus_t aclblasSetWorkspace(aclblasHandle_t handle, void* workspace, size_t workspaceSize);
/* aclblasGetVersion, cann_ops_blas.h:108 */
aclblasStatus_t aclblasGetVersion(aclblasHandle_t handle, int* version);
/* aclblasCgemm, cann_ops_blas.h:492 (definition cgemm_host.cpp:732-738) */
aclblasStatus_t aclblasCgemm(aclblasHandle_t handle, aclblasOperation_t transa, aclblasOperation_t transb, int m,
                             int n, int k, const aclblasComplex* alpha, const aclblasComplex* A, int lda,
                             const aclblasComplex* B, int ldb, const aclblasComplex* beta, aclblasComplex* C, int ldc);
/* aclblasCgemm3m, cann_ops_blas.h:497-500 (definition cgemm3m_host.cpp:17-23) */
aclblasStatus_t aclblasCgemm3m(aclblasHandle_t handle, aclblasOperation_t transa, aclblasOperation_t transb, int m,
                               int n, int k, const aclblasComplex* alpha, const aclblasComplex* A, int lda,
                               const aclblasComplex* B, int ldb, const aclblasComplex* beta, aclblasComplex* C,
                               int ldc);
/* aclblasCgemm3mStridedBatched, cann_ops_blas.h:652 */
aclblasStatus_t aclblasCgemm3mStridedBatched(aclblasHandle_t handle, aclblasOperation_t transa,
                                             aclblasOperation_t transb, int m, int n, int k,
                                             const aclblasComplex* alpha, const aclblasComplex* A, int lda,
                                             int64_t strideA, const aclblasComplex* B, int ldb, int64_t strideB,
                                             const aclblasComplex* beta, aclblasComplex* C, int ldc, int64_t strideC,
                                             int batchCount);

#ifdef __cplusplus
}
#endif

#endif /* CG3M_ACLBLAS_H_ */
