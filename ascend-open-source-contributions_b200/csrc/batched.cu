// batched.cu -- heterogeneous batched form.
#include "cg3m_internal.h"

extern "C" {
cg3mStatus_t cg3mBatchPlanCreate(cg3mHandle_t, const cg3mProblem*, int, int, cg3mBatchPlan_t*, int*)
{
    return CG3M_STATUS_NOT_SUPPORTED;
}
cg3mStatus_t cg3mBatchPlanExecute(cg3mHandle_t, cg3mBatchPlan_t, int) { return CG3M_STATUS_NOT_SUPPORTED; }
cg3mStatus_t cg3mBatchPlanDestroy(cg3mBatchPlan_t) { return CG3M_STATUS_NOT_SUPPORTED; }
cg3mStatus_t cg3mBatchPlanDescribe(cg3mBatchPlan_t, int*, int*, int*) { return CG3M_STATUS_NOT_SUPPORTED; }
}
