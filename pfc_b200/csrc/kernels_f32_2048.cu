// FP32 STEP kernels specialised on the length 2048 (kernels_impl.cuh: Spec, CtPlan),
// U = 1 and 2; one file per length so that the lengths compile in parallel.
#define PFCG_CT_TU 2048
#include "kernels_impl.cuh"

namespace pfcg {

PFCG_CT_DECL(, 1, 2048)
PFCG_CT_DECL(, 2, 2048)

} // namespace pfcg
