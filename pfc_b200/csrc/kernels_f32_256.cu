// FP32 STEP kernels specialised on the length 256 (kernels_impl.cuh: Spec, CtPlan),
// U = 1 and 2; one file per length so that the lengths compile in parallel.
#define PFCG_CT_TU 256
#include "kernels_impl.cuh"

namespace pfcg {

PFCG_CT_DECL(, 1, 256)
PFCG_CT_DECL(, 2, 256)

} // namespace pfcg
