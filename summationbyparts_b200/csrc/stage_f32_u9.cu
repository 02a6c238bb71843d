// Instantiations of the fused stage kernel: Upwind9/Upwind9h2 operator pairs, compensated f32 state.
#include "stage_dispatch.h"
#include "stage_kernel.cuh"

namespace sbp {

#define CASE(OX, OY, UPW) \
    if (opx == OX && opy == OY && upw == UPW) return reinterpret_cast<const void*>(&stage_kernel<OX, OY, float, UPW, true>);

const void* stage_ptr_f32_u9(int opx, int opy, bool upw) {
    CASE(UPWIND9, UPWIND9, true)
    CASE(UPWIND9, UPWIND9, false)
    CASE(UPWIND9H2, UPWIND9H2, true)
    CASE(UPWIND9H2, UPWIND9H2, false)
    CASE(UPWIND9, UPWIND9H2, true)
    CASE(UPWIND9, UPWIND9H2, false)
    CASE(UPWIND9H2, UPWIND9, true)
    CASE(UPWIND9H2, UPWIND9, false)
    return nullptr;
}

}  // namespace sbp
