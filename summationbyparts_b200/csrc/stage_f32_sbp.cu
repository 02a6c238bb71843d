// Instantiations of the fused stage kernel: SBP4/SBP8 operator pairs, compensated f32 state.
#include "stage_dispatch.h"
#include "stage_kernel.cuh"

namespace sbp {

#define CASE(OX, OY, UPW) \
    if (opx == OX && opy == OY && upw == UPW) return reinterpret_cast<const void*>(&stage_kernel<OX, OY, float, UPW, true>);

const void* stage_ptr_f32_sbp(int opx, int opy, bool upw) {
    CASE(SBP4, SBP4, false)
    CASE(SBP8, SBP8, false)
    return nullptr;
}

}  // namespace sbp
