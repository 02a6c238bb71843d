// Instantiations of the fused stage kernel: Upwind4/Upwind4h2 operator pairs, f64 state (reference arithmetic, built with -fmad=false).
#include "stage_dispatch.h"
#include "stage_kernel.cuh"

namespace sbp {

#define CASE(OX, OY, UPW) \
    if (opx == OX && opy == OY && upw == UPW) return reinterpret_cast<const void*>(&stage_kernel<OX, OY, double, UPW, false>);

const void* stage_ptr_f64_u4(int opx, int opy, bool upw) {
    CASE(UPWIND4, UPWIND4, true)
    CASE(UPWIND4, UPWIND4, false)
    CASE(UPWIND4H2, UPWIND4H2, true)
    CASE(UPWIND4H2, UPWIND4H2, false)
    CASE(UPWIND4, UPWIND4H2, true)
    CASE(UPWIND4, UPWIND4H2, false)
    CASE(UPWIND4H2, UPWIND4, true)
    CASE(UPWIND4H2, UPWIND4, false)
    return nullptr;
}

}  // namespace sbp
