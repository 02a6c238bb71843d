// Instantiations of the fused stage kernel: Upwind9/Upwind9h2 operator pairs, f64 state (reference arithmetic, built with -fmad=false).
#include "stage_dispatch.h"
#include "stage_kernel.cuh"

namespace sbp {

#define CASE(OX, OY, UPW) \
    if (opx == OX && opy == OY && upw == UPW) return reinterpret_cast<const void*>(&stage_kernel<OX, OY, double, UPW, false>);

const void* stage_ptr_f64_u9(int opx, int opy, bool upw) {
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
