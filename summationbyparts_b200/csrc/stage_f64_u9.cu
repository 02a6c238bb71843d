// Instantiations of the fused stage kernel: Upwind9/Upwind9h2 operator pairs, f64 state (reference arithmetic, built with -fmad=false).
#include "stage_dispatch.h"
#include "stage_kernel.cuh"

namespace sbp {

#define CASE(OX, OY, UPW, TYV)                                   \
    if (opx == OX && opy == OY && upw == UPW && ty == TYV)        \
        return reinterpret_cast<const void*>(&stage_kernel<OX, OY, double, UPW, false, TYV>);

const void* stage_ptr_f64_u9(int opx, int opy, bool upw, int ty, int sc) {
    (void)sc;  // the f64 kernels take the stage at run time
    CASE(UPWIND9, UPWIND9, true, 16)
    CASE(UPWIND9, UPWIND9, true, 32)
    CASE(UPWIND9, UPWIND9, false, 16)
    CASE(UPWIND9, UPWIND9, false, 32)
    CASE(UPWIND9H2, UPWIND9H2, true, 16)
    CASE(UPWIND9H2, UPWIND9H2, true, 32)
    CASE(UPWIND9H2, UPWIND9H2, false, 16)
    CASE(UPWIND9H2, UPWIND9H2, false, 32)
    CASE(UPWIND9, UPWIND9H2, true, 16)
    CASE(UPWIND9, UPWIND9H2, true, 32)
    CASE(UPWIND9, UPWIND9H2, false, 16)
    CASE(UPWIND9, UPWIND9H2, false, 32)
    CASE(UPWIND9H2, UPWIND9, true, 16)
    CASE(UPWIND9H2, UPWIND9, true, 32)
    CASE(UPWIND9H2, UPWIND9, false, 16)
    CASE(UPWIND9H2, UPWIND9, false, 32)
    return nullptr;
}

}  // namespace sbp
