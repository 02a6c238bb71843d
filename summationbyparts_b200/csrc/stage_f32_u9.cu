// Instantiations of the fused stage kernel: Upwind9/Upwind9h2 operator pairs, compensated f32 state.
#include "stage_dispatch.h"
#include "stage_kernel.cuh"
#include "stage_kernel_vec.cuh"

namespace sbp {

// 16-row tiles: stage_kernel; 32-row tiles: the 2 x 2 micro-tile kernel (stage_kernel_vec).
#define CASE(OX, OY, UPW, TYV)                                                        \
    if (opx == OX && opy == OY && upw == UPW && ty == 16 && TYV == 16)                \
        return reinterpret_cast<const void*>(&stage_kernel<OX, OY, float, UPW, true, 16>); \
    if (opx == OX && opy == OY && upw == UPW && ty == kVecRows && TYV == kVecRows)    \
        return vec_entry<OX, OY, UPW>(sc);

const void* stage_ptr_f32_u9(int opx, int opy, bool upw, int ty, int sc) {
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
