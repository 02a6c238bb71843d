// Instantiations of the fused stage kernel for the SBP4/SBP8 operator pairs and of the edge (SAT) kernel, compensated f32 state.
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

const void* stage_ptr_f32_sbp(int opx, int opy, bool upw, int ty, int sc) {
    CASE(SBP4, SBP4, false, 16)
    CASE(SBP4, SBP4, false, 32)
    CASE(SBP8, SBP8, false, 16)
    CASE(SBP8, SBP8, false, 32)
    return nullptr;
}

const void* sat_ptr_f32() { return reinterpret_cast<const void*>(&sat_kernel<float, true>); }
const void* eval_ptr_f32() { return reinterpret_cast<const void*>(&eval_kernel<float>); }

}  // namespace sbp
