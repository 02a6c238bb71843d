// Instantiations of the fused stage kernel: SBP4/SBP8 operator pairs, f64 state (reference arithmetic, built with -fmad=false).
#include "stage_dispatch.h"
#include "stage_kernel.cuh"

namespace sbp {

#define CASE(OX, OY, UPW) \
    if (opx == OX && opy == OY && upw == UPW) return reinterpret_cast<const void*>(&stage_kernel<OX, OY, double, UPW, false>);

const void* stage_ptr_f64_sbp(int opx, int opy, bool upw) {
    CASE(SBP4, SBP4, false)
    CASE(SBP8, SBP8, false)
    return nullptr;
}

}  // namespace sbp
