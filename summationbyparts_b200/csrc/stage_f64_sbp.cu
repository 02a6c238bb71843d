// Instantiations of the fused stage kernel for the SBP4/SBP8 operator pairs and of the edge (SAT) kernel, f64 state (reference arithmetic, built with -fmad=false).
#include "stage_dispatch.h"
#include "stage_kernel.cuh"

namespace sbp {

#define CASE(OX, OY, UPW, TYV)                                   \
    if (opx == OX && opy == OY && upw == UPW && ty == TYV)        \
        return reinterpret_cast<const void*>(&stage_kernel<OX, OY, double, UPW, false, TYV>);

const void* stage_ptr_f64_sbp(int opx, int opy, bool upw, int ty, int sc) {
    (void)sc;  // the f64 kernels take the stage at run time
    CASE(SBP4, SBP4, false, 16)
    CASE(SBP4, SBP4, false, 32)
    CASE(SBP8, SBP8, false, 16)
    CASE(SBP8, SBP8, false, 32)
    return nullptr;
}

const void* sat_ptr_f64() { return reinterpret_cast<const void*>(&sat_kernel<double, false>); }
const void* eval_ptr_f64() { return reinterpret_cast<const void*>(&eval_kernel<double>); }

}  // namespace sbp
