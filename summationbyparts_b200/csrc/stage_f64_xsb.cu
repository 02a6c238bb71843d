// Instantiations of the fused stage kernel for operator pairs of two families: an SBP4/SBP8 xi operator with an upwind eta operator, and SBP8 xi with SBP4 eta;
// f64 state (reference arithmetic, built with -fmad=false).  The reference composes any (eta, xi)
// pair of its six operators (sbp/src/operators.rs:115-150, multigrid/src/parsing.rs:153-164); the
// upwind form needs an upwind operator in both directions, every other pair runs RHS_trad.
#include "stage_dispatch.h"
#include "stage_kernel.cuh"

namespace sbp {

#define CASE(OX, OY, UPW)                                                                           \
    if (opx == OX && opy == OY && upw == UPW) {                                                      \
        if (ty == 16) return reinterpret_cast<const void*>(&stage_kernel<OX, OY, double, UPW, false, 16>); \
        if (ty == 32) return reinterpret_cast<const void*>(&stage_kernel<OX, OY, double, UPW, false, 32>); \
    }

const void* stage_ptr_f64_xsb(int opx, int opy, bool upw, int ty, int sc) {
    (void)sc;  // the f64 kernels take the stage at run time
    CASE(SBP4, UPWIND4, false)
    CASE(SBP4, UPWIND4H2, false)
    CASE(SBP4, UPWIND9, false)
    CASE(SBP4, UPWIND9H2, false)
    CASE(SBP8, UPWIND4, false)
    CASE(SBP8, UPWIND4H2, false)
    CASE(SBP8, UPWIND9, false)
    CASE(SBP8, UPWIND9H2, false)
    CASE(SBP8, SBP4, false)
    return nullptr;
}

}  // namespace sbp
