// Instantiations of the fused stage kernel for operator pairs of two families: an Upwind4-family operator in one direction and an Upwind9-family operator in the other;
// compensated f32 state.  The reference composes any (eta, xi) pair of its six operators
// (sbp/src/operators.rs:115-150, multigrid/src/parsing.rs:153-164); the upwind form needs an
// upwind operator in both directions, every other pair runs RHS_trad.
#include "stage_dispatch.h"
#include "stage_kernel.cuh"
#include "stage_kernel_vec.cuh"

namespace sbp {

// 16-row tiles: stage_kernel; 32-row tiles: the 2 x 2 micro-tile kernel.
#define CASE(OX, OY, UPW)                                                                          \
    if (opx == OX && opy == OY && upw == UPW) {                                                     \
        if (ty == 16) return reinterpret_cast<const void*>(&stage_kernel<OX, OY, float, UPW, true, 16>); \
        if (ty == kVecRows) return vec_entry<OX, OY, UPW>(sc);   \
    }

const void* stage_ptr_f32_x49(int opx, int opy, bool upw, int ty, int sc) {
    CASE(UPWIND4, UPWIND9, true)
    CASE(UPWIND4, UPWIND9, false)
    CASE(UPWIND4, UPWIND9H2, true)
    CASE(UPWIND4, UPWIND9H2, false)
    CASE(UPWIND4H2, UPWIND9, true)
    CASE(UPWIND4H2, UPWIND9, false)
    CASE(UPWIND4H2, UPWIND9H2, true)
    CASE(UPWIND4H2, UPWIND9H2, false)
    CASE(UPWIND9, UPWIND4, true)
    CASE(UPWIND9, UPWIND4, false)
    CASE(UPWIND9, UPWIND4H2, true)
    CASE(UPWIND9, UPWIND4H2, false)
    CASE(UPWIND9H2, UPWIND4, true)
    CASE(UPWIND9H2, UPWIND4, false)
    CASE(UPWIND9H2, UPWIND4H2, true)
    CASE(UPWIND9H2, UPWIND4H2, false)
    return nullptr;
}

}  // namespace sbp
