// Lookup of the instantiated fused stage kernels (stage_*.cu).
#pragma once

namespace sbp {
// prec 0 = f64, 1 = f32 compensated; ty = tile rows (16 or 32); sc = RK stage class (0: stage 0,
// 1: stages 1 and 2, 2: stage 3), which only the compensated 32-row kernel is specialised on.
// Returns the kernel entry (a __global__ function pointer usable with cudaLaunchKernel) or
// nullptr if not built.
const void* stage_kernel_ptr(int prec, int opx, int opy, bool upw, int ty, int sc);

const void* stage_ptr_f64_u4(int opx, int opy, bool upw, int ty, int sc);
const void* stage_ptr_f64_u9(int opx, int opy, bool upw, int ty, int sc);
const void* stage_ptr_f64_sbp(int opx, int opy, bool upw, int ty, int sc);
const void* stage_ptr_f32_u4(int opx, int opy, bool upw, int ty, int sc);
const void* stage_ptr_f32_u9(int opx, int opy, bool upw, int ty, int sc);
const void* stage_ptr_f32_sbp(int opx, int opy, bool upw, int ty, int sc);
// pairs of operators from two families (stage_f64_x49a/b.cu, stage_f64_xsa/b.cu, stage_f32_x49.cu,
// stage_f32_xs.cu)
const void* stage_ptr_f64_x49a(int opx, int opy, bool upw, int ty, int sc);
const void* stage_ptr_f64_x49b(int opx, int opy, bool upw, int ty, int sc);
const void* stage_ptr_f64_xsa(int opx, int opy, bool upw, int ty, int sc);
const void* stage_ptr_f64_xsb(int opx, int opy, bool upw, int ty, int sc);
const void* stage_ptr_f32_x49(int opx, int opy, bool upw, int ty, int sc);
const void* stage_ptr_f32_xs(int opx, int opy, bool upw, int ty, int sc);
// Edge (SAT) kernel entries, one per precision.
const void* sat_ptr_f64();
const void* sat_ptr_f32();
// Expression-boundary (SBP_BC_EVAL) data kernel entries, one per precision.
const void* eval_ptr_f64();
const void* eval_ptr_f32();
}  // namespace sbp
