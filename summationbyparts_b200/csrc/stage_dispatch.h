// Lookup of the instantiated fused stage kernels (stage_*.cu).
#pragma once

namespace sbp {
// prec 0 = f64, 1 = f32 compensated; ty = tile rows (16 or 32).  Returns the kernel entry (a
// __global__ function pointer usable with cudaLaunchKernel) or nullptr if not built.
const void* stage_kernel_ptr(int prec, int opx, int opy, bool upw, int ty);

const void* stage_ptr_f64_u4(int opx, int opy, bool upw, int ty);
const void* stage_ptr_f64_u9(int opx, int opy, bool upw, int ty);
const void* stage_ptr_f64_sbp(int opx, int opy, bool upw, int ty);
const void* stage_ptr_f32_u4(int opx, int opy, bool upw, int ty);
const void* stage_ptr_f32_u9(int opx, int opy, bool upw, int ty);
const void* stage_ptr_f32_sbp(int opx, int opy, bool upw, int ty);
// pairs of operators from two families (stage_f64_x49a/b.cu, stage_f64_xsa/b.cu, stage_f32_x49.cu,
// stage_f32_xs.cu)
const void* stage_ptr_f64_x49a(int opx, int opy, bool upw, int ty);
const void* stage_ptr_f64_x49b(int opx, int opy, bool upw, int ty);
const void* stage_ptr_f64_xsa(int opx, int opy, bool upw, int ty);
const void* stage_ptr_f64_xsb(int opx, int opy, bool upw, int ty);
const void* stage_ptr_f32_x49(int opx, int opy, bool upw, int ty);
const void* stage_ptr_f32_xs(int opx, int opy, bool upw, int ty);
// Edge (SAT) kernel entries, one per precision.
const void* sat_ptr_f64();
const void* sat_ptr_f32();
// Expression-boundary (SBP_BC_EVAL) data kernel entries, one per precision.
const void* eval_ptr_f64();
const void* eval_ptr_f32();
}  // namespace sbp
