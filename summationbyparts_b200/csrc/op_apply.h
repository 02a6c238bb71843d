// Launchers of the standalone operator kernels (op_apply.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace sbp {
// dir 0 = xi (rows), 1 = eta (columns); kind 0 = DIFF, 1 = DISS; dtype 0 = f64, 1 = f32.
// Arrays are nbatch (ny, nx) C-order planes spaced bstride elements apart.
cudaError_t op_apply(int op, int dir, int kind, int dtype, const void* in, void* out, int64_t ny, int64_t nx,
                     int64_t nbatch, int64_t bstride, cudaStream_t st);
}  // namespace sbp
