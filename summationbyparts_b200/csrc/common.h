// Host-side helpers shared by the C-ABI translation units: error strings and status plumbing.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../include/sbp_b200.h"

namespace sbp {

void set_error(const char* fmt, ...);
void clear_error();

inline sbp_status cuda_status(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return SBP_OK;
    set_error("%s: %s", what, cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation) return SBP_ERR_OUT_OF_MEMORY;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return SBP_ERR_NO_DEVICE;
    return SBP_ERR_CUDA;
}

#define SBP_TRY_CUDA(expr)                                  \
    do {                                                    \
        cudaError_t _e = (expr);                            \
        if (_e != cudaSuccess) return cuda_status(_e, #expr); \
    } while (0)

#define SBP_TRY(expr)                 \
    do {                              \
        sbp_status _s = (expr);       \
        if (_s != SBP_OK) return _s;  \
    } while (0)

// Operator shape facts used by host-side validation (mirrors OpShape<OP>).
struct OpInfo {
    int M, N, D;
    bool h2, upwind;
};
bool op_info(int op, OpInfo& out);

}  // namespace sbp
