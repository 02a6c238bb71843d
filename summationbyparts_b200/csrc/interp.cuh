// Interpolation operators of 2:1 block interfaces (sbp/src/operators/interpolation*.rs) on the
// device: the tables and one output of the reference's `interpolate`
// (sbp/src/operators/interpolation.rs:15-50).  Every translation unit that includes this header
// gets its own copy of the (few kB of) tables in device memory.
#pragma once

#include <cstdint>

#include "interp_coefficients.h"

namespace sbp {

template <class T>
struct InterpDev {
    int brows, bcols, drows, dcols, jump0, jump1;
    const T* block;
    const T* diag;
};

#define SBPI_DEVICE_TABLES(P)                                                                          \
    static __device__ const double kSbpI##P##_F2C_B[] = {SBPI_##P##_F2C_BLOCK};                        \
    static __device__ const double kSbpI##P##_F2C_D[] = {SBPI_##P##_F2C_DIAG};                         \
    static __device__ const double kSbpI##P##_C2F_B[] = {SBPI_##P##_C2F_BLOCK};                        \
    static __device__ const double kSbpI##P##_C2F_D[] = {SBPI_##P##_C2F_DIAG};                         \
    static __device__ const float kSbpJ##P##_F2C_B[] = {SBPI_##P##_F2C_BLOCK_F32};                     \
    static __device__ const float kSbpJ##P##_F2C_D[] = {SBPI_##P##_F2C_DIAG_F32};                      \
    static __device__ const float kSbpJ##P##_C2F_B[] = {SBPI_##P##_C2F_BLOCK_F32};                     \
    static __device__ const float kSbpJ##P##_C2F_D[] = {SBPI_##P##_C2F_DIAG_F32};
SBPI_DEVICE_TABLES(4)
SBPI_DEVICE_TABLES(8)
SBPI_DEVICE_TABLES(9)
SBPI_DEVICE_TABLES(9H2)
#undef SBPI_DEVICE_TABLES

#define SBPI_ENTRY(K, P, D)                                                                            \
    {SBPI_##P##_##D##_BROWS, SBPI_##P##_##D##_BCOLS, SBPI_##P##_##D##_DROWS, SBPI_##P##_##D##_DCOLS,   \
     SBPI_##P##_##D##_JUMP0, SBPI_##P##_##D##_JUMP1, K##P##_##D##_B, K##P##_##D##_D}

// Operator op (sbp_interpolation) in direction fine2coarse, in the precision of T.
template <class T>
__device__ __forceinline__ InterpDev<T> interp_dev(int op, bool fine2coarse) {
    if constexpr (sizeof(T) == 8) {
        switch (op * 2 + (fine2coarse ? 1 : 0)) {
            case 0: return InterpDev<T>SBPI_ENTRY(kSbpI, 4, C2F);
            case 1: return InterpDev<T>SBPI_ENTRY(kSbpI, 4, F2C);
            case 2: return InterpDev<T>SBPI_ENTRY(kSbpI, 8, C2F);
            case 3: return InterpDev<T>SBPI_ENTRY(kSbpI, 8, F2C);
            case 4: return InterpDev<T>SBPI_ENTRY(kSbpI, 9, C2F);
            case 5: return InterpDev<T>SBPI_ENTRY(kSbpI, 9, F2C);
            case 6: return InterpDev<T>SBPI_ENTRY(kSbpI, 9H2, C2F);
            default: return InterpDev<T>SBPI_ENTRY(kSbpI, 9H2, F2C);
        }
    } else {
        switch (op * 2 + (fine2coarse ? 1 : 0)) {
            case 0: return InterpDev<T>SBPI_ENTRY(kSbpJ, 4, C2F);
            case 1: return InterpDev<T>SBPI_ENTRY(kSbpJ, 4, F2C);
            case 2: return InterpDev<T>SBPI_ENTRY(kSbpJ, 8, C2F);
            case 3: return InterpDev<T>SBPI_ENTRY(kSbpJ, 8, F2C);
            case 4: return InterpDev<T>SBPI_ENTRY(kSbpJ, 9, C2F);
            case 5: return InterpDev<T>SBPI_ENTRY(kSbpJ, 9, F2C);
            case 6: return InterpDev<T>SBPI_ENTRY(kSbpJ, 9H2, C2F);
            default: return InterpDev<T>SBPI_ENTRY(kSbpJ, 9H2, F2C);
        }
    }
}
#undef SBPI_ENTRY

// Output i of `interpolate` for nin inputs and nout outputs; in(k) returns input k.  The sum
// starts at 0 and adds in * c over every column of the row, zeros included, each product
// rounded before the add (compile with -fmad=false for the reference's rounding).
template <class T, class IN>
__device__ __forceinline__ T interp_at(const InterpDev<T>& I, int64_t i, int64_t nin, int64_t nout, IN in) {
    T t = T(0);
    if (i < I.brows) {
        for (int k = 0; k < I.bcols; ++k) t = t + in(k) * I.block[i * I.bcols + k];
    } else if (nout - i <= I.brows) {
        const int64_t row = nout - i - 1;
        const int64_t index = nin - I.bcols;
        for (int k = 0; k < I.bcols; ++k) t = t + in(index + k) * I.block[row * I.bcols + (I.bcols - k - 1)];
    } else {
        const int64_t n = i - I.brows;
        const int64_t index = I.jump0 + I.jump1 * (n / I.drows);
        const int64_t row = n % I.drows;
        for (int k = 0; k < I.dcols; ++k) t = t + in(index + k) * I.diag[row * I.dcols + k];
    }
    return t;
}

// The size relation the operator asserts: fine = 2 coarse - 1 (2 (coarse - 1) for 9h2).
__host__ __device__ inline bool interp_sizes_ok(int op, int64_t fine, int64_t coarse) {
    return op == 3 ? fine == 2 * (coarse - 1) : fine == 2 * coarse - 1;
}

struct InterpDims {
    int brows, bcols, drows, dcols, jump0, jump1;
};
#define SBPI_DIMS(P, D)                                                                                \
    InterpDims {                                                                                       \
        SBPI_##P##_##D##_BROWS, SBPI_##P##_##D##_BCOLS, SBPI_##P##_##D##_DROWS, SBPI_##P##_##D##_DCOLS, \
            SBPI_##P##_##D##_JUMP0, SBPI_##P##_##D##_JUMP1                                             \
    }
inline InterpDims interp_dims(int op, bool fine2coarse) {
    switch (op * 2 + (fine2coarse ? 1 : 0)) {
        case 0: return SBPI_DIMS(4, C2F);
        case 1: return SBPI_DIMS(4, F2C);
        case 2: return SBPI_DIMS(8, C2F);
        case 3: return SBPI_DIMS(8, F2C);
        case 4: return SBPI_DIMS(9, C2F);
        case 5: return SBPI_DIMS(9, F2C);
        case 6: return SBPI_DIMS(9H2, C2F);
        default: return SBPI_DIMS(9H2, F2C);
    }
}
#undef SBPI_DIMS

// Every input `interpolate` reads for nin inputs and nout outputs lies in [0, nin) (the reference
// would stop on an out-of-range index otherwise).
inline bool interp_reads_in_range(int op, bool fine2coarse, int64_t nin, int64_t nout) {
    const InterpDims D = interp_dims(op, fine2coarse);
    if (nin < D.bcols || nout < 1) return false;
    const int64_t interior = nout - 2 * (int64_t)D.brows;
    if (interior > 0) {
        const int64_t index = D.jump0 + D.jump1 * ((interior - 1) / D.drows);
        if (index + D.dcols > nin) return false;
    }
    return true;
}

}  // namespace sbp
