// Device-side SBP operators: shapes, coefficient tables in constant memory, and the
// stencil sums in the two rounding orders the reference uses.
//
//  * Row direction (diffxi/dissxi): the reference runs diff_op_1d_slice on every row
//    (sbp/src/operators/algos.rs:101-187), whose sums are matmul_float_into without fma
//    (utils/constmatrix/src/lib.rs:120-146): t = c0*p0; t = t + ck*pk; then t*idx.
//  * Column direction (diffeta/disseta): the operator on the transposed view, which the
//    reference dispatches to diff_op_2d_sliceable_y_simd (algos.rs:371-519): for columns
//    j < L*floor(nx/L) (L = 8 for f64, 16 for f32) an fma chain from zero in tap order,
//    then *idx; for the remaining columns unfused products added to 0.0.
//
// Files that need bit-identical results are compiled with -fmad=false, so the unfused
// forms below stay unfused and only __fma_rn fuses.
#pragma once

#include <cstdint>

#include "sbp_coefficients.h"

namespace sbp {

enum OpId { UPWIND4 = 0, UPWIND4H2 = 1, UPWIND9 = 2, UPWIND9H2 = 3, SBP4 = 4, SBP8 = 5 };
enum Kind { DIFF = 0, DISS = 1 };

template <int OP>
struct OpShape;
#define SBP_SHAPE(OP, TAG, H2, UPW)                                                      \
    template <>                                                                          \
    struct OpShape<OP> {                                                                 \
        static constexpr int M = SBPC_##TAG##_M, N = SBPC_##TAG##_N, D = SBPC_##TAG##_D; \
        static constexpr int H = (D - 1) / 2;                                            \
        static constexpr bool h2 = H2, upwind = UPW;                                      \
    };
SBP_SHAPE(UPWIND4, UPWIND4, false, true)
SBP_SHAPE(UPWIND4H2, UPWIND4H2, true, true)
SBP_SHAPE(UPWIND9, UPWIND9, false, true)
SBP_SHAPE(UPWIND9H2, UPWIND9H2, true, true)
SBP_SHAPE(SBP4, SBP4, false, false)
SBP_SHAPE(SBP8, SBP8, false, false)
#undef SBP_SHAPE

// Constant-memory tables (start block and interior diagonal; the end block is derived).
#define SBP_CTABLES(TAG)                                                                          \
    static __constant__ double c_##TAG##_DIFF_START_D[] = {SBPC_##TAG##_DIFF_START(SBPC_LIT_F64)}; \
    static __constant__ double c_##TAG##_DIFF_DIAG_D[] = {SBPC_##TAG##_DIFF_DIAG(SBPC_LIT_F64)};   \
    static __constant__ float c_##TAG##_DIFF_START_F[] = {SBPC_##TAG##_DIFF_START(SBPC_LIT_F32)};  \
    static __constant__ float c_##TAG##_DIFF_DIAG_F[] = {SBPC_##TAG##_DIFF_DIAG(SBPC_LIT_F32)};
#define SBP_CTABLES_DISS(TAG)                                                                     \
    static __constant__ double c_##TAG##_DISS_START_D[] = {SBPC_##TAG##_DISS_START(SBPC_LIT_F64)}; \
    static __constant__ double c_##TAG##_DISS_DIAG_D[] = {SBPC_##TAG##_DISS_DIAG(SBPC_LIT_F64)};   \
    static __constant__ float c_##TAG##_DISS_START_F[] = {SBPC_##TAG##_DISS_START(SBPC_LIT_F32)};  \
    static __constant__ float c_##TAG##_DISS_DIAG_F[] = {SBPC_##TAG##_DISS_DIAG(SBPC_LIT_F32)};
SBP_CTABLES(UPWIND4)
SBP_CTABLES(UPWIND4H2)
SBP_CTABLES(UPWIND9)
SBP_CTABLES(UPWIND9H2)
SBP_CTABLES(SBP4)
SBP_CTABLES(SBP8)
SBP_CTABLES_DISS(UPWIND4)
SBP_CTABLES_DISS(UPWIND4H2)
SBP_CTABLES_DISS(UPWIND9)
SBP_CTABLES_DISS(UPWIND9H2)
#undef SBP_CTABLES
#undef SBP_CTABLES_DISS

// Coef<OP, KIND, T>::start(i) / diag(d) read the tables; end(i) is the start block flipped in
// both axes, sign-flipped for DIFF (utils/constmatrix/src/lib.rs:302-345).
template <int OP, int KIND, class T>
struct Coef;
#define SBP_COEF(OP, TAG, KINDV, KINDN, T, SUF)                                             \
    template <>                                                                             \
    struct Coef<OP, KINDV, T> {                                                             \
        __device__ __forceinline__ static T start(int i) { return c_##TAG##_##KINDN##_START_##SUF[i]; } \
        __device__ __forceinline__ static T diag(int d) { return c_##TAG##_##KINDN##_DIAG_##SUF[d]; }   \
    };
#define SBP_COEF_ALL(OP, TAG)                       \
    SBP_COEF(OP, TAG, DIFF, DIFF, double, D)        \
    SBP_COEF(OP, TAG, DIFF, DIFF, float, F)
#define SBP_COEF_ALL_DISS(OP, TAG)                  \
    SBP_COEF(OP, TAG, DISS, DISS, double, D)        \
    SBP_COEF(OP, TAG, DISS, DISS, float, F)
SBP_COEF_ALL(UPWIND4, UPWIND4)
SBP_COEF_ALL(UPWIND4H2, UPWIND4H2)
SBP_COEF_ALL(UPWIND9, UPWIND9)
SBP_COEF_ALL(UPWIND9H2, UPWIND9H2)
SBP_COEF_ALL(SBP4, SBP4)
SBP_COEF_ALL(SBP8, SBP8)
SBP_COEF_ALL_DISS(UPWIND4, UPWIND4)
SBP_COEF_ALL_DISS(UPWIND4H2, UPWIND4H2)
SBP_COEF_ALL_DISS(UPWIND9, UPWIND9)
SBP_COEF_ALL_DISS(UPWIND9H2, UPWIND9H2)
#undef SBP_COEF
#undef SBP_COEF_ALL
#undef SBP_COEF_ALL_DISS


// The interior diagonals (v) and start-closure blocks (st, M x N by rows) in f32 as
// compile-time constants (the same literals as the constant tables): the micro-tile kernel takes
// its stencil coefficients from here, so each tap's coefficient is an immediate and the zero tap
// of a central difference is skipped.
template <int OP, int KIND>
struct CDiag;
#define SBP_CD(OP, TAG, KINDV, KINDN)                                              \
    template <>                                                                     \
    struct CDiag<OP, KINDV> {                                                       \
        static constexpr float v[] = {SBPC_##TAG##_##KINDN##_DIAG(SBPC_LIT_F32)};   \
        static constexpr float st[] = {SBPC_##TAG##_##KINDN##_START(SBPC_LIT_F32)}; \
    };
SBP_CD(UPWIND4, UPWIND4, DIFF, DIFF)
SBP_CD(UPWIND4H2, UPWIND4H2, DIFF, DIFF)
SBP_CD(UPWIND9, UPWIND9, DIFF, DIFF)
SBP_CD(UPWIND9H2, UPWIND9H2, DIFF, DIFF)
SBP_CD(SBP4, SBP4, DIFF, DIFF)
SBP_CD(SBP8, SBP8, DIFF, DIFF)
SBP_CD(UPWIND4, UPWIND4, DISS, DISS)
SBP_CD(UPWIND4H2, UPWIND4H2, DISS, DISS)
SBP_CD(UPWIND9, UPWIND9, DISS, DISS)
SBP_CD(UPWIND9H2, UPWIND9H2, DISS, DISS)
#undef SBP_CD

template <int OP, int KIND, class T>
__device__ __forceinline__ T coef_end(int i, int k) {
    constexpr int M = OpShape<OP>::M, N = OpShape<OP>::N;
    const T v = Coef<OP, KIND, T>::start((M - 1 - i) * N + (N - 1 - k));
    return KIND == DIFF ? -v : v;
}

// idx = 1 / (1 / (n-1)) (or n-2 for h2 operators), algos.rs:125-130, in the working type.
template <class T>
__host__ __device__ inline T inv_spacing(bool h2, int64_t n) {
    const T dx = h2 ? T(1) / T(n - 2) : T(1) / T(n - 1);
    return T(1) / dx;
}

// The input taps one output at index i of an n-long line reads, as [lo, hi).
template <int OP>
__host__ __device__ inline void taps_of(int i, int n, int& lo, int& hi) {
    constexpr int M = OpShape<OP>::M, N = OpShape<OP>::N, H = OpShape<OP>::H;
    if (i < M) {
        lo = 0;
        hi = N;
    } else if (i >= n - M) {
        lo = n - N;
        hi = n;
    } else {
        lo = i - H;
        hi = i + H + 1;
    }
}

// Input range [lo, hi) needed by outputs [a0, a1) of an n-long line.
template <int OP>
__host__ __device__ inline void region_of(int a0, int a1, int n, int& lo, int& hi) {
    constexpr int M = OpShape<OP>::M, N = OpShape<OP>::N, H = OpShape<OP>::H;
    lo = a0 - H;
    hi = a1 + H;
    if (a0 < M) {
        lo = 0;
        hi = hi > N ? hi : N;
    }
    if (a1 > n - M) {
        lo = lo < n - N ? lo : n - N;
        hi = n;
    }
    if (lo < 0) lo = 0;
    if (hi > n) hi = n;
}

__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// ---------------------------------------------------------------------------------------
// Sums.  `p(k)` returns the input at line position k.  Results are NOT scaled by idx.
// ---------------------------------------------------------------------------------------

// Row order: t = c0*p0; t = t + ck*pk (matmul_float_into without fma).
template <int OP, int KIND, class T, class P>
__device__ __forceinline__ T sum_unfused(int i, int n, P&& p) {
    constexpr int M = OpShape<OP>::M, N = OpShape<OP>::N, D = OpShape<OP>::D, H = OpShape<OP>::H;
    using C = Coef<OP, KIND, T>;
    T t;
    if (i < M) {
        t = C::start(i * N) * p(0);
#pragma unroll
        for (int k = 1; k < N; ++k) t = t + C::start(i * N + k) * p(k);
    } else if (i >= n - M) {
        const int r = i - (n - M), b = n - N;
        t = coef_end<OP, KIND, T>(r, 0) * p(b);
#pragma unroll
        for (int k = 1; k < N; ++k) t = t + coef_end<OP, KIND, T>(r, k) * p(b + k);
    } else {
        const int b = i - H;
        t = C::diag(0) * p(b);
#pragma unroll
        for (int d = 1; d < D; ++d) t = t + C::diag(d) * p(b + d);
    }
    return t;
}

// Interior row sum only; p(d) is the input at i - H + d.
template <int OP, int KIND, class T, class P>
__device__ __forceinline__ T diag_unfused(P&& p) {
    constexpr int D = OpShape<OP>::D;
    using C = Coef<OP, KIND, T>;
    T t = C::diag(0) * p(0);
#pragma unroll
    for (int d = 1; d < D; ++d) t = t + C::diag(d) * p(d);
    return t;
}

// Column order of the SIMD lanes: f = 0; f = fma(p_k, c_k, f).
template <int OP, int KIND, class T, class P>
__device__ __forceinline__ T sum_fused(int i, int n, P&& p) {
    constexpr int M = OpShape<OP>::M, N = OpShape<OP>::N, D = OpShape<OP>::D, H = OpShape<OP>::H;
    using C = Coef<OP, KIND, T>;
    T f = T(0);
    if (i < M) {
#pragma unroll
        for (int k = 0; k < N; ++k) f = fma_rn(p(k), C::start(i * N + k), f);
    } else if (i >= n - M) {
        const int r = i - (n - M), b = n - N;
#pragma unroll
        for (int k = 0; k < N; ++k) f = fma_rn(p(b + k), coef_end<OP, KIND, T>(r, k), f);
    } else {
        const int b = i - H;
#pragma unroll
        for (int d = 0; d < D; ++d) f = fma_rn(p(b + d), C::diag(d), f);
    }
    return f;
}

// Column order of the scalar remainder: f = 0.0; f = f + c_k*p_k.
template <int OP, int KIND, class T, class P>
__device__ __forceinline__ T sum_unfused0(int i, int n, P&& p) {
    constexpr int M = OpShape<OP>::M, N = OpShape<OP>::N, D = OpShape<OP>::D, H = OpShape<OP>::H;
    using C = Coef<OP, KIND, T>;
    T f = T(0);
    if (i < M) {
#pragma unroll
        for (int k = 0; k < N; ++k) f = f + C::start(i * N + k) * p(k);
    } else if (i >= n - M) {
        const int r = i - (n - M), b = n - N;
#pragma unroll
        for (int k = 0; k < N; ++k) f = f + coef_end<OP, KIND, T>(r, k) * p(b + k);
    } else {
        const int b = i - H;
#pragma unroll
        for (int d = 0; d < D; ++d) f = f + C::diag(d) * p(b + d);
    }
    return f;
}

// Closure rows only (i < M or i >= n - M), as rolled loops with runtime-indexed coefficients:
// the same sums in the same order as the unrolled forms above, in a fraction of the code.
// FUSED selects the fma chain from zero, otherwise t = c0*p0; t = t + ck*pk (ZERO_START = false)
// or f = 0 + ck*pk (ZERO_START = true).
template <int OP, int KIND, class T, int MODE, class P>
__device__ __noinline__ T closure_sum(int i, int n, P p) {
    constexpr int M = OpShape<OP>::M, N = OpShape<OP>::N;
    using C = Coef<OP, KIND, T>;
    const bool start = i < M;
    const int r = start ? i : i - (n - M);
    const int b = start ? 0 : n - N;
    auto coef = [&](int k) { return start ? C::start(r * N + k) : coef_end<OP, KIND, T>(r, k); };
    if (MODE == 0) {  // row order, unfused
        T t = coef(0) * p(b);
#pragma unroll 1
        for (int k = 1; k < N; ++k) t = t + coef(k) * p(b + k);
        return t;
    }
    T f = T(0);
    if (MODE == 1) {  // fused column lanes
#pragma unroll 1
        for (int k = 0; k < N; ++k) f = fma_rn(p(b + k), coef(k), f);
    } else {  // unfused column remainder
#pragma unroll 1
        for (int k = 0; k < N; ++k) f = f + coef(k) * p(b + k);
    }
    return f;
}

// Column sum with the lane split: `fused` is (column < L*floor(nx/L)).
template <int OP, int KIND, class T, class P>
__device__ __forceinline__ T sum_column(bool fused, int i, int n, P&& p) {
    return fused ? sum_fused<OP, KIND, T>(i, n, p) : sum_unfused0<OP, KIND, T>(i, n, p);
}

// Lanes of the reference's column SIMD type (f64x8 / f32x16).
template <class T>
__host__ __device__ constexpr int simd_lanes() {
    return sizeof(T) == 8 ? 8 : 16;
}

}  // namespace sbp
