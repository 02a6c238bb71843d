// Standalone SBP operator application: SbpOperator2d::diffxi/diffeta and
// UpwindOperator2d::dissxi/disseta on device arrays (sbp/src/operators.rs:55-106).
// Compiled with -fmad=false: results are bit-identical to the reference's row path
// (xi) and column path (eta) in the same dtype.
//
// Aligned arrays (rows and batch stride multiples of 16 bytes, 16-byte aligned base pointers)
// take the bulk-staged kernels: one tile per CTA, every input row segment of the tile (with its
// halo or closure region) brought into shared memory by one cp.async.bulk copy that completes
// on an mbarrier, so a CTA has its whole tile in flight at once and no thread spends
// instructions on the loads.  Row tiles: kXiBulkRows rows x 128 vectors of 16 bytes (256 f64 or
// 512 f32 outputs per row), each thread one 16-byte output vector per row.  Column tiles:
// kEtaBulkRows rows x 1 KB of adjacent columns, each thread one column over its share of the
// rows with the D-tap window in a register ring.  Other arrays take the kernels below.
//
// Row direction: a CTA stages kXiRows row segments (plus halo) in shared memory, with 16-byte
// loads when the rows are 16-byte aligned; each thread
// then reads its window with 16-byte vector loads and produces 16/sizeof(T) consecutive
// outputs (2 f64 or 4 f32) per row, stored as one 16-byte vector.  Boundary-closure outputs
// (first/last M of the row) read global memory directly.
//
// Column direction: one thread per 16 bytes of adjacent columns (2 f64 or 4 f32; one column
// where the rows are not 16-byte aligned) marches down a chunk of rows with the D-tap windows
// of its columns held in registers (fully unrolled ring, so no register moves), every row one
// 16-byte load and one 16-byte store coalesced across the warp; rows inside the boundary
// closures use the M x N blocks.  The reference's fused / unfused column split falls on a
// multiple of 8 (f64) or 16 (f32) columns, so a thread's columns are all on the same side.
#include <cuda_runtime.h>

#include <cstdint>

#include "bulk_copy.cuh"
#include "op_apply.h"
#include "sbp_ops.cuh"

namespace sbp {

namespace {

constexpr int kThreads = 256;
constexpr int kEtaRows = 64;  // rows per column chunk: enough CTAs for even waves on 4096^2 fields
constexpr int kXiRows = 1;

template <class T>
struct Vec;
template <>
struct Vec<double> {
    using type = double2;
};
template <>
struct Vec<float> {
    using type = float4;
};

template <int OP, int KIND, class T>
__global__ void __launch_bounds__(kThreads)
    op_xi_kernel(const T* __restrict__ in, T* __restrict__ out, int ny, int nx, int64_t nbatch, int64_t bstride,
                 T idx, bool vec_ok) {
    constexpr int M = OpShape<OP>::M, H = OpShape<OP>::H;
    constexpr int K = 16 / sizeof(T);           // outputs per thread
    constexpr int PAD = ((H + K - 1) / K) * K;  // left/right halo, multiple of the vector width
    constexpr int SEG = kThreads * K;
    constexpr int NV = (K + 2 * PAD) / K;  // vectors in one thread's window
    constexpr int BW = SEG + 2 * PAD;      // buffer width of one row
    using V = typename Vec<T>::type;
    __shared__ __align__(16) T buf[kXiRows * BW];

    const int nseg = (nx + SEG - 1) / SEG;
    const int nrg = (ny + kXiRows - 1) / kXiRows;
    const int64_t items = nbatch * (int64_t)nrg * nseg;
    for (int64_t it = blockIdx.x; it < items; it += gridDim.x) {
        const int seg = (int)(it % nseg);
        const int64_t rr = it / nseg;
        const int row0 = (int)(rr % nrg) * kXiRows;
        const int64_t b = rr / nrg;
        const int nrows = min(kXiRows, ny - row0);
        const int s0 = seg * SEG;
        const int base = s0 - PAD;  // column of buf[row][0]
        const int c_lo = base < 0 ? 0 : base;
        const int c_hi = min(nx, s0 + SEG + PAD);
        // every load of the kXiRows rows is issued before the barrier
        for (int r = 0; r < nrows; ++r) {
            const T* src = in + b * bstride + (int64_t)(row0 + r) * nx;
            T* bb = buf + r * BW;
            if (vec_ok) {
                // c_lo and c_hi are multiples of K (or nx, itself a multiple of K)
                for (int c = c_lo + K * threadIdx.x; c < c_hi; c += K * kThreads)
                    *reinterpret_cast<V*>(bb + c - base) = __ldg(reinterpret_cast<const V*>(src + c));
            } else {
                for (int c = c_lo + threadIdx.x; c < c_hi; c += kThreads) bb[c - base] = __ldg(src + c);
            }
        }
        __syncthreads();

        const int c0 = s0 + K * threadIdx.x;
        for (int r = 0; r < nrows && c0 < nx; ++r) {
            const T* src = in + b * bstride + (int64_t)(row0 + r) * nx;
            T* dst = out + b * bstride + (int64_t)(row0 + r) * nx;
            const T* rbuf = buf + r * BW;
            T o[K];
            const bool interior = c0 >= M && c0 + K - 1 < nx - M;
            if (interior) {
                T w[K + 2 * PAD];
                const V* bv = reinterpret_cast<const V*>(rbuf + K * threadIdx.x);
#pragma unroll
                for (int v = 0; v < NV; ++v) reinterpret_cast<V*>(w)[v] = bv[v];
                // w[j] holds column c0 - PAD + j
#pragma unroll
                for (int j = 0; j < K; ++j)
                    o[j] = diag_unfused<OP, KIND, T>([&](int d) { return w[j + d + PAD - H]; }) * idx;
            } else {
#pragma unroll
                for (int j = 0; j < K; ++j)
                    if (c0 + j < nx)
                        o[j] = sum_unfused<OP, KIND, T>(c0 + j, nx, [&](int kk) { return __ldg(src + kk); }) * idx;
            }
            if (vec_ok && c0 + K <= nx) {
                *reinterpret_cast<V*>(dst + c0) = *reinterpret_cast<V*>(o);
            } else {
#pragma unroll
                for (int j = 0; j < K; ++j)
                    if (c0 + j < nx) dst[c0 + j] = o[j];
            }
        }
        __syncthreads();
    }
}

template <int OP, int KIND, class T>
__global__ void __launch_bounds__(kThreads)
    op_eta_kernel(const T* __restrict__ in, T* __restrict__ out, int ny, int nx, int64_t nbatch, int64_t bstride,
                  T idx, int simd) {
    constexpr int M = OpShape<OP>::M, D = OpShape<OP>::D, H = OpShape<OP>::H;
    const int ncb = (nx + kThreads - 1) / kThreads;
    const int nrc = (ny + kEtaRows - 1) / kEtaRows;
    const int64_t items = nbatch * (int64_t)ncb * nrc;
    for (int64_t it = blockIdx.x; it < items; it += gridDim.x) {
        const int cb = (int)(it % ncb);
        const int64_t r1_ = it / ncb;
        const int rc = (int)(r1_ % nrc);
        const int64_t b = r1_ / nrc;
        const int col = cb * kThreads + threadIdx.x;
        if (col >= nx) continue;
        const T* src = in + b * bstride + col;
        T* dst = out + b * bstride + col;
        const bool fused = col < simd;
        const int y0 = rc * kEtaRows, y1 = min(ny, y0 + kEtaRows);
        auto at = [&](int r) { return __ldg(src + (int64_t)r * nx); };
        // closure rows in this chunk
        for (int r = y0; r < y1 && r < M; ++r) dst[(int64_t)r * nx] = sum_column<OP, KIND, T>(fused, r, ny, at) * idx;
        for (int r = max(y0, ny - M); r < y1; ++r)
            dst[(int64_t)r * nx] = sum_column<OP, KIND, T>(fused, r, ny, at) * idx;
        // interior rows: register ring
        const int i0 = max(y0, M), i1 = min(y1, ny - M);
        if (i0 >= i1) continue;
        T w[D];
#pragma unroll
        for (int k = 0; k < D - 1; ++k) w[k] = at(i0 - H + k);
        int r = i0;
        for (; r + D <= i1; r += D) {
#pragma unroll
            for (int u = 0; u < D; ++u) {
                w[(u + D - 1) % D] = at(r + u + H);
                T f = T(0);
                if (fused) {
#pragma unroll
                    for (int k = 0; k < D; ++k) f = fma_rn(w[(u + k) % D], Coef<OP, KIND, T>::diag(k), f);
                } else {
#pragma unroll
                    for (int k = 0; k < D; ++k) f = f + Coef<OP, KIND, T>::diag(k) * w[(u + k) % D];
                }
                dst[(int64_t)(r + u) * nx] = f * idx;
            }
        }
        for (; r < i1; ++r) dst[(int64_t)r * nx] = sum_column<OP, KIND, T>(fused, r, ny, at) * idx;
    }
}

// Column direction, K = 16 / sizeof(T) adjacent columns per thread (see the file comment).
// Requires nx and bstride multiples of K and 16-byte aligned arrays.
template <int OP, int KIND, class T>
__global__ void __launch_bounds__(kThreads)
    op_eta_vec_kernel(const T* __restrict__ in, T* __restrict__ out, int ny, int nx, int64_t nbatch, int64_t bstride,
                      T idx, int simd) {
    constexpr int M = OpShape<OP>::M, D = OpShape<OP>::D, H = OpShape<OP>::H;
    constexpr int K = 16 / sizeof(T);
    using V = typename Vec<T>::type;
    const int ngroups = nx / K;
    const int ncb = (ngroups + kThreads - 1) / kThreads;
    const int nrc = (ny + kEtaRows - 1) / kEtaRows;
    const int64_t items = nbatch * (int64_t)ncb * nrc;
    for (int64_t it = blockIdx.x; it < items; it += gridDim.x) {
        const int cb = (int)(it % ncb);
        const int64_t r1_ = it / ncb;
        const int rc = (int)(r1_ % nrc);
        const int64_t b = r1_ / nrc;
        const int grp = cb * kThreads + threadIdx.x;
        if (grp >= ngroups) continue;
        const int col0 = grp * K;
        const T* src = in + b * bstride + col0;
        T* dst = out + b * bstride + col0;
        const bool fused = col0 < simd;  // simd is a multiple of K: all K columns agree
        const int y0 = rc * kEtaRows, y1 = min(ny, y0 + kEtaRows);
        auto row_vec = [&](int r) { return __ldg(reinterpret_cast<const V*>(src + (int64_t)r * nx)); };
        auto closure_row = [&](int r) {
            T o[K];
#pragma unroll
            for (int j = 0; j < K; ++j)
                o[j] = sum_column<OP, KIND, T>(fused, r, ny, [&](int rr) { return __ldg(src + (int64_t)rr * nx + j); }) *
                       idx;
            *reinterpret_cast<V*>(dst + (int64_t)r * nx) = *reinterpret_cast<V*>(o);
        };
        for (int r = y0; r < y1 && r < M; ++r) closure_row(r);
        for (int r = max(y0, ny - M); r < y1; ++r) closure_row(r);
        const int i0 = max(y0, M), i1 = min(y1, ny - M);
        if (i0 >= i1) continue;
        V w[D];
#pragma unroll
        for (int k = 0; k < D - 1; ++k) w[k] = row_vec(i0 - H + k);
        int r = i0;
        for (; r + D <= i1; r += D) {
#pragma unroll
            for (int u = 0; u < D; ++u) {
                w[(u + D - 1) % D] = row_vec(r + u + H);
                T o[K];
#pragma unroll
                for (int j = 0; j < K; ++j) {
                    T f = T(0);
                    if (fused) {
#pragma unroll
                        for (int k = 0; k < D; ++k)
                            f = fma_rn(reinterpret_cast<const T*>(&w[(u + k) % D])[j], Coef<OP, KIND, T>::diag(k), f);
                    } else {
#pragma unroll
                        for (int k = 0; k < D; ++k)
                            f = f + Coef<OP, KIND, T>::diag(k) * reinterpret_cast<const T*>(&w[(u + k) % D])[j];
                    }
                    o[j] = f * idx;
                }
                *reinterpret_cast<V*>(dst + (int64_t)(r + u) * nx) = *reinterpret_cast<V*>(o);
            }
        }
        for (; r < i1; ++r) closure_row(r);
    }
}

constexpr int kBulkWait = 1 << 22;  // mbarrier polls before a tile gives up
// Tiles whose staged rows did not arrive within kBulkWait polls; their outputs are not written.
__device__ unsigned g_bulk_timeouts = 0;

constexpr int kXiBulkRows = 16;
template <class T>
constexpr int xi_bulk_cols() { return 128 * (16 / (int)sizeof(T)); }
template <class T>
constexpr int xi_bulk_pitch() { return xi_bulk_cols<T>() + 32; }  // covers the halo, closures and alignment
template <class T>
constexpr size_t xi_bulk_smem() { return (size_t)kXiBulkRows * xi_bulk_pitch<T>() * sizeof(T) + 16; }

// Row direction, bulk-staged tile (see the file comment).  Requires nx and bstride multiples of
// K = 16 / sizeof(T) and 16-byte aligned arrays.
template <int OP, int KIND, class T>
__global__ void __launch_bounds__(kThreads)
    op_xi_bulk_kernel(const T* __restrict__ in, T* __restrict__ out, int ny, int nx, int64_t bstride, T idx) {
    constexpr int M = OpShape<OP>::M, H = OpShape<OP>::H;
    constexpr int K = 16 / sizeof(T);
    constexpr int TC = xi_bulk_cols<T>(), P = xi_bulk_pitch<T>(), TR = kXiBulkRows;
    constexpr int PAD = ((H + K - 1) / K) * K;
    constexpr int NV = (K + 2 * PAD) / K;
    using V = typename Vec<T>::type;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    T* buf = reinterpret_cast<T*>(smem_raw);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + (size_t)TR * P * sizeof(T));
    const int ncb = (nx + TC - 1) / TC, nrg = (ny + TR - 1) / TR;
    int64_t it = blockIdx.x;
    const int cb = (int)(it % ncb);
    it /= ncb;
    const int rg = (int)(it % nrg);
    const int64_t b = it / nrg;
    const int c0 = cb * TC, c1 = min(nx, c0 + TC);
    const int y0 = rg * TR, nrows = min(TR, ny - y0);
    int lo, hi;
    region_of<OP>(c0, c1, nx, lo, hi);
    lo -= lo % K;                              // 16-byte aligned segment start
    hi = min(nx, (hi + K - 1) / K * K);        // and a whole number of 16-byte vectors
    const uint32_t row_bytes = (uint32_t)(hi - lo) * (uint32_t)sizeof(T);
    const T* src = in + b * bstride + (int64_t)y0 * nx + lo;
    if (threadIdx.x == 0) bulk_mbar_init(bar, 1);
    __syncthreads();
    if (threadIdx.x < 32) {
        if (threadIdx.x == 0) bulk_expect(bar, row_bytes * (uint32_t)nrows);
        for (int r = threadIdx.x; r < nrows; r += 32) bulk_g2s(buf + r * P, src + (int64_t)r * nx, row_bytes, bar);
    }
    if (!bulk_wait(bar, 0, kBulkWait)) {
        if (threadIdx.x == 0) atomicAdd(&g_bulk_timeouts, 1u);
        return;
    }
    const int sub = threadIdx.x / 128, v = threadIdx.x % 128;
    const int c = c0 + K * v;  // first of this thread's K outputs; buf column 0 is input column lo
    if (c >= c1) return;
    const bool interior = c >= M && c + K - 1 < nx - M;
    for (int r = sub; r < nrows; r += 2) {
        const T* rb = buf + r * P;
        T* dst = out + b * bstride + (int64_t)(y0 + r) * nx;
        T o[K];
        if (interior) {
            T w[K + 2 * PAD];  // w[j] holds column c - PAD + j
            const V* bv = reinterpret_cast<const V*>(rb + (c - PAD - lo));
#pragma unroll
            for (int q = 0; q < NV; ++q) reinterpret_cast<V*>(w)[q] = bv[q];
#pragma unroll
            for (int j = 0; j < K; ++j)
                o[j] = diag_unfused<OP, KIND, T>([&](int d) { return w[j + d + PAD - H]; }) * idx;
        } else {
#pragma unroll
            for (int j = 0; j < K; ++j)
                o[j] = sum_unfused<OP, KIND, T>(c + j, nx, [&](int kk) { return rb[kk - lo]; }) * idx;
        }
        *reinterpret_cast<V*>(dst + c) = *reinterpret_cast<V*>(o);
    }
}

constexpr int kEtaBulkRows = 48;
template <int OP, class T>
constexpr int eta_bulk_region() {  // input rows a column tile can need (region_of's extent)
    constexpr int M = OpShape<OP>::M, N = OpShape<OP>::N, H = OpShape<OP>::H;
    constexpr int a = kEtaBulkRows + H + (H > M - 1 ? H : M - 1);
    return a > N ? a : N;
}
template <int OP, class T>
constexpr size_t eta_bulk_smem() { return (size_t)eta_bulk_region<OP, T>() * 1024 + 16; }

// Column direction, bulk-staged tile (see the file comment).  Same requirements as the row tile.
template <int OP, int KIND, class T>
__global__ void __launch_bounds__(kThreads)
    op_eta_bulk_kernel(const T* __restrict__ in, T* __restrict__ out, int ny, int nx, int64_t bstride, T idx,
                       int simd) {
    constexpr int M = OpShape<OP>::M, D = OpShape<OP>::D, H = OpShape<OP>::H;
    constexpr int TC = 1024 / sizeof(T), TR = kEtaBulkRows;
    constexpr int GROUPS = kThreads / TC;  // row groups (2 in f64, 1 in f32)
    constexpr int RG = TR / GROUPS;        // rows of one thread
    extern __shared__ __align__(128) unsigned char smem_raw[];
    T* buf = reinterpret_cast<T*>(smem_raw);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + (size_t)eta_bulk_region<OP, T>() * 1024);
    const int ncb = (nx + TC - 1) / TC, nrc = (ny + TR - 1) / TR;
    int64_t it = blockIdx.x;  // vertically adjacent tiles are adjacent in launch order (shared halos in L2)
    const int rc = (int)(it % nrc);
    it /= nrc;
    const int cb = (int)(it % ncb);
    const int64_t b = it / ncb;
    const int y0 = rc * TR, y1 = min(ny, y0 + TR), c0 = cb * TC, tw = min(TC, nx - c0);
    int lo, hi;
    region_of<OP>(y0, y1, ny, lo, hi);
    const int nrows = hi - lo;
    const uint32_t row_bytes = (uint32_t)tw * (uint32_t)sizeof(T);
    const T* src = in + b * bstride + (int64_t)lo * nx + c0;
    if (threadIdx.x == 0) bulk_mbar_init(bar, 1);
    __syncthreads();
    if (threadIdx.x < 32) {
        if (threadIdx.x == 0) bulk_expect(bar, row_bytes * (uint32_t)nrows);
        for (int r = threadIdx.x; r < nrows; r += 32) bulk_g2s(buf + r * TC, src + (int64_t)r * nx, row_bytes, bar);
    }
    if (!bulk_wait(bar, 0, kBulkWait)) {
        if (threadIdx.x == 0) atomicAdd(&g_bulk_timeouts, 1u);
        return;
    }
    const int j = threadIdx.x % TC, g = threadIdx.x / TC;
    if (j >= tw) return;
    const int col = c0 + j;
    const bool fused = col < simd;
    T* dst = out + b * bstride + col;
    auto at = [&](int r) { return buf[(r - lo) * TC + j]; };
    const int ra = y0 + g * RG, rb = min(y1, ra + RG);
    for (int r = ra; r < rb && r < M; ++r) dst[(int64_t)r * nx] = sum_column<OP, KIND, T>(fused, r, ny, at) * idx;
    for (int r = max(ra, ny - M); r < rb; ++r) dst[(int64_t)r * nx] = sum_column<OP, KIND, T>(fused, r, ny, at) * idx;
    const int i0 = max(ra, M), i1 = min(rb, ny - M);
    if (i0 >= i1) return;
    T w[D];
#pragma unroll
    for (int k = 0; k < D - 1; ++k) w[k] = at(i0 - H + k);
    int r = i0;
    for (; r + D <= i1; r += D) {
#pragma unroll
        for (int u = 0; u < D; ++u) {
            w[(u + D - 1) % D] = at(r + u + H);
            T f = T(0);
            if (fused) {
#pragma unroll
                for (int k = 0; k < D; ++k) f = fma_rn(w[(u + k) % D], Coef<OP, KIND, T>::diag(k), f);
            } else {
#pragma unroll
                for (int k = 0; k < D; ++k) f = f + Coef<OP, KIND, T>::diag(k) * w[(u + k) % D];
            }
            dst[(int64_t)(r + u) * nx] = f * idx;
        }
    }
    for (; r < i1; ++r) dst[(int64_t)r * nx] = sum_column<OP, KIND, T>(fused, r, ny, at) * idx;
}

int g_num_sms = 0;

int num_sms() {
    if (g_num_sms == 0) {
        int dev = 0, n = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        g_num_sms = n;
    }
    return g_num_sms;
}

template <int OP, int KIND, class T>
cudaError_t launch_t(int dir, const T* in, T* out, int64_t ny, int64_t nx, int64_t nbatch, int64_t bstride,
                     cudaStream_t st) {
    // One work item per CTA (the grid-stride loops only matter beyond this cap): the block
    // scheduler then overlaps one CTA's loads with another's arithmetic, which the measured
    // throughput prefers to a persistent grid that loops load -> compute -> store.
    const int blocks_cap = 1 << 30;
    (void)num_sms;
    constexpr int K = 16 / sizeof(T);
    const bool aligned = (nx % K == 0) && (bstride % K == 0) && (reinterpret_cast<uintptr_t>(in) % 16 == 0) &&
                         (reinterpret_cast<uintptr_t>(out) % 16 == 0);
    if (aligned) {
        // bulk-staged tiles, one per CTA
        if (dir == 0) {
            const T idx = inv_spacing<T>(OpShape<OP>::h2, nx);
            constexpr int TC = xi_bulk_cols<T>();
            const int64_t items = nbatch * ((ny + kXiBulkRows - 1) / kXiBulkRows) * ((nx + TC - 1) / TC);
            op_xi_bulk_kernel<OP, KIND, T><<<(unsigned)items, kThreads, xi_bulk_smem<T>(), st>>>(
                in, out, (int)ny, (int)nx, bstride, idx);
        } else {
            const T idx = inv_spacing<T>(OpShape<OP>::h2, ny);
            const int simd = (int)(simd_lanes<T>() * (nx / simd_lanes<T>()));
            constexpr int TC = 1024 / sizeof(T);
            constexpr size_t smem = eta_bulk_smem<OP, T>();
            static bool configured = false;  // per instantiation: the attribute belongs to the function
            if (!configured) {
                const cudaError_t e = cudaFuncSetAttribute(op_eta_bulk_kernel<OP, KIND, T>,
                                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                if (e != cudaSuccess) return e;
                configured = true;
            }
            const int64_t items = nbatch * ((ny + kEtaBulkRows - 1) / kEtaBulkRows) * ((nx + TC - 1) / TC);
            op_eta_bulk_kernel<OP, KIND, T><<<(unsigned)items, kThreads, smem, st>>>(in, out, (int)ny, (int)nx, bstride,
                                                                                     idx, simd);
        }
        return cudaGetLastError();
    }
    if (dir == 0) {
        const T idx = inv_spacing<T>(OpShape<OP>::h2, nx);
        const int64_t nseg = (nx + kThreads * K - 1) / (kThreads * K);
        const int64_t items = nbatch * ((ny + kXiRows - 1) / kXiRows) * nseg;
        const int grid = (int)(items < blocks_cap ? items : blocks_cap);
        const bool vec_ok = (nx % K == 0) && (bstride % K == 0) && (reinterpret_cast<uintptr_t>(out) % 16 == 0) &&
                            (reinterpret_cast<uintptr_t>(in) % 16 == 0);
        op_xi_kernel<OP, KIND, T><<<grid, kThreads, 0, st>>>(in, out, (int)ny, (int)nx, nbatch, bstride, idx, vec_ok);
    } else {
        const T idx = inv_spacing<T>(OpShape<OP>::h2, ny);
        const int simd = (int)(simd_lanes<T>() * (nx / simd_lanes<T>()));
        constexpr int K = 16 / sizeof(T);
        const bool vec_ok = (nx % K == 0) && (bstride % K == 0) && (reinterpret_cast<uintptr_t>(in) % 16 == 0) &&
                            (reinterpret_cast<uintptr_t>(out) % 16 == 0);
        if (vec_ok) {
            const int64_t items = nbatch * ((nx / K + kThreads - 1) / kThreads) * ((ny + kEtaRows - 1) / kEtaRows);
            const int grid = (int)(items < blocks_cap ? items : blocks_cap);
            op_eta_vec_kernel<OP, KIND, T><<<grid, kThreads, 0, st>>>(in, out, (int)ny, (int)nx, nbatch, bstride, idx,
                                                                      simd);
        } else {
            const int64_t items = nbatch * ((nx + kThreads - 1) / kThreads) * ((ny + kEtaRows - 1) / kEtaRows);
            const int grid = (int)(items < blocks_cap ? items : blocks_cap);
            op_eta_kernel<OP, KIND, T><<<grid, kThreads, 0, st>>>(in, out, (int)ny, (int)nx, nbatch, bstride, idx,
                                                                  simd);
        }
    }
    return cudaGetLastError();
}

template <int OP, class T>
cudaError_t launch_kind(int dir, int kind, const void* in, void* out, int64_t ny, int64_t nx, int64_t nbatch,
                        int64_t bstride, cudaStream_t st) {
    const T* i = static_cast<const T*>(in);
    T* o = static_cast<T*>(out);
    if (kind == DIFF) return launch_t<OP, DIFF, T>(dir, i, o, ny, nx, nbatch, bstride, st);
    if constexpr (OpShape<OP>::upwind) return launch_t<OP, DISS, T>(dir, i, o, ny, nx, nbatch, bstride, st);
    return cudaErrorInvalidValue;
}

template <class T>
cudaError_t launch_op(int op, int dir, int kind, const void* in, void* out, int64_t ny, int64_t nx, int64_t nbatch,
                      int64_t bstride, cudaStream_t st) {
    switch (op) {
        case UPWIND4: return launch_kind<UPWIND4, T>(dir, kind, in, out, ny, nx, nbatch, bstride, st);
        case UPWIND4H2: return launch_kind<UPWIND4H2, T>(dir, kind, in, out, ny, nx, nbatch, bstride, st);
        case UPWIND9: return launch_kind<UPWIND9, T>(dir, kind, in, out, ny, nx, nbatch, bstride, st);
        case UPWIND9H2: return launch_kind<UPWIND9H2, T>(dir, kind, in, out, ny, nx, nbatch, bstride, st);
        case SBP4: return launch_kind<SBP4, T>(dir, kind, in, out, ny, nx, nbatch, bstride, st);
        case SBP8: return launch_kind<SBP8, T>(dir, kind, in, out, ny, nx, nbatch, bstride, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

cudaError_t op_apply(int op, int dir, int kind, int dtype, const void* in, void* out, int64_t ny, int64_t nx,
                     int64_t nbatch, int64_t bstride, cudaStream_t st) {
    if (dtype == 0) return launch_op<double>(op, dir, kind, in, out, ny, nx, nbatch, bstride, st);
    return launch_op<float>(op, dir, kind, in, out, ny, nx, nbatch, bstride, st);
}

}  // namespace sbp
