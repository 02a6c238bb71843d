// Kernels of the learned correction network: a 5-layer 3x3 convolutional network on the 64 x 64
// coarse grid (4 -> 32 -> 32 -> 32 -> 32 -> 4 channels, GELU between layers).  Activations are
// BF16 in NHWC layout (channels innermost), accumulation is FP32 on the tensor cores
// (mma.sync m16n8k16 bf16), pre-activations, outputs, gradients and parameters are FP32.
//
// Channel counts are padded to what one MMA step consumes: the 4-channel input is stored with
// 16 channels (zeros above 4), the 4-channel output with 8, and the gradient of the output with
// 16.  Padded weights, biases and their gradients are zero and stay zero.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace sbp {
namespace cnn {

constexpr int kImg = 64;           // image side: the coarse grid
constexpr int kPix = kImg * kImg;  // pixels per image
constexpr int kBand = 2;           // image rows per CTA in the convolution kernels (128 pixels)
constexpr int kConvThreads = 128;  // 4 warps, 32 pixels each
constexpr int kWgradRows = 16;     // image rows per CTA in the weight-gradient kernel
constexpr int kWgradThreads = 288; // 9 warps, one per filter tap

enum Epilogue { EPI_GELU = 0, EPI_LINEAR = 1, EPI_DGELU = 2 };

// D = A * B + D for one 16x16 (row) by 16x8 (col) bf16 tile with f32 accumulators.
__device__ __forceinline__ void mma_bf16(float c[4], const unsigned a[4], const unsigned b[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Four transposed 8x8 b16 matrices from shared memory; lane i gives the address of row i % 8
// of matrix i / 8 (16-byte aligned rows).
__device__ __forceinline__ void ldsm_x4_trans(unsigned r[4], const void* row_addr) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(row_addr);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(a));
}

// GELU with the Gaussian CDF, x * Phi(x), and its derivative Phi(x) + x * phi(x).
__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const unsigned*>(&v);
}

// 3x3 convolution with zero padding as an implicit GEMM: out[p][n] = sum over taps t and input
// channels k of x[p + off(t)][k] * w[n][t][k], off(t) = (t / 3 - 1, t % 3 - 1).  One CTA takes
// kBand image rows: their halo (kBand + 2 rows x 66 columns) and all weights go to shared
// memory, warp w computes 32 pixels of row w / 2 for all COUT channels.  Epilogues:
//   EPI_GELU   z = acc + bias -> zout (f32), gelu(z) -> yout (bf16)   (hidden layers)
//   EPI_LINEAR acc + bias -> zout (f32)                                (output layer)
//   EPI_DGELU  acc * gelu'(zprev) -> yout (bf16)                       (gradient of a hidden layer)
// Shared rows are padded by 8 bf16 so the fragment loads of 8 consecutive pixels (or output
// channels) fall in distinct banks.
template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(kConvThreads) conv3x3_kernel(const __nv_bfloat16* __restrict__ x,
                                                               const __nv_bfloat16* __restrict__ w,
                                                               const float* __restrict__ bias,
                                                               const float* __restrict__ zprev,
                                                               float* __restrict__ zout,
                                                               __nv_bfloat16* __restrict__ yout) {
    static_assert(CIN % 16 == 0 && COUT % 8 == 0, "channel padding");
    constexpr int SP = CIN + 8;
    constexpr int HR = kBand + 2, HC = kImg + 2;
    constexpr int NT = COUT / 8;
    __shared__ __align__(16) __nv_bfloat16 sx[HR * HC * SP];
    __shared__ __align__(16) __nv_bfloat16 sw[COUT * 9 * SP];
    const int img = blockIdx.x / (kImg / kBand);
    const int r0 = (blockIdx.x % (kImg / kBand)) * kBand;
    for (int i = threadIdx.x; i < COUT * 9 * (CIN / 8); i += kConvThreads) {
        const int row = i / (CIN / 8), v = i % (CIN / 8);
        *reinterpret_cast<uint4*>(sw + row * SP + v * 8) = *reinterpret_cast<const uint4*>(w + row * CIN + v * 8);
    }
    for (int i = threadIdx.x; i < HR * HC * (CIN / 8); i += kConvThreads) {
        const int pix = i / (CIN / 8), v = i % (CIN / 8);
        const int hr = pix / HC, hc = pix % HC;
        const int gr = r0 + hr - 1, gc = hc - 1;
        uint4 val = make_uint4(0u, 0u, 0u, 0u);
        if (gr >= 0 && gr < kImg && gc >= 0 && gc < kImg)
            val = *reinterpret_cast<const uint4*>(x + ((int64_t)(img * kImg + gr) * kImg + gc) * CIN + v * 8);
        *reinterpret_cast<uint4*>(sx + pix * SP + v * 8) = val;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wr = warp >> 1, wc0 = (warp & 1) * 32;
    const int g = lane >> 2, q = lane & 3;
    float acc[2][NT][4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[mt][nt][e] = 0.0f;
#pragma unroll 1
    for (int tap = 0; tap < 9; ++tap) {
        const int dy = tap / 3, dx = tap % 3;
#pragma unroll
        for (int c0 = 0; c0 < CIN; c0 += 16) {
            unsigned a[2][4];
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                const __nv_bfloat16* p0 = sx + ((wr + dy) * HC + wc0 + mt * 16 + g + dx) * SP + c0 + 2 * q;
                const __nv_bfloat16* p1 = p0 + 8 * SP;
                a[mt][0] = *reinterpret_cast<const unsigned*>(p0);
                a[mt][1] = *reinterpret_cast<const unsigned*>(p1);
                a[mt][2] = *reinterpret_cast<const unsigned*>(p0 + 8);
                a[mt][3] = *reinterpret_cast<const unsigned*>(p1 + 8);
            }
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) {
                const __nv_bfloat16* pb = sw + ((nt * 8 + g) * 9 + tap) * SP + c0 + 2 * q;
                const unsigned b[2] = {*reinterpret_cast<const unsigned*>(pb),
                                       *reinterpret_cast<const unsigned*>(pb + 8)};
                mma_bf16(acc[0][nt], a[0], b);
                mma_bf16(acc[1][nt], a[1], b);
            }
        }
    }
    const int row = r0 + wr;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int col = wc0 + mt * 16 + g + half * 8;
            const int64_t p = (int64_t)(img * kImg + row) * kImg + col;
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) {
                const int co = nt * 8 + 2 * q;
                const float v0 = acc[mt][nt][2 * half], v1 = acc[mt][nt][2 * half + 1];
                if constexpr (EPI == EPI_GELU) {
                    const float z0 = v0 + bias[co], z1 = v1 + bias[co + 1];
                    *reinterpret_cast<float2*>(zout + p * COUT + co) = make_float2(z0, z1);
                    *reinterpret_cast<unsigned*>(yout + p * COUT + co) = pack_bf16(gelu(z0), gelu(z1));
                } else if constexpr (EPI == EPI_LINEAR) {
                    *reinterpret_cast<float2*>(zout + p * COUT + co) = make_float2(v0 + bias[co], v1 + bias[co + 1]);
                } else {
                    const float2 zp = *reinterpret_cast<const float2*>(zprev + p * COUT + co);
                    *reinterpret_cast<unsigned*>(yout + p * COUT + co) =
                        pack_bf16(v0 * gelu_grad(zp.x), v1 * gelu_grad(zp.y));
                }
            }
        }
}

// Weight and bias gradients of one layer: dw[m][t][k] = sum over pixels p of dz[p][m] *
// x[p + off(t)][k], db[m] = sum over p of dz[p][m], as partial sums per CTA (kWgradRows image
// rows each) that wgrad_reduce_kernel adds up in a fixed order.  M = channels of dz as stored
// (16 or 32), MSTORE = rows of the layer's weight tensor (<= M).  Warp t computes tap t; both
// GEMM operands are pixel-major in memory and reach the MMA through transposing ldmatrix.
template <int CIN, int M, int MSTORE>
__global__ void __launch_bounds__(kWgradThreads) wgrad_kernel(const __nv_bfloat16* __restrict__ x,
                                                              const __nv_bfloat16* __restrict__ dz,
                                                              float* __restrict__ part_w,
                                                              float* __restrict__ part_b) {
    static_assert(CIN % 16 == 0 && M % 16 == 0 && MSTORE <= M, "channel padding");
    constexpr int SPX = CIN + 8, SPZ = M + 8;
    constexpr int HR = kBand + 2, HC = kImg + 2;
    constexpr int MT = M / 16, NT = CIN / 8;
    __shared__ __align__(16) __nv_bfloat16 sx[HR * HC * SPX];
    __shared__ __align__(16) __nv_bfloat16 sz[kBand * kImg * SPZ];
    constexpr int chunks_per_img = kImg / kWgradRows;
    const int img = blockIdx.x / chunks_per_img;
    const int rbase = (blockIdx.x % chunks_per_img) * kWgradRows;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tap = warp, dy = tap / 3, dx = tap % 3;
    float acc[MT][NT][4];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[mt][nt][e] = 0.0f;
    float bsum = 0.0f;
    // ldmatrix row selection: lane i serves row i % 8 of matrix i / 8
    const int lm = lane >> 3, lr = lane & 7;
#pragma unroll 1
    for (int r0 = rbase; r0 < rbase + kWgradRows; r0 += kBand) {
        __syncthreads();
        for (int i = threadIdx.x; i < HR * HC * (CIN / 8); i += kWgradThreads) {
            const int pix = i / (CIN / 8), v = i % (CIN / 8);
            const int hr = pix / HC, hc = pix % HC;
            const int gr = r0 + hr - 1, gc = hc - 1;
            uint4 val = make_uint4(0u, 0u, 0u, 0u);
            if (gr >= 0 && gr < kImg && gc >= 0 && gc < kImg)
                val = *reinterpret_cast<const uint4*>(x + ((int64_t)(img * kImg + gr) * kImg + gc) * CIN + v * 8);
            *reinterpret_cast<uint4*>(sx + pix * SPX + v * 8) = val;
        }
        for (int i = threadIdx.x; i < kBand * kImg * (M / 8); i += kWgradThreads) {
            const int pix = i / (M / 8), v = i % (M / 8);
            *reinterpret_cast<uint4*>(sz + pix * SPZ + v * 8) = *reinterpret_cast<const uint4*>(
                dz + ((int64_t)img * kPix + (int64_t)r0 * kImg + pix) * M + v * 8);
        }
        __syncthreads();
        if (threadIdx.x < M)
            for (int pix = 0; pix < kBand * kImg; ++pix) bsum += __bfloat162float(sz[pix * SPZ + threadIdx.x]);
#pragma unroll 1
        for (int k0 = 0; k0 < kBand * kImg; k0 += 16) {
            // 16 consecutive pixels of one image row
            const int prow = k0 / kImg, pcol = k0 % kImg;
            unsigned a[MT][4];
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) {
                // matrices: (k 0-7, m 0-7), (k 0-7, m 8-15), (k 8-15, m 0-7), (k 8-15, m 8-15)
                const int kk = k0 + (lm >> 1) * 8 + lr;
                const int mm = mt * 16 + (lm & 1) * 8;
                ldsm_x4_trans(a[mt], sz + kk * SPZ + mm);
            }
#pragma unroll
            for (int nt = 0; nt < NT; nt += 2) {
                // matrices: (k 0-7, n 0-7), (k 8-15, n 0-7), (k 0-7, n 8-15), (k 8-15, n 8-15)
                const int kc = pcol + (lm & 1) * 8 + lr;
                const int nn = (nt + (lm >> 1)) * 8;
                unsigned b[4];
                ldsm_x4_trans(b, sx + ((prow + dy) * HC + kc + dx) * SPX + nn);
                const unsigned b0[2] = {b[0], b[1]}, b1[2] = {b[2], b[3]};
#pragma unroll
                for (int mt = 0; mt < MT; ++mt) {
                    mma_bf16(acc[mt][nt], a[mt], b0);
                    mma_bf16(acc[mt][nt + 1], a[mt], b1);
                }
            }
        }
    }
    const int g = lane >> 2, q = lane & 3;
    float* pw = part_w + (int64_t)blockIdx.x * (MSTORE * 9 * CIN);
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                const int m = mt * 16 + g + half * 8;
                const int k = nt * 8 + 2 * q;
                if (m < MSTORE) {
                    pw[(m * 9 + tap) * CIN + k] = acc[mt][nt][2 * half];
                    pw[(m * 9 + tap) * CIN + k + 1] = acc[mt][nt][2 * half + 1];
                }
            }
    if (threadIdx.x < MSTORE) part_b[(int64_t)blockIdx.x * MSTORE + threadIdx.x] = bsum;
}

// Sum of the per-CTA partials in CTA order: grad[e] for the weights (nw elements) then the
// biases (nb elements).
__global__ void wgrad_reduce_kernel(const float* __restrict__ part_w, const float* __restrict__ part_b, int nparts,
                                    int nw, int nb, float* __restrict__ gw, float* __restrict__ gb) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < nw) {
        float s = 0.0f;
        for (int c = 0; c < nparts; ++c) s += part_w[(int64_t)c * nw + e];
        gw[e] = s;
    } else if (e < nw + nb) {
        const int j = e - nw;
        float s = 0.0f;
        for (int c = 0; c < nparts; ++c) s += part_b[(int64_t)c * nb + j];
        gb[j] = s;
    }
}

}  // namespace cnn
}  // namespace sbp
