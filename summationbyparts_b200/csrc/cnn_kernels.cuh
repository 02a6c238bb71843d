// Kernels of the learned correction network: a 5-layer 3x3 convolutional network on the 64 x 64
// coarse grid (4 -> 32 -> 32 -> 32 -> 32 -> 4 channels, GELU between layers).  Activations are
// BF16 in NHWC layout (channels innermost), accumulation is FP32 on the tcgen05 tensor cores
// with TMEM accumulators (convolutions forward and backward-data, and the weight gradients);
// pre-activations, outputs, gradients and parameters are FP32.
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
constexpr int kBand = 4;           // image rows per CTA of the convolution kernel (256 pixels)
constexpr int kConvThreads = 256;  // 8 warps: one pixel of the band per thread
constexpr int kWgradThreads = 128; // 4 warps: one accumulator row of a 128-row tile per thread
constexpr int kWgradRows = 4;      // image rows per CTA in the weight-gradient kernel

enum Epilogue { EPI_GELU = 0, EPI_LINEAR = 1, EPI_DGELU = 2 };

// erf(z) by the rational approximation of Abramowitz and Stegun, Handbook of Mathematical
// Functions, formula 7.1.26: erf(z) = 1 - t (a1 + t (a2 + t (a3 + t (a4 + t a5)))) exp(-z^2),
// t = 1 / (1 + p z) for z >= 0, odd in z; |error| <= 1.5e-7 in exact arithmetic, 5.4e-7 in this
// f32 evaluation (checked against a double-precision erf on [-6, 6]).  g returns exp(-z^2),
// which the GELU derivative shares.  The activations are rounded to bf16 (3.9e-3 relative).
__device__ __forceinline__ float erf_as(float z, float& g) {
    const float az = fabsf(z);
    const float t = __fdividef(1.0f, fmaf(0.3275911f, az, 1.0f));
    g = __expf(-az * az);
    const float poly =
        t * fmaf(t, fmaf(t, fmaf(t, fmaf(t, 1.061405429f, -1.453152027f), 1.421413741f), -0.284496736f), 0.254829592f);
    return copysignf(fmaf(-poly, g, 1.0f), z);
}

// GELU with the Gaussian CDF, x * Phi(x), and its derivative Phi(x) + x * phi(x), with
// Phi(x) = (1 + erf(x / sqrt 2)) / 2 and phi(x) = exp(-x^2 / 2) / sqrt(2 pi).
__device__ __forceinline__ float gelu(float x) {
    float g;
    return 0.5f * x * (1.0f + erf_as(x * 0.70710678118654752f, g));
}
__device__ __forceinline__ float gelu_grad(float x) {
    float g;
    const float e = erf_as(x * 0.70710678118654752f, g);
    return fmaf(0.5f, 1.0f + e, x * 0.39894228040143268f * g);
}

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const unsigned*>(&v);
}

// ---- tcgen05 (5th-generation tensor core) helpers, sm_100a --------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor of a K-major bf16 operand in the canonical layout without
// swizzling: core matrices of 8 rows x 16 bytes (128 contiguous bytes, row after row), adjacent
// core matrices `lbo` bytes apart along K and `sbo` bytes apart along M (or N).  Fields: start
// address / 16 (bits 0-13), lbo / 16 (16-29), sbo / 16 (32-45), descriptor version 1 (46-47),
// base offset 0, layout type 0 = no swizzle (61-63).
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor of tcgen05.mma kind::f16 with bf16 A and B (both K-major) and an f32
// accumulator, M x N: D format (bits 4-5) = f32, A and B formats (7-9, 10-12) = bf16, N / 8
// (17-22), M / 16 (24-28).
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D (tmem) = A * B (+ D when accumulate != 0), issued by one thread.
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// Arrive on the mbarrier once every tcgen05.mma issued so far by this thread has completed.
__device__ __forceinline__ void umma_commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* mbar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n.reg .pred q;\nmbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\nselp.b32 %0, 1, 0, q;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(mbar)), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive f32 TMEM columns of this thread's lane (32x32b shape: warp w reads lanes
// 32 w .. 32 w + 31, so the lane field of taddr must be 32 w).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float v[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,"
        "%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 16-byte asynchronous global -> shared copy; src_bytes = 0 fills the destination with zeros.
__device__ __forceinline__ void cp_async16(void* dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}

// Bit of the network's device status word set when a convolution gave up waiting for its
// tensor-core work (the wait is bounded, so a fault cannot hang the stream).
constexpr unsigned kStatusMmaTimeout = 1u;
constexpr int kMmaWaitLimit = 1 << 22;  // mbarrier polls before giving up

// Shared-memory layout of the tcgen05 convolution (dynamic, 1024-byte aligned base).
template <int CIN, int COUT>
struct ConvTcLayout {
    static constexpr int NP = COUT < 16 ? 16 : COUT;        // N of the MMA (multiple of 16 for M = 128)
    static constexpr int HR = kBand + 2;                    // halo rows
    static constexpr int TILES = kBand * kImg / 128;        // M = 128 accumulator tiles (2)
    static constexpr int TMEM_COLS = TILES * NP <= 32 ? 32 : 64;
    static constexpr int PIX = HR * kImg;                   // pixels of one shifted copy
    static constexpr int CH = CIN / 8;                      // 16-byte channel chunks per pixel
    static constexpr int SBO = CH * 128;                    // bytes between 8-row groups
    static constexpr int A_BYTES = PIX * CIN * 2;           // one shifted copy
    static constexpr int B_TAP = NP * CIN * 2;              // weights of one tap
    static constexpr int B_OFF = 3 * A_BYTES;
    static constexpr int BAR_OFF = B_OFF + 9 * B_TAP;
    static constexpr int BYTES = BAR_OFF + 16;
};
// Byte offset of (row, 16-byte chunk kc) in a canonical no-swizzle K-major operand.
template <int CH>
__device__ __forceinline__ int canon_off(int row, int kc) {
    return ((row >> 3) * CH + kc) * 128 + (row & 7) * 16;
}

// 3x3 convolution with zero padding as an implicit GEMM on the tcgen05 tensor cores:
// out[p][n] = sum over taps t and input channels k of x[p + off(t)][k] * w[n][t][k],
// off(t) = (t / 3 - 1, t % 3 - 1).  One CTA of 256 threads computes kBand = 4 image rows
// (two M = 128 pixel tiles, each 2 image rows) for all output channels (N = COUT, at least 16),
// so the weights are staged once per 256 pixels: the input halo goes to
// shared memory as three copies shifted by 0, 1 and 2 columns, each in the canonical K-major
// layout, so the A operand of tap (dy, dx) is copy dx started dy image rows down -- an aligned
// descriptor offset, no per-tap copy (tile h starts 2 h image rows further); the weights of the
// 9 taps follow in the same layout.  One thread issues the 2 x 9 x CIN / 16 MMAs (K = 16 each)
// into two TMEM accumulators of 128 lanes x N f32 columns and commits them to an mbarrier; after
// the (bounded) wait warp w reads lanes 32 (w % 4) .. of tile w / 4 -- one pixel per thread, all
// channels -- and runs the epilogue:
//   EPI_GELU   z = acc + bias -> zout (f32), gelu(z) -> yout (bf16)   (hidden layers)
//   EPI_LINEAR acc + bias -> zout (f32)                                (output layer)
//   EPI_DGELU  acc * gelu'(zprev) -> yout (bf16)                       (gradient of a hidden layer)
template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(kConvThreads) conv3x3_tc_kernel(const __nv_bfloat16* __restrict__ x,
                                                                  const __nv_bfloat16* __restrict__ w,
                                                                  const float* __restrict__ bias,
                                                                  const float* __restrict__ zprev,
                                                                  float* __restrict__ zout,
                                                                  __nv_bfloat16* __restrict__ yout,
                                                                  unsigned* __restrict__ status) {
    using L = ConvTcLayout<CIN, COUT>;
    static_assert(CIN % 16 == 0 && COUT % 8 == 0 && L::NP <= 32, "channel padding");
    extern __shared__ __align__(1024) unsigned char smem[];
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + L::BAR_OFF);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + L::BAR_OFF + 8);
    const int img = blockIdx.x / (kImg / kBand);
    const int r0 = (blockIdx.x % (kImg / kBand)) * kBand;
    const int tid = threadIdx.x, warp = tid >> 5;

    if (warp == 0) {
        // TILES accumulators of 128 lanes x NP f32 columns (32 columns is the allocation minimum)
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(L::TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // Operands by asynchronous 16-byte copies straight into the canonical layout, all of a
    // thread's copies in flight at once.  Weights: B[n][k] of tap t = w[n][t][k], rows n >= COUT
    // zero-filled.
    for (int i = tid; i < L::NP * 9 * L::CH; i += kConvThreads) {
        const int kc = i % L::CH, t = (i / L::CH) % 9, n = i / (L::CH * 9);
        const bool in = n < COUT;
        cp_async16(smem + L::B_OFF + t * L::B_TAP + canon_off<L::CH>(n, kc),
                   w + ((int64_t)(in ? n : 0) * 9 + t) * CIN + kc * 8, in ? 16u : 0u);
    }
    // input halo: rows r0 - 1 .. r0 + kBand, columns -1 .. 64 (zero outside the image), into the
    // copies shifted by dx: copy dx, pixel (hr, c) = halo (hr, c + dx), i.e. image column c + dx - 1
    for (int i = tid; i < 3 * L::HR * kImg * L::CH; i += kConvThreads) {
        const int kc = i % L::CH, c = (i / L::CH) % kImg, hr = (i / (L::CH * kImg)) % L::HR;
        const int dx = i / (L::CH * kImg * L::HR);
        const int gr = r0 + hr - 1, gc = c + dx - 1;
        const bool in = gr >= 0 && gr < kImg && gc >= 0 && gc < kImg;
        const int64_t pix = in ? (int64_t)(img * kImg + gr) * kImg + gc : 0;
        cp_async16(smem + dx * L::A_BYTES + canon_off<L::CH>(hr * kImg + c, kc), x + pix * CIN + kc * 8,
                   in ? 16u : 0u);
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    // the operands written through the generic proxy become visible to the tensor core's proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    if (tid == 0) {
        constexpr uint32_t idesc = umma_idesc_bf16(128, L::NP);
        const uint32_t base = smem_u32(smem);
        uint32_t acc = 0;
#pragma unroll 1
        for (int t = 0; t < 9; ++t) {
            const int dy = t / 3, dx = t % 3;
#pragma unroll
            for (int j = 0; j < CIN / 16; ++j) {
                const uint32_t b = base + L::B_OFF + t * L::B_TAP + 2 * j * 128;
#pragma unroll
                for (int h = 0; h < L::TILES; ++h) {
                    const uint32_t a = base + dx * L::A_BYTES + (2 * h + dy) * (kImg / 8) * L::SBO + 2 * j * 128;
                    umma_bf16(tmem + h * L::NP, umma_desc(a, 128, L::SBO), umma_desc(b, 128, L::SBO), idesc, acc);
                }
                acc = 1;
            }
        }
        umma_commit(mbar);
    }
    bool done = false;
    for (int it = 0; it < kMmaWaitLimit && !done; ++it) done = mbar_try_wait(mbar, 0);
    tc_fence_after();
    if (done) {
        // thread tid holds row tid % 128 of accumulator tid / 128: pixel (r0 + tid / 64, tid % 64)
        const int64_t p = (int64_t)(img * kImg + r0 + tid / kImg) * kImg + tid % kImg;
        const uint32_t taddr = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (tid / 128) * L::NP;
        float v[32];
        if constexpr (L::NP == 32) tmem_ld32(taddr, v);
        else tmem_ld16(taddr, v);
#pragma unroll
        for (int co = 0; co < COUT; co += 2) {
            const float v0 = v[co], v1 = v[co + 1];
            if constexpr (EPI == EPI_GELU) {
                const float z0 = v0 + bias[co], z1 = v1 + bias[co + 1];
                *reinterpret_cast<float2*>(zout + p * COUT + co) = make_float2(z0, z1);
                *reinterpret_cast<unsigned*>(yout + p * COUT + co) = pack_bf16(gelu(z0), gelu(z1));
            } else if constexpr (EPI == EPI_LINEAR) {
                *reinterpret_cast<float2*>(zout + p * COUT + co) = make_float2(v0 + bias[co], v1 + bias[co + 1]);
            } else {
                const float2 zp = *reinterpret_cast<const float2*>(zprev + p * COUT + co);
                *reinterpret_cast<unsigned*>(yout + p * COUT + co) = pack_bf16(v0 * gelu_grad(zp.x), v1 * gelu_grad(zp.y));
            }
        }
    } else if ((tid & 31) == 0) {
        atomicOr(status, kStatusMmaTimeout);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(L::TMEM_COLS) : "memory");
    }
}

// Word k (0..3, a compile-time constant after unrolling) of a 16-byte vector, selected without
// taking the vector's address (which would move it to local memory).
__device__ __forceinline__ unsigned word_of(const uint4& u, int k) {
    return k == 0 ? u.x : (k == 1 ? u.y : (k == 2 ? u.z : u.w));
}

// 8 x 8 transpose of bf16: in[j] holds 8 channels of pixel j, out[i] 8 pixels of channel i.
__device__ __forceinline__ void transpose8x8_bf16(const uint4 in[8], uint4 out[8]) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const unsigned sel = (i & 1) ? 0x7632u : 0x5410u;  // high or low halves of word i / 2
        unsigned w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) w[q] = __byte_perm(word_of(in[2 * q], i >> 1), word_of(in[2 * q + 1], i >> 1), sel);
        out[i] = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// Shared-memory layout of the tcgen05 weight-gradient kernel: the canonical A and B operands of
// one image row, then the CTA's raw input rows (x with one halo row on each side, dz) as copied
// from global memory.  Raw rows hold pixels channel-innermost with 16 bytes of padding after every
// 8 pixels, so 8 threads reading the same channel chunk of 8 consecutive pixel groups hit 8
// different 16-byte bank groups.
template <int CIN, int M>
struct WgradTcLayout {
    static constexpr int ROWS = 9 * CIN + 1;                // (tap, input channel) rows + the ones row
    static constexpr int TILES = (ROWS + 127) / 128;        // M = 128 tiles
    static constexpr int AROWS = TILES * 128;
    static constexpr int P = kImg;                          // pixels per chunk (one image row)
    static constexpr int SBO = (P / 8) * 128;               // bytes between 8-row groups
    static constexpr int A_BYTES = AROWS * P * 2;
    static constexpr int B_OFF = A_BYTES;
    static constexpr int XROW = P * CIN * 2 + (P / 8) * 16;  // bytes of one raw x row
    static constexpr int ZROW = P * M * 2 + (P / 8) * 16;    // bytes of one raw dz row
    static constexpr int XR_OFF = B_OFF + M * P * 2;
    static constexpr int ZR_OFF = XR_OFF + (kWgradRows + 2) * XROW;
    static constexpr int BAR_OFF = ZR_OFF + kWgradRows * ZROW;
    static constexpr int BYTES = BAR_OFF + 16;
    static constexpr int TMEM_COLS = TILES * M <= 32 ? 32 : (TILES * M <= 64 ? 64 : 128);
};

// Byte offset of pixel c, channel chunk kc of a raw row (C channels per pixel).
template <int C>
__device__ __forceinline__ int raw_off(int c, int kc) {
    return c * C * 2 + (c >> 3) * 16 + kc * 16;
}

// Weight and bias gradients of one layer on the tcgen05 tensor cores, as partial sums per CTA
// (kWgradRows image rows each) that wgrad_reduce_kernel adds up in a fixed order:
// dw[m][t][k] = sum over pixels p of dz[p][m] * x[p + off(t)][k], db[m] = sum over p of dz[p][m].
// The GEMM D[(t, k)][m] = sum over p of A[(t, k)][p] * B[m][p] has the 9 CIN (tap, channel) pairs
// as its rows (M, in tiles of 128), the dz channels as N and the pixels as K.  The CTA's raw rows
// of x (with the halo rows, zero outside the image) and dz arrive first, by 16-byte asynchronous
// copies all in flight at once.  Per image row (64 pixels) the threads then write A and B in the
// canonical K-major layout -- each 8 x 8 core matrix the register transpose of 8 pixels' 16-byte
// channel vectors read from the raw rows -- and one thread issues TILES x 4 MMAs (K = 16)
// accumulating in TMEM across the CTA's rows.  Row 9 CIN of A is all ones, so D's row 9 CIN is
// the bias gradient; the remaining padding rows are zero.
// M = channels of dz as stored (16 or 32), MSTORE = rows of the layer's weight tensor (<= M).
template <int CIN, int M, int MSTORE>
__global__ void __launch_bounds__(kWgradThreads) wgrad_tc_kernel(const __nv_bfloat16* __restrict__ x,
                                                                const __nv_bfloat16* __restrict__ dz,
                                                                float* __restrict__ part_w,
                                                                float* __restrict__ part_b,
                                                                unsigned* __restrict__ status) {
    using L = WgradTcLayout<CIN, M>;
    static_assert(CIN % 16 == 0 && M % 16 == 0 && MSTORE <= M && L::TILES * M <= 128, "channel padding");
    constexpr int XCH = CIN / 8, ZCH = M / 8;
    extern __shared__ __align__(1024) unsigned char smem[];
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + L::BAR_OFF);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + L::BAR_OFF + 8);
    constexpr int chunks_per_img = kImg / kWgradRows;
    const int img = blockIdx.x / chunks_per_img;
    const int rbase = (blockIdx.x % chunks_per_img) * kWgradRows;
    const int tid = threadIdx.x, warp = tid >> 5;
    // raw rows: x rows rbase - 1 .. rbase + kWgradRows (zero-filled outside the image), dz rows
    // rbase .. rbase + kWgradRows - 1
    for (int i = tid; i < (kWgradRows + 2) * L::P * XCH; i += kWgradThreads) {
        const int kc = i % XCH, c = (i / XCH) % L::P, hr = i / (XCH * L::P);
        const int gr = rbase + hr - 1;
        const bool in = gr >= 0 && gr < kImg;
        cp_async16(smem + L::XR_OFF + hr * L::XROW + raw_off<CIN>(c, kc),
                   x + ((int64_t)(img * kImg + (in ? gr : 0)) * kImg + c) * CIN + kc * 8, in ? 16u : 0u);
    }
    for (int i = tid; i < kWgradRows * L::P * ZCH; i += kWgradThreads) {
        const int kc = i % ZCH, c = (i / ZCH) % L::P, hr = i / (ZCH * L::P);
        cp_async16(smem + L::ZR_OFF + hr * L::ZROW + raw_off<M>(c, kc),
                   dz + ((int64_t)(img * kImg + rbase + hr) * kImg + c) * M + kc * 8, 16u);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(L::TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // rows 9 CIN .. AROWS - 1 of A: the ones row, then zeros; written once
    {
        constexpr int first_group = (9 * CIN) / 8, groups = L::AROWS / 8 - first_group;
        for (int i = tid; i < groups * (L::P / 8) * 8; i += kWgradThreads) {
            const int row = first_group * 8 + (i / ((L::P / 8) * 8)) * 8 + (i % 8);
            const int pg = (i / 8) % (L::P / 8);
            const unsigned one = row == 9 * CIN ? 0x3F803F80u : 0u;  // bf16 1.0 pairs
            *reinterpret_cast<uint4*>(smem + (row >> 3) * L::SBO + pg * 128 + (row & 7) * 16) =
                make_uint4(one, one, one, one);
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    constexpr uint32_t idesc = umma_idesc_bf16(128, M);
    bool ok = true;
    uint32_t phase = 0;
#pragma unroll 1
    for (int lr = 0; lr < kWgradRows && ok; ++lr) {
        // A core matrices: (tap t, channel block kc, pixel group pg) = transpose of the 8 x 8 block
        // x[pixels 8 pg + j shifted by the tap][channels 8 kc + i] (zero outside the image).
        // Consecutive threads take consecutive pixel groups: conflict-free raw reads (padding) and
        // canonical writes (128 bytes apart).
        for (int i = tid; i < 9 * XCH * (L::P / 8); i += kWgradThreads) {
            const int pg = i % (L::P / 8), kc = (i / (L::P / 8)) % XCH, t = i / ((L::P / 8) * XCH);
            const unsigned char* src = smem + L::XR_OFF + (lr + t / 3) * L::XROW;
            uint4 v[8], o[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int gc = 8 * pg + j + t % 3 - 1;
                v[j] = (gc >= 0 && gc < kImg) ? *reinterpret_cast<const uint4*>(src + raw_off<CIN>(gc, kc))
                                              : make_uint4(0u, 0u, 0u, 0u);
            }
            transpose8x8_bf16(v, o);
            const int r0 = t * CIN + kc * 8;
            uint4* dst = reinterpret_cast<uint4*>(smem + (r0 >> 3) * L::SBO + pg * 128);
#pragma unroll
            for (int k = 0; k < 8; ++k) dst[k] = o[k];
        }
        // B core matrices: (channel block mc, pixel group pg) = transpose of dz[pixels][channels]
        for (int i = tid; i < ZCH * (L::P / 8); i += kWgradThreads) {
            const int pg = i % (L::P / 8), mc = i / (L::P / 8);
            const unsigned char* src = smem + L::ZR_OFF + lr * L::ZROW;
            uint4 v[8], o[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = *reinterpret_cast<const uint4*>(src + raw_off<M>(8 * pg + j, mc));
            transpose8x8_bf16(v, o);
            uint4* dst = reinterpret_cast<uint4*>(smem + L::B_OFF + mc * L::SBO + pg * 128);
#pragma unroll
            for (int k = 0; k < 8; ++k) dst[k] = o[k];
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (tid == 0) {
            const uint32_t base = smem_u32(smem);
#pragma unroll 1
            for (int tile = 0; tile < L::TILES; ++tile)
#pragma unroll
                for (int s = 0; s < L::P / 16; ++s) {
                    const uint32_t a = base + tile * (128 / 8) * L::SBO + 2 * s * 128;
                    const uint32_t b = base + L::B_OFF + 2 * s * 128;
                    umma_bf16(tmem + tile * M, umma_desc(a, 128, L::SBO), umma_desc(b, 128, L::SBO), idesc,
                              (lr > 0 || s > 0) ? 1u : 0u);
                }
            umma_commit(mbar);
        }
        // the operands are rewritten for the next row only after these MMAs have read them
        bool done = false;
        for (int it = 0; it < kMmaWaitLimit && !done; ++it) done = mbar_try_wait(mbar, phase);
        phase ^= 1u;
        if (!done) {
            ok = false;
            if ((tid & 31) == 0) atomicOr(status, kStatusMmaTimeout);
        }
        tc_fence_after();
        __syncthreads();
    }
    if (ok) {
        float* pw = part_w + (int64_t)blockIdx.x * (MSTORE * 9 * CIN);
#pragma unroll 1
        for (int tile = 0; tile < L::TILES; ++tile) {
            const int r = tile * 128 + tid;  // this thread's accumulator row
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + tile * M;
            float v[32];
            if constexpr (M == 32) tmem_ld32(taddr, v);
            else tmem_ld16(taddr, v);
            if (r < 9 * CIN) {
                const int t = r / CIN, k = r % CIN;
#pragma unroll
                for (int m = 0; m < MSTORE; ++m) pw[(m * 9 + t) * CIN + k] = v[m];
            } else if (r == 9 * CIN) {
#pragma unroll
                for (int m = 0; m < MSTORE; ++m) part_b[(int64_t)blockIdx.x * MSTORE + m] = v[m];
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(L::TMEM_COLS)
                     : "memory");
    }
}

// Sum of the per-CTA partials in a fixed order: grad[e] for the weights (nw elements) then the
// biases (nb elements).  A CTA of 32 x kReduceSplit threads covers 32 elements: thread (lane, g)
// sums the partials g, g + kReduceSplit, ... of element lane in that order (coalesced across
// lanes), and lane's kReduceSplit sums are then added in order of g.
constexpr int kReduceSplit = 32;
__global__ void __launch_bounds__(32 * kReduceSplit) wgrad_reduce_kernel(const float* __restrict__ part_w,
                                                                       const float* __restrict__ part_b, int nparts,
                                                                       int nw, int nb, float* __restrict__ gw,
                                                                       float* __restrict__ gb) {
    __shared__ float sums[kReduceSplit][32];
    const int lane = threadIdx.x & 31, g = threadIdx.x >> 5;
    const int e = blockIdx.x * 32 + lane;
    const bool is_w = e < nw;
    const int j = is_w ? e : e - nw;
    const float* src = is_w ? part_w : part_b;
    const int stride = is_w ? nw : nb;
    float s = 0.0f;
    if (e < nw + nb) {
#pragma unroll 4
        for (int c = g; c < nparts; c += kReduceSplit) s += src[(int64_t)c * stride + j];
    }
    sums[g][lane] = s;
    __syncthreads();
    if (g == 0 && e < nw + nb) {
        float t = sums[0][lane];
#pragma unroll
        for (int k = 1; k < kReduceSplit; ++k) t += sums[k][lane];
        (is_w ? gw : gb)[j] = t;
    }
}

}  // namespace cnn
}  // namespace sbp
