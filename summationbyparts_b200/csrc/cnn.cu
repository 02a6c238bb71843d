// The learned correction of the coarse solve: a small convolutional network that maps the
// coarse-grid (64 x 64) state at the end time toward the restriction of a fine-grid solve, its
// training on the GPU (forward, backward, Adam) and the restriction operator that makes the
// training targets.  No counterpart in the reference; see cnn_kernels.cuh for the kernels.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "cnn_kernels.cuh"
#include "common.h"

using namespace sbp;
using namespace sbp::cnn;

namespace {

constexpr int kLayers = 5;
constexpr int kCinP[kLayers] = {16, 32, 32, 32, 32};   // stored input channels
constexpr int kCoutP[kLayers] = {32, 32, 32, 32, 8};   // stored output channels (weights' rows)
constexpr int kCinReal[kLayers] = {4, 32, 32, 32, 32};
constexpr int kCoutReal[kLayers] = {32, 32, 32, 32, 4};
constexpr int kDzP[kLayers] = {32, 32, 32, 32, 16};    // stored channels of each layer's output gradient

// Elementwise kernels around the network ----------------------------------------------------

// a0[n][p][c] = (state[n][c][p] - mean[c]) * inv[c] for c < 4, 0 for the 12 padding channels.
template <class T>
__global__ void pack_input_kernel(const T* __restrict__ st, int64_t img_stride, int n, float4 mean, float4 inv,
                                  __nv_bfloat16* __restrict__ a0) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)n * kPix) return;
    const int64_t img = i / kPix, p = i % kPix;
    const T* s = st + img * img_stride + p;
    const float v0 = (float(s[0]) - mean.x) * inv.x, v1 = (float(s[kPix]) - mean.y) * inv.y;
    const float v2 = (float(s[2 * kPix]) - mean.z) * inv.z, v3 = (float(s[3 * kPix]) - mean.w) * inv.w;
    uint4 lo, hi = make_uint4(0u, 0u, 0u, 0u);
    lo.x = pack_bf16(v0, v1);
    lo.y = pack_bf16(v2, v3);
    lo.z = 0u;
    lo.w = 0u;
    uint4* d = reinterpret_cast<uint4*>(a0 + i * 16);
    d[0] = lo;
    d[1] = hi;
}

// Loss and output gradient: t = (fine_r - coarse) / out_scale per channel, the squared error
// summed per CTA into part (CTA order), dy = 2 (y - t) / count into dz4 (16 channels, zeros
// above 4).
template <class T>
__global__ void loss_kernel(const float* __restrict__ y, const T* __restrict__ coarse, int64_t img_stride,
                            const double* __restrict__ fine_r, int n, float4 oscale, float inv_count,
                            __nv_bfloat16* __restrict__ dz4, float* __restrict__ part) {
    __shared__ float red[256];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    float se = 0.0f;
    if (i < (int64_t)n * kPix) {
        const int64_t img = i / kPix, p = i % kPix;
        const T* c = coarse + img * img_stride + p;
        const double* f = fine_r + img * 4 * kPix + p;
        const float sc[4] = {oscale.x, oscale.y, oscale.z, oscale.w};
        float g[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float t = float(f[k * kPix] - double(c[k * kPix])) / sc[k];
            const float d = y[i * 8 + k] - t;
            se += d * d;
            g[k] = 2.0f * d * inv_count;
        }
        uint4 lo, hi = make_uint4(0u, 0u, 0u, 0u);
        lo.x = pack_bf16(g[0], g[1]);
        lo.y = pack_bf16(g[2], g[3]);
        lo.z = 0u;
        lo.w = 0u;
        uint4* d = reinterpret_cast<uint4*>(dz4 + i * 16);
        d[0] = lo;
        d[1] = hi;
    }
    red[threadIdx.x] = se;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// corrected[n][c][p] = coarse[n][c][p] + y[n][p][c] * out_scale[c]  (f64 output planes)
template <class T>
__global__ void apply_kernel(const float* __restrict__ y, const T* __restrict__ coarse, int64_t img_stride, int n,
                             float4 oscale, double* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)n * kPix) return;
    const int64_t img = i / kPix, p = i % kPix;
    const T* c = coarse + img * img_stride + p;
    double* o = out + img * 4 * kPix + p;
    const float sc[4] = {oscale.x, oscale.y, oscale.z, oscale.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) o[k * kPix] = double(c[k * kPix]) + double(y[i * 8 + k]) * double(sc[k]);
}

// Adam (Kingma & Ba) on one layer's weights (nw elements, [cout][9][cin]) and biases (nb), with
// the bias corrections c1 = 1 / (1 - beta1^t), c2 = 1 / (1 - beta2^t) from the host.  Writes the
// bf16 weights and, when wt is given, the bf16 weights of the gradient convolution:
// wt[ci][8 - tap][co] (dz channels dzp) = w[co][tap][ci].
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int nw, int nb, float lr, float b1, float b2, float c1, float c2,
                            float eps, int cout, int cin, int dzp, __nv_bfloat16* __restrict__ wb,
                            __nv_bfloat16* __restrict__ wt) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nw + nb) return;
    const float ge = g[e];
    const float me = b1 * m[e] + (1.0f - b1) * ge;
    const float ve = b2 * v[e] + (1.0f - b2) * ge * ge;
    m[e] = me;
    v[e] = ve;
    const float pe = p[e] - lr * (me * c1) / (sqrtf(ve * c2) + eps);
    p[e] = pe;
    if (e < nw) {
        const __nv_bfloat16 h = __float2bfloat16_rn(pe);
        wb[e] = h;
        if (wt) {
            const int co = e / (9 * cin), tap = (e / cin) % 9, ci = e % cin;
            wt[((int64_t)ci * 9 + (8 - tap)) * dzp + co] = h;
        }
    }
}

// bf16 copies of the parameters (after set_params)
__global__ void weights_bf16_kernel(const float* __restrict__ p, int nw, int cout, int cin, int dzp,
                                    __nv_bfloat16* __restrict__ wb, __nv_bfloat16* __restrict__ wt) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nw) return;
    const __nv_bfloat16 h = __float2bfloat16_rn(p[e]);
    wb[e] = h;
    if (wt) {
        const int co = e / (9 * cin), tap = (e / cin) % 9, ci = e % cin;
        wt[((int64_t)ci * 9 + (8 - tap)) * dzp + co] = h;
    }
}

// Tensor-product restriction: out[n][c][i][j] = sum_a sum_b wy[i][a] wx[j][b] f[n][c][iy[i]+a][ix[j]+b]
// with 6-point stencils (index base per coarse index in idx, weights in w).
__global__ void restrict_kernel(const double* __restrict__ fine, int nf, int nc, int n, const int* __restrict__ base,
                                const double* __restrict__ w, double* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t per = (int64_t)nc * nc;
    if (i >= (int64_t)n * 4 * per) return;
    const int64_t plane = i / per;
    const int r = (int)((i % per) / nc), c = (int)(i % nc);
    const double* f = fine + plane * (int64_t)nf * nf;
    double s = 0.0;
    for (int a = 0; a < 6; ++a) {
        const double* fr = f + (int64_t)(base[r] + a) * nf + base[c];
        double t = 0.0;
        for (int b = 0; b < 6; ++b) t += w[c * 6 + b] * fr[b];
        s += w[r * 6 + a] * t;
    }
    out[i] = s;
}

// Per image relative L2 difference: out[k] = |a_k - b_k| / |b_k| over 4 planes of np points.
template <class TA, class TB>
__global__ void rel_l2_kernel(const TA* __restrict__ a, int64_t sa, const TB* __restrict__ b, int64_t sb, int64_t np,
                              double* __restrict__ out) {
    __shared__ double rd[256], rn[256];
    const int img = blockIdx.x;
    double d2 = 0.0, n2 = 0.0;
    for (int64_t k = threadIdx.x; k < 4 * np; k += blockDim.x) {
        const double bv = double(b[img * sb + k]);
        const double dv = double(a[img * sa + k]) - bv;
        d2 += dv * dv;
        n2 += bv * bv;
    }
    rd[threadIdx.x] = d2;
    rn[threadIdx.x] = n2;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            rd[threadIdx.x] += rd[threadIdx.x + s];
            rn[threadIdx.x] += rn[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[img] = sqrt(rd[0]) / sqrt(rn[0]);
}

// Host-side pieces ------------------------------------------------------------------------

uint64_t splitmix64(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Lagrange weights of the 6 nodes xs[0..5] at x.
void lagrange6(const double* xs, double x, double* w) {
    for (int a = 0; a < 6; ++a) {
        double v = 1.0;
        for (int b = 0; b < 6; ++b)
            if (b != a) v *= (x - xs[b]) / (xs[a] - xs[b]);
        w[a] = v;
    }
}

}  // namespace

struct sbp_cnn {
    int device = 0;
    int max_batch = 0;
    cudaStream_t own = nullptr, user = nullptr;
    bool has_user = false;
    int64_t w_off[kLayers], b_off[kLayers], nw[kLayers], nparams = 0;
    float *P = nullptr, *G = nullptr, *Mo = nullptr, *Ve = nullptr;
    __nv_bfloat16 *Wb[kLayers] = {}, *Wt[kLayers] = {};
    __nv_bfloat16* a[kLayers] = {};   // layer inputs
    float* z[kLayers - 1] = {};       // hidden pre-activations
    float* y = nullptr;               // output [B][kPix][8]
    __nv_bfloat16* dz[kLayers] = {};  // output gradients
    float *part_w = nullptr, *part_b = nullptr, *part_loss = nullptr;
    unsigned* status = nullptr;       // device status word of the tensor-core kernels
    float4 in_mean{0, 0, 0, 0}, in_inv{1, 1, 1, 1}, out_scale{1, 1, 1, 1};
    int adam_t = 0;
    std::vector<void*> allocs;
    cudaStream_t st() const { return has_user ? user : own; }
};

namespace {

template <int CIN, int COUT, int EPI>
cudaError_t conv(const sbp_cnn* c, int n, const __nv_bfloat16* x, const __nv_bfloat16* w, const float* bias,
                 const float* zprev, float* zout, __nv_bfloat16* yout) {
    constexpr int bytes = ConvTcLayout<CIN, COUT>::BYTES;
    static bool configured = false;  // per instantiation; the attribute is per function
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(conv3x3_tc_kernel<CIN, COUT, EPI>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    conv3x3_tc_kernel<CIN, COUT, EPI><<<n * (kImg / kBand), kConvThreads, bytes, c->st()>>>(x, w, bias, zprev, zout,
                                                                                            yout, c->status);
    return cudaGetLastError();
}

// The device status word after the stream has drained: a tensor-core wait that gave up.
sbp_status device_status(sbp_cnn* c) {
    unsigned h = 0;
    SBP_TRY_CUDA(cudaMemcpyAsync(&h, c->status, sizeof h, cudaMemcpyDeviceToHost, c->st()));
    SBP_TRY_CUDA(cudaStreamSynchronize(c->st()));
    if (h & kStatusMmaTimeout) {
        set_error("a convolution's tensor-core work did not complete in time");
        return SBP_ERR_CUDA;
    }
    return SBP_OK;
}

template <int CIN, int M, int MSTORE>
cudaError_t wgrad(const sbp_cnn* c, int n, int layer, const __nv_bfloat16* x, const __nv_bfloat16* dz) {
    const int parts = n * (kImg / kWgradRows);
    constexpr int bytes = WgradTcLayout<CIN, M>::BYTES;
    static bool configured = false;  // per instantiation; the attribute is per function
    if (!configured) {
        const cudaError_t e = cudaFuncSetAttribute(wgrad_tc_kernel<CIN, M, MSTORE>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    wgrad_tc_kernel<CIN, M, MSTORE><<<parts, kWgradThreads, bytes, c->st()>>>(x, dz, c->part_w, c->part_b, c->status);
    const int nw = MSTORE * 9 * CIN, nb = MSTORE;
    wgrad_reduce_kernel<<<(nw + nb + 31) / 32, 32 * kReduceSplit, 0, c->st()>>>(
        c->part_w, c->part_b, parts, nw, nb, c->G + c->w_off[layer], c->G + c->b_off[layer]);
    return cudaGetLastError();
}

sbp_status check_batch(const sbp_cnn* c, int n) {
    if (!c || n <= 0 || n > c->max_batch) {
        set_error("batch %d outside 1..%d", n, c ? c->max_batch : 0);
        return SBP_ERR_INVALID_ARGUMENT;
    }
    return SBP_OK;
}

sbp_status forward(sbp_cnn* c, int n, const void* state, int dtype, int64_t img_stride) {
    const int64_t total = (int64_t)n * kPix;
    const int blocks = (int)((total + 255) / 256);
    if (dtype == SBP_F64)
        pack_input_kernel<double><<<blocks, 256, 0, c->st()>>>(static_cast<const double*>(state), img_stride, n,
                                                               c->in_mean, c->in_inv, c->a[0]);
    else
        pack_input_kernel<float><<<blocks, 256, 0, c->st()>>>(static_cast<const float*>(state), img_stride, n,
                                                              c->in_mean, c->in_inv, c->a[0]);
    SBP_TRY_CUDA(cudaGetLastError());
    const float* P = c->P;
    SBP_TRY_CUDA((conv<16, 32, EPI_GELU>(c, n, c->a[0], c->Wb[0], P + c->b_off[0], nullptr, c->z[0], c->a[1])));
    for (int l = 1; l < 4; ++l)
        SBP_TRY_CUDA(
            (conv<32, 32, EPI_GELU>(c, n, c->a[l], c->Wb[l], P + c->b_off[l], nullptr, c->z[l], c->a[l + 1])));
    SBP_TRY_CUDA((conv<32, 8, EPI_LINEAR>(c, n, c->a[4], c->Wb[4], P + c->b_off[4], nullptr, c->y, nullptr)));
    return SBP_OK;
}

// Loss and gradients of all parameters into G; the loss (mean squared error of the normalised
// correction) to *loss if given (synchronises the stream).
sbp_status backward(sbp_cnn* c, int n, const void* coarse, int dtype, int64_t img_stride, const double* fine_r,
                    float* loss) {
    const int64_t total = (int64_t)n * kPix;
    const int blocks = (int)((total + 255) / 256);
    const float inv_count = 1.0f / float(total * 4);
    if (dtype == SBP_F64)
        loss_kernel<double><<<blocks, 256, 0, c->st()>>>(c->y, static_cast<const double*>(coarse), img_stride, fine_r,
                                                         n, c->out_scale, inv_count, c->dz[4], c->part_loss);
    else
        loss_kernel<float><<<blocks, 256, 0, c->st()>>>(c->y, static_cast<const float*>(coarse), img_stride, fine_r,
                                                        n, c->out_scale, inv_count, c->dz[4], c->part_loss);
    SBP_TRY_CUDA(cudaGetLastError());
    SBP_TRY_CUDA((wgrad<32, 16, 8>(c, n, 4, c->a[4], c->dz[4])));
    SBP_TRY_CUDA((conv<16, 32, EPI_DGELU>(c, n, c->dz[4], c->Wt[4], nullptr, c->z[3], nullptr, c->dz[3])));
    for (int l = 3; l >= 1; --l) {
        SBP_TRY_CUDA((wgrad<32, 32, 32>(c, n, l, c->a[l], c->dz[l])));
        SBP_TRY_CUDA((conv<32, 32, EPI_DGELU>(c, n, c->dz[l], c->Wt[l], nullptr, c->z[l - 1], nullptr, c->dz[l - 1])));
    }
    SBP_TRY_CUDA((wgrad<16, 32, 32>(c, n, 0, c->a[0], c->dz[0])));
    if (loss) {
        std::vector<float> h(blocks);
        SBP_TRY_CUDA(cudaMemcpyAsync(h.data(), c->part_loss, blocks * sizeof(float), cudaMemcpyDeviceToHost, c->st()));
        SBP_TRY(device_status(c));
        double s = 0.0;
        for (float v : h) s += v;
        *loss = float(s / double(total * 4));
    }
    return SBP_OK;
}

sbp_status refresh_bf16(sbp_cnn* c) {
    for (int l = 0; l < kLayers; ++l) {
        const int nw = (int)c->nw[l];
        weights_bf16_kernel<<<(nw + 255) / 256, 256, 0, c->st()>>>(c->P + c->w_off[l], nw, kCoutP[l], kCinP[l],
                                                                  kDzP[l], c->Wb[l], l > 0 ? c->Wt[l] : nullptr);
        SBP_TRY_CUDA(cudaGetLastError());
    }
    return SBP_OK;
}

}  // namespace

extern "C" {

sbp_status sbp_cnn_create(int device, int max_batch, unsigned long long seed, sbp_cnn** out) {
    clear_error();
    if (!out || max_batch <= 0 || max_batch > 4096) {
        set_error("max_batch %d outside 1..4096", max_batch);
        return SBP_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    SBP_TRY_CUDA(cudaSetDevice(device));
    sbp_cnn* c = new sbp_cnn;
    c->device = device;
    c->max_batch = max_batch;
    auto fail = [&](sbp_status s) {
        for (void* p : c->allocs) cudaFree(p);
        if (c->own) cudaStreamDestroy(c->own);
        delete c;
        return s;
    };
    if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess)
        return fail(cuda_status(cudaGetLastError(), "stream"));
    for (int l = 0; l < kLayers; ++l) {
        c->nw[l] = (int64_t)kCoutP[l] * 9 * kCinP[l];
        c->w_off[l] = c->nparams;
        c->b_off[l] = c->nparams + c->nw[l];
        c->nparams += c->nw[l] + kCoutP[l];
    }
    auto alloc = [&](void** p, size_t bytes) {
        cudaError_t e = cudaMalloc(p, bytes);
        if (e == cudaSuccess) {
            c->allocs.push_back(*p);
            e = cudaMemsetAsync(*p, 0, bytes, c->own);
        }
        return e;
    };
    const int64_t B = max_batch;
    cudaError_t e = cudaSuccess;
    e = e ?: alloc((void**)&c->P, c->nparams * 4);
    e = e ?: alloc((void**)&c->G, c->nparams * 4);
    e = e ?: alloc((void**)&c->Mo, c->nparams * 4);
    e = e ?: alloc((void**)&c->Ve, c->nparams * 4);
    for (int l = 0; l < kLayers; ++l) {
        e = e ?: alloc((void**)&c->Wb[l], c->nw[l] * 2);
        if (l > 0) e = e ?: alloc((void**)&c->Wt[l], (int64_t)kCinP[l] * 9 * kDzP[l] * 2);
        e = e ?: alloc((void**)&c->a[l], B * kPix * kCinP[l] * 2);
        e = e ?: alloc((void**)&c->dz[l], B * kPix * kDzP[l] * 2);
        if (l < 4) e = e ?: alloc((void**)&c->z[l], B * kPix * 32 * 4);
    }
    e = e ?: alloc((void**)&c->y, B * kPix * 8 * 4);
    e = e ?: alloc((void**)&c->part_w, B * (kImg / kWgradRows) * (32 * 9 * 32) * 4);
    e = e ?: alloc((void**)&c->part_b, B * (kImg / kWgradRows) * 32 * 4);
    e = e ?: alloc((void**)&c->part_loss, (B * kPix + 255) / 256 * 4);
    e = e ?: alloc((void**)&c->status, sizeof(unsigned));
    if (e != cudaSuccess) return fail(cuda_status(e, "network allocation"));
    // He-style initialisation for the GELU layers, a small output layer so the initial
    // correction is close to zero; padded entries stay zero.
    std::vector<float> h(c->nparams, 0.0f);
    uint64_t s = seed;
    for (int l = 0; l < kLayers; ++l) {
        const double fan_in = 9.0 * kCinReal[l];
        const double a = std::sqrt(6.0 / fan_in) * (l == kLayers - 1 ? 0.1 : 1.0);
        for (int co = 0; co < kCoutP[l]; ++co)
            for (int t = 0; t < 9; ++t)
                for (int ci = 0; ci < kCinP[l]; ++ci) {
                    const double u = double(splitmix64(s) >> 11) * 0x1.0p-53;
                    if (co < kCoutReal[l] && ci < kCinReal[l])
                        h[c->w_off[l] + ((int64_t)co * 9 + t) * kCinP[l] + ci] = float((2.0 * u - 1.0) * a);
                }
    }
    e = cudaMemcpyAsync(c->P, h.data(), c->nparams * 4, cudaMemcpyHostToDevice, c->own);
    if (e != cudaSuccess) return fail(cuda_status(e, "parameter upload"));
    sbp_status rs = refresh_bf16(c);
    if (rs != SBP_OK) return fail(rs);
    e = cudaStreamSynchronize(c->own);
    if (e != cudaSuccess) return fail(cuda_status(e, "network set-up"));
    *out = c;
    return SBP_OK;
}

sbp_status sbp_cnn_destroy(sbp_cnn* c) {
    clear_error();
    if (!c) return SBP_OK;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->st());
    for (void* p : c->allocs) cudaFree(p);
    if (c->own) cudaStreamDestroy(c->own);
    delete c;
    return SBP_OK;
}

sbp_status sbp_cnn_set_stream(sbp_cnn* c, void* stream) {
    clear_error();
    if (!c) return SBP_ERR_INVALID_ARGUMENT;
    // NULL is the legacy default stream (handle 0), as for a kernel launch: a caller that works
    // on the default stream must get its work ordered there, not on the network's own stream.
    c->user = static_cast<cudaStream_t>(stream);
    c->has_user = true;
    return SBP_OK;
}

int64_t sbp_cnn_param_count(const sbp_cnn* c) { return c ? c->nparams : -1; }

sbp_status sbp_cnn_set_normalisation(sbp_cnn* c, const float* in_mean, const float* in_scale, const float* out_scale) {
    clear_error();
    if (!c || !in_mean || !in_scale || !out_scale) return SBP_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < 4; ++k)
        if (!(in_scale[k] > 0.0f) || !(out_scale[k] > 0.0f)) {
            set_error("scales must be positive");
            return SBP_ERR_INVALID_ARGUMENT;
        }
    c->in_mean = make_float4(in_mean[0], in_mean[1], in_mean[2], in_mean[3]);
    c->in_inv = make_float4(1.0f / in_scale[0], 1.0f / in_scale[1], 1.0f / in_scale[2], 1.0f / in_scale[3]);
    c->out_scale = make_float4(out_scale[0], out_scale[1], out_scale[2], out_scale[3]);
    return SBP_OK;
}

sbp_status sbp_cnn_get_params(sbp_cnn* c, float* host) {
    clear_error();
    if (!c || !host) return SBP_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    SBP_TRY_CUDA(cudaMemcpyAsync(host, c->P, c->nparams * 4, cudaMemcpyDeviceToHost, c->st()));
    SBP_TRY_CUDA(cudaStreamSynchronize(c->st()));
    return SBP_OK;
}

sbp_status sbp_cnn_set_params(sbp_cnn* c, const float* host) {
    clear_error();
    if (!c || !host) return SBP_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    SBP_TRY_CUDA(cudaMemcpyAsync(c->P, host, c->nparams * 4, cudaMemcpyHostToDevice, c->st()));
    SBP_TRY(refresh_bf16(c));
    SBP_TRY_CUDA(cudaStreamSynchronize(c->st()));
    c->adam_t = 0;
    SBP_TRY_CUDA(cudaMemsetAsync(c->Mo, 0, c->nparams * 4, c->st()));
    SBP_TRY_CUDA(cudaMemsetAsync(c->Ve, 0, c->nparams * 4, c->st()));
    return SBP_OK;
}

sbp_status sbp_cnn_forward(sbp_cnn* c, int n, const void* d_coarse, int dtype, int64_t img_stride) {
    clear_error();
    SBP_TRY(check_batch(c, n));
    if (!d_coarse || (dtype != SBP_F64 && dtype != SBP_F32) || img_stride < 4 * kPix) return SBP_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    return forward(c, n, d_coarse, dtype, img_stride);
}

sbp_status sbp_cnn_output(sbp_cnn* c, int n, float* d_y) {
    clear_error();
    SBP_TRY(check_batch(c, n));
    if (!d_y) return SBP_ERR_INVALID_ARGUMENT;
    SBP_TRY_CUDA(cudaMemcpyAsync(d_y, c->y, (size_t)n * kPix * 8 * 4, cudaMemcpyDeviceToDevice, c->st()));
    return SBP_OK;
}

sbp_status sbp_cnn_gradients(sbp_cnn* c, int n, const void* d_coarse, int dtype, int64_t img_stride,
                             const double* d_fine_r, float* loss, float* host_grads) {
    clear_error();
    SBP_TRY(check_batch(c, n));
    if (!d_coarse || !d_fine_r || (dtype != SBP_F64 && dtype != SBP_F32) || img_stride < 4 * kPix)
        return SBP_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    SBP_TRY(forward(c, n, d_coarse, dtype, img_stride));
    SBP_TRY(backward(c, n, d_coarse, dtype, img_stride, d_fine_r, loss));
    if (host_grads) {
        SBP_TRY_CUDA(cudaMemcpyAsync(host_grads, c->G, c->nparams * 4, cudaMemcpyDeviceToHost, c->st()));
        SBP_TRY(device_status(c));
    }
    return SBP_OK;
}

sbp_status sbp_cnn_train_step(sbp_cnn* c, int n, const void* d_coarse, int dtype, int64_t img_stride,
                              const double* d_fine_r, float lr, float* loss) {
    clear_error();
    if (!(lr > 0.0f)) return SBP_ERR_INVALID_ARGUMENT;
    SBP_TRY(sbp_cnn_gradients(c, n, d_coarse, dtype, img_stride, d_fine_r, loss, nullptr));
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    c->adam_t += 1;
    const float c1 = float(1.0 / (1.0 - std::pow(double(b1), c->adam_t)));
    const float c2 = float(1.0 / (1.0 - std::pow(double(b2), c->adam_t)));
    for (int l = 0; l < kLayers; ++l) {
        const int nw = (int)c->nw[l], nb = kCoutP[l];
        // weights and biases of a layer are adjacent in P / G / Mo / Ve
        adam_kernel<<<(nw + nb + 255) / 256, 256, 0, c->st()>>>(c->P + c->w_off[l], c->G + c->w_off[l],
                                                                c->Mo + c->w_off[l], c->Ve + c->w_off[l], nw, nb, lr,
                                                                b1, b2, c1, c2, eps, kCoutP[l], kCinP[l], kDzP[l],
                                                                c->Wb[l], l > 0 ? c->Wt[l] : nullptr);
        SBP_TRY_CUDA(cudaGetLastError());
    }
    return SBP_OK;
}

sbp_status sbp_cnn_apply(sbp_cnn* c, int n, const void* d_coarse, int dtype, int64_t img_stride, double* d_out) {
    clear_error();
    SBP_TRY(sbp_cnn_forward(c, n, d_coarse, dtype, img_stride));
    if (!d_out) return SBP_ERR_INVALID_ARGUMENT;
    const int64_t total = (int64_t)n * kPix;
    const int blocks = (int)((total + 255) / 256);
    if (dtype == SBP_F64)
        apply_kernel<double><<<blocks, 256, 0, c->st()>>>(c->y, static_cast<const double*>(d_coarse), img_stride, n,
                                                          c->out_scale, d_out);
    else
        apply_kernel<float><<<blocks, 256, 0, c->st()>>>(c->y, static_cast<const float*>(d_coarse), img_stride, n,
                                                         c->out_scale, d_out);
    SBP_TRY_CUDA(cudaGetLastError());
    return SBP_OK;
}

sbp_status sbp_cnn_synchronize(sbp_cnn* c) {
    clear_error();
    if (!c) return SBP_ERR_INVALID_ARGUMENT;
    SBP_TRY_CUDA(cudaStreamSynchronize(c->st()));
    return device_status(c);
}

sbp_status sbp_restrict_linspace(int n, int nf, int nc, const double* d_fine, double* d_coarse, void* stream) {
    clear_error();
    if (n <= 0 || nf < 6 || nc < 2 || nc > nf || !d_fine || !d_coarse) {
        set_error("bad restriction arguments (n %d, fine %d, coarse %d)", n, nf, nc);
        return SBP_ERR_INVALID_ARGUMENT;
    }
    // nodes x_j = j / (nf - 1) (the common linspace scaled to [0, 1]); target X_i = i / (nc - 1)
    std::vector<int> base(nc);
    std::vector<double> w(6 * nc);
    for (int i = 0; i < nc; ++i) {
        const double X = double(i) / double(nc - 1);
        const double pos = X * double(nf - 1);
        int b = (int)std::floor(pos) - 2;
        if (b < 0) b = 0;
        if (b > nf - 6) b = nf - 6;
        double xs[6];
        for (int a = 0; a < 6; ++a) xs[a] = double(b + a) / double(nf - 1);
        base[i] = b;
        lagrange6(xs, X, &w[6 * i]);
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int* d_base = nullptr;
    double* d_w = nullptr;
    SBP_TRY_CUDA(cudaMallocAsync((void**)&d_base, nc * sizeof(int), st));
    SBP_TRY_CUDA(cudaMallocAsync((void**)&d_w, 6 * nc * sizeof(double), st));
    SBP_TRY_CUDA(cudaMemcpyAsync(d_base, base.data(), nc * sizeof(int), cudaMemcpyHostToDevice, st));
    SBP_TRY_CUDA(cudaMemcpyAsync(d_w, w.data(), 6 * nc * sizeof(double), cudaMemcpyHostToDevice, st));
    const int64_t total = (int64_t)n * 4 * nc * nc;
    restrict_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(d_fine, nf, nc, n, d_base, d_w, d_coarse);
    cudaError_t e = cudaGetLastError();
    cudaFreeAsync(d_base, st);
    cudaFreeAsync(d_w, st);
    SBP_TRY_CUDA(e);
    SBP_TRY_CUDA(cudaStreamSynchronize(st));
    return SBP_OK;
}

sbp_status sbp_rel_l2_images(int n, int64_t points, const void* d_a, int dtype_a, int64_t stride_a, const void* d_b,
                             int dtype_b, int64_t stride_b, double* d_out, void* stream) {
    clear_error();
    if (n <= 0 || points <= 0 || !d_a || !d_b || !d_out || stride_a < 4 * points || stride_b < 4 * points ||
        (dtype_a != SBP_F64 && dtype_a != SBP_F32) || (dtype_b != SBP_F64 && dtype_b != SBP_F32))
        return SBP_ERR_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (dtype_a == SBP_F64 && dtype_b == SBP_F64)
        rel_l2_kernel<double, double><<<n, 256, 0, st>>>(static_cast<const double*>(d_a), stride_a,
                                                         static_cast<const double*>(d_b), stride_b, points, d_out);
    else if (dtype_a == SBP_F32 && dtype_b == SBP_F64)
        rel_l2_kernel<float, double><<<n, 256, 0, st>>>(static_cast<const float*>(d_a), stride_a,
                                                        static_cast<const double*>(d_b), stride_b, points, d_out);
    else if (dtype_a == SBP_F64 && dtype_b == SBP_F32)
        rel_l2_kernel<double, float><<<n, 256, 0, st>>>(static_cast<const double*>(d_a), stride_a,
                                                        static_cast<const float*>(d_b), stride_b, points, d_out);
    else
        rel_l2_kernel<float, float><<<n, 256, 0, st>>>(static_cast<const float*>(d_a), stride_a,
                                                       static_cast<const float*>(d_b), stride_b, points, d_out);
    SBP_TRY_CUDA(cudaGetLastError());
    return SBP_OK;
}

}  // extern "C"
