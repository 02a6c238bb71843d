// System-level kernels: metric assembly, vortex data, error norms, CFL speeds, time update and
// state packing.  Compiled with -fmad=false so the f64 arithmetic matches the reference's.
#include <cuda_runtime.h>

#include "op_apply.h"
#include "system_kernels.h"

namespace sbp {

namespace {

constexpr int kT = 256;

__global__ void metrics_combine_kernel(const double* __restrict__ x_xi, const double* __restrict__ x_eta,
                                       const double* __restrict__ y_xi, const double* __restrict__ y_eta, int64_t n,
                                       double* __restrict__ out, int64_t ps, unsigned* status) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double a = x_xi[i], b = x_eta[i], c = y_xi[i], d = y_eta[i];
        const double detj = a * d - b * c;
        if (!(detj > 0.0)) atomicOr(status, STATUS_DETJ);
        out[i] = detj;
        out[ps + i] = d;
        out[2 * ps + i] = -b;
        out[3 * ps + i] = -c;
        out[4 * ps + i] = a;
    }
}

__global__ void narrow_kernel(const double* __restrict__ in, float* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = float(in[i]);
}

__device__ __forceinline__ void split_f32(double v, float& hi, float& lo) {
    hi = float(v);
    lo = float(v - double(hi));
}

// Store the absolute f64 state value v at element g: as is in f64, as the (hi, lo) split of its
// deviation from the instance's reference state in the compensated form.
__device__ __forceinline__ void store_state(int prec, void* q_hi, void* q_lo, int64_t g, double v, double qref) {
    if (prec == 0) {
        static_cast<double*>(q_hi)[g] = v;
    } else {
        float h, l;
        split_f32(v - qref, h, l);
        static_cast<float*>(q_hi)[g] = h;
        static_cast<float*>(q_lo)[g] = l;
    }
}

__global__ void vortex_init_kernel(const BlockDev* __restrict__ blocks, const InstanceDev* __restrict__ inst,
                                   int instance, double gamma, double t, const double* __restrict__ xy, int prec,
                                   void* q_hi, void* q_lo) {
    const BlockDev& B = blocks[blockIdx.y];
    if (instance >= 0 && B.instance != instance) return;
    const int64_t n = (int64_t)B.nx * B.ny, np = B.npad;
    const InstanceDev& I = inst[B.instance];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double q[4];
        vortex_point(I, gamma, t, xy[B.x_off + i], xy[B.x_off + np + i], q);
        for (int c = 0; c < 4; ++c) store_state(prec, q_hi, q_lo, B.q_off + c * np + i, q[c], I.qref[c]);
    }
}

// Absolute state at element g (qref: the instance's reference value of the component, added to
// the stored deviation in the compensated form; hi + lo is exact in f64).
__device__ __forceinline__ double state_at(int prec, const void* q_hi, const void* q_lo, int64_t g, double qref) {
    if (prec == 0) return static_cast<const double*>(q_hi)[g];
    return qref + (double(static_cast<const float*>(q_hi)[g]) + double(static_cast<const float*>(q_lo)[g]));
}

__global__ void error_kernel(const BlockDev* __restrict__ blocks, const InstanceDev* __restrict__ inst, double gamma,
                             const double* __restrict__ xy, int prec, const void* q_hi, const void* q_lo,
                             const double* __restrict__ hw, const int64_t* __restrict__ h_off,
                             double* __restrict__ partials) {
    const int b = blockIdx.y;
    const BlockDev& B = blocks[b];
    const int64_t n = (int64_t)B.nx * B.ny, np = B.npad;
    const InstanceDev& I = inst[B.instance];
    const double* hx = hw + h_off[b];
    const double* hy = hx + B.nx;
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int row = (int)(i / B.nx), col = (int)(i - (int64_t)row * B.nx);
        double v[4];
        vortex_point(I, gamma, I.time, xy[B.x_off + i], xy[B.x_off + np + i], v);
        for (int c = 0; c < 4; ++c) {
            const double d = state_at(prec, q_hi, q_lo, B.q_off + c * np + i, I.qref[c]) - v[c];
            s += d * d * hx[col] * hy[row];
        }
    }
    // block reduction
    __shared__ double red[kT / 32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (kT / 32) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) partials[(int64_t)b * gridDim.x + blockIdx.x] = s;
    }
}

__global__ void diff_kernel(const BlockDev* __restrict__ blk, const InstanceDev* __restrict__ inst, int prec,
                            const void* q_hi, const void* q_lo, const double* __restrict__ dense,
                            const double* __restrict__ hx, const double* __restrict__ hy,
                            double* __restrict__ partials) {
    const BlockDev& B = *blk;
    const InstanceDev& I = inst[B.instance];
    const int64_t n = (int64_t)B.nx * B.ny, np = B.npad;
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int row = (int)(i / B.nx), col = (int)(i - (int64_t)row * B.nx);
        for (int c = 0; c < 4; ++c) {
            const double d = state_at(prec, q_hi, q_lo, B.q_off + c * np + i, I.qref[c]) - dense[c * n + i];
            s += d * d * hx[col] * hy[row];
        }
    }
    __shared__ double red[kT / 32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (kT / 32) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) partials[blockIdx.x] = s;
    }
}

// out[j] = sum of partials[j * nper .. j * nper + nper) in index order: the norms come out the
// same on every run (no floating-point atomics).
__global__ void sum_partials_kernel(const double* __restrict__ partials, int nper, int nsum, double* __restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nsum) return;
    double s = 0.0;
    for (int k = 0; k < nper; ++k) s += partials[(int64_t)j * nper + k];
    out[j] = s;
}

__global__ void max_speed_kernel(const BlockDev* __restrict__ blocks, const InstanceDev* __restrict__ inst, int prec,
                                 const void* q_hi, const void* q_lo, const double* __restrict__ met64,
                                 unsigned long long* out) {
    const int b = blockIdx.y;
    const BlockDev& B = blocks[b];
    const InstanceDev& I = inst[B.instance];
    const int64_t n = (int64_t)B.nx * B.ny, np = B.npad;
    double mu = 0.0, mv = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double rho = state_at(prec, q_hi, q_lo, B.q_off + i, I.qref[0]);
        const double rhou = state_at(prec, q_hi, q_lo, B.q_off + np + i, I.qref[1]);
        const double rhov = state_at(prec, q_hi, q_lo, B.q_off + 2 * np + i, I.qref[2]);
        const double* m = met64 + B.m_off;
        const double u = rhou / rho, v = rhov / rho;
        const double uhat = m[np + i] * u + m[2 * np + i] * v;
        const double vhat = m[3 * np + i] * u + m[4 * np + i] * v;
        mu = fmax(mu, fabs(uhat));
        mv = fmax(mv, fabs(vhat));
    }
    for (int o = 16; o > 0; o >>= 1) {
        mu = fmax(mu, __shfl_down_sync(0xffffffffu, mu, o));
        mv = fmax(mv, __shfl_down_sync(0xffffffffu, mv, o));
    }
    if ((threadIdx.x & 31) == 0) {
        // non-negative doubles order like their bit patterns
        atomicMax(out + 2 * b, (unsigned long long)__double_as_longlong(mu));
        atomicMax(out + 2 * b + 1, (unsigned long long)__double_as_longlong(mv));
    }
}

__global__ void combine_kernel(const BlockDev* __restrict__ blocks, const InstanceDev* __restrict__ inst,
                               const double* base, double* out, StageCombination cm) {
    const BlockDev& B = blocks[blockIdx.y];
    const double dt = cm.dt_fixed >= 0.0 ? cm.dt_fixed : inst[B.instance].dt;
    double sc[kMaxStages];
#pragma unroll
    for (int j = 0; j < kMaxStages; ++j) sc[j] = cm.coef[j] * dt;  // (a * dt), then times k
    const int64_t n4 = 4 * (int64_t)B.npad;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n4; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t g = B.q_off + i;
        double v = base[g];
        for (int j = 0; j < cm.nk; ++j)
            if (cm.coef[j] != 0.0) v = v + sc[j] * cm.k[j][g];
        out[g] = v;
    }
}

__global__ void time_update_kernel(InstanceDev* inst, const int* __restrict__ active, int ninst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ninst && active[i]) inst[i].time = inst[i].time + inst[i].dt;
}

__global__ void pack_kernel(const BlockDev* __restrict__ blocks, const InstanceDev* __restrict__ inst,
                            const int64_t* __restrict__ poff, int prec, int dtype, const void* q_hi, const void* q_lo,
                            void* packed) {
    const BlockDev& B = blocks[blockIdx.y];
    const InstanceDev& I = inst[B.instance];
    const int64_t n = (int64_t)B.nx * B.ny, np = B.npad;
    const int64_t o = poff[blockIdx.y];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        for (int c = 0; c < 4; ++c) {
            const double v = state_at(prec, q_hi, q_lo, B.q_off + c * np + i, I.qref[c]);
            if (dtype == 0) {
                static_cast<double*>(packed)[o + c * n + i] = v;
            } else {
                float* p = static_cast<float*>(packed) + o;
                float h, l;
                split_f32(v, h, l);
                p[c * n + i] = h;
                p[4 * n + c * n + i] = l;
            }
        }
    }
}

__global__ void unpack_kernel(const BlockDev* __restrict__ blocks, const InstanceDev* __restrict__ inst,
                              const int64_t* __restrict__ poff, int prec, int dtype, const void* packed, void* q_hi,
                              void* q_lo) {
    const BlockDev& B = blocks[blockIdx.y];
    const InstanceDev& I = inst[B.instance];
    const int64_t n = (int64_t)B.nx * B.ny, np = B.npad;
    const int64_t o = poff[blockIdx.y];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        for (int c = 0; c < 4; ++c) {
            double v;
            if (dtype == 0) {
                v = static_cast<const double*>(packed)[o + c * n + i];
            } else {
                const float* p = static_cast<const float*>(packed) + o;
                v = double(p[c * n + i]) + double(p[4 * n + c * n + i]);
            }
            store_state(prec, q_hi, q_lo, B.q_off + c * np + i, v, I.qref[c]);
        }
    }
}

// alpha_u and alpha_v of the compensated form's reference state on one block's metrics
// (upwind_dissipation, euler/src/lib.rs:619-674, at q = q_r), with the metrics rounded to f32
// as the stage kernels read them, into dense (ny, nx) planes.
__global__ void alpha_ref_kernel(const BlockDev* __restrict__ blk, const InstanceDev* __restrict__ inst, double gamma,
                                 const double* __restrict__ met64, double* __restrict__ au, double* __restrict__ av) {
    const BlockDev& B = *blk;
    const InstanceDev& I = inst[B.instance];
    const int64_t n = (int64_t)B.nx * B.ny, np = B.npad;
    const double* m = met64 + B.m_off;
    const double ur = double(I.ref.u), vr = double(I.ref.v), cr = double(I.ref.c);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double jxx = float(m[np + i]), jxy = float(m[2 * np + i]);
        const double jyx = float(m[3 * np + i]), jyy = float(m[4 * np + i]);
        au[i] = fabs(jxx * ur + jxy * vr) + cr * sqrt(jxx * jxx + jxy * jxy);
        av[i] = fabs(jyx * ur + jyy * vr) + cr * sqrt(jyx * jyx + jyy * jyy);
    }
}

// rinf = (diss_xi(alpha_u,r) + diss_eta(alpha_v,r)) / detJ, narrowed to f32, at the block's r_off.
__global__ void rinf_kernel(const BlockDev* __restrict__ blk, const double* __restrict__ met64,
                            const double* __restrict__ dxi, const double* __restrict__ deta, float* __restrict__ rinf) {
    const BlockDev& B = *blk;
    const int64_t n = (int64_t)B.nx * B.ny;
    const double* detj = met64 + B.m_off;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        rinf[B.r_off + i] = float((dxi[i] + deta[i]) / detj[i]);
}

dim3 per_block_grid(int nblocks, int64_t max_points) {
    int64_t gx = (max_points + kT - 1) / kT;
    if (gx > 1024) gx = 1024;
    if (gx < 1) gx = 1;
    return dim3((unsigned)gx, (unsigned)nblocks, 1);
}

// Grid of the norm kernels: at most kNormParts CTAs per block, each writing one partial sum.
dim3 norm_grid(int nblocks, int64_t max_points) {
    dim3 g = per_block_grid(nblocks, max_points);
    if (g.x > (unsigned)kNormParts) g.x = kNormParts;
    return g;
}

int flat_grid(int64_t n) {
    int64_t g = (n + kT - 1) / kT;
    if (g > 148 * 32) g = 148 * 32;
    return (int)(g < 1 ? 1 : g);
}

}  // namespace

cudaError_t metrics_combine(const double* x_xi, const double* x_eta, const double* y_xi, const double* y_eta,
                            int64_t n, double* out, int64_t pstride, unsigned* status, cudaStream_t st) {
    metrics_combine_kernel<<<flat_grid(n), kT, 0, st>>>(x_xi, x_eta, y_xi, y_eta, n, out, pstride, status);
    return cudaGetLastError();
}

cudaError_t narrow_f32(const double* in, float* out, int64_t n, cudaStream_t st) {
    narrow_kernel<<<flat_grid(n), kT, 0, st>>>(in, out, n);
    return cudaGetLastError();
}

// The single-precision metrics of the compensated stage kernels: plane 0 holds 1 / J (rounded
// once from the f64 quotient), so the flux divergence is scaled by a product; planes 1-2 (J dxi/dx,
// J dxi/dy) are multiplied by the block's xi spacing factor idx_xi and planes 3-4 by idx_eta (in
// f64, then rounded), so every stencil input of a direction carries its factor and the stencil
// sums need no final scaling (the operators are linear and the dissipation coefficients are
// homogeneous of degree one in the metrics).
__global__ void jacobian_inverse_kernel(const BlockDev* __restrict__ blocks, const double* __restrict__ met64,
                                        float* __restrict__ met32) {
    const BlockDev& B = blocks[blockIdx.y];
    const int64_t n = (int64_t)B.nx * B.ny, np = B.npad;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double* m = met64 + B.m_off + i;
        float* o = met32 + B.m_off + i;
        const double j = m[0];
        o[0] = j != 0.0 ? float(1.0 / j) : 0.0f;
        o[np] = float(m[np] * B.idx_xi);
        o[2 * np] = float(m[2 * np] * B.idx_xi);
        o[3 * np] = float(m[3 * np] * B.idx_eta);
        o[4 * np] = float(m[4 * np] * B.idx_eta);
    }
}

cudaError_t jacobian_inverse_f32(const BlockDev* blocks, int nblocks, const double* met64, float* met32,
                                 int64_t max_points, cudaStream_t st) {
    jacobian_inverse_kernel<<<per_block_grid(nblocks, max_points), kT, 0, st>>>(blocks, met64, met32);
    return cudaGetLastError();
}

cudaError_t vortex_init(const BlockDev* blocks, const InstanceDev* inst, int nblocks, int instance, double gamma,
                        double t, const double* xy, int prec, void* q_hi, void* q_lo, int64_t max_points,
                        cudaStream_t st) {
    vortex_init_kernel<<<per_block_grid(nblocks, max_points), kT, 0, st>>>(blocks, inst, instance, gamma, t, xy, prec,
                                                                          q_hi, q_lo);
    return cudaGetLastError();
}

cudaError_t error_terms(const BlockDev* blocks, const InstanceDev* inst, int nblocks, double gamma,
                        const double* xy, int prec, const void* q_hi, const void* q_lo, const double* hweights,
                        const int64_t* h_off, int64_t max_points, double* block_sums, double* partials,
                        cudaStream_t st) {
    const dim3 g = norm_grid(nblocks, max_points);
    error_kernel<<<g, kT, 0, st>>>(blocks, inst, gamma, xy, prec, q_hi, q_lo, hweights, h_off, partials);
    sum_partials_kernel<<<(nblocks + kT - 1) / kT, kT, 0, st>>>(partials, (int)g.x, nblocks, block_sums);
    return cudaGetLastError();
}

cudaError_t diff_terms(const BlockDev* block, const InstanceDev* inst, int prec, const void* q_hi, const void* q_lo,
                       const double* dense, const double* hx, const double* hy, int64_t max_points, double* sum,
                       double* partials, cudaStream_t st) {
    const dim3 g = norm_grid(1, max_points);
    diff_kernel<<<g.x, kT, 0, st>>>(block, inst, prec, q_hi, q_lo, dense, hx, hy, partials);
    sum_partials_kernel<<<1, 32, 0, st>>>(partials, (int)g.x, 1, sum);
    return cudaGetLastError();
}

cudaError_t max_speeds(const BlockDev* blocks, const InstanceDev* inst, int nblocks, int prec, const void* q_hi,
                       const void* q_lo, const double* met64, int64_t max_points, unsigned long long* out2,
                       cudaStream_t st) {
    max_speed_kernel<<<per_block_grid(nblocks, max_points), kT, 0, st>>>(blocks, inst, prec, q_hi, q_lo, met64, out2);
    return cudaGetLastError();
}

cudaError_t combine_stages(const BlockDev* blocks, const InstanceDev* inst, int nblocks, const double* base,
                           double* out, const StageCombination& cm, int64_t max_points, cudaStream_t st) {
    combine_kernel<<<per_block_grid(nblocks, 4 * max_points), kT, 0, st>>>(blocks, inst, base, out, cm);
    return cudaGetLastError();
}

cudaError_t free_stream_dissipation(const BlockDev* block, const InstanceDev* inst, double gamma, int op_xi,
                                    int op_eta, int nx, int ny, const double* met64, double* work, float* rinf,
                                    cudaStream_t st) {
    const int64_t n = (int64_t)nx * ny;
    double* au = work;
    double* av = work + n;
    double* dxi = work + 2 * n;
    double* deta = work + 3 * n;
    alpha_ref_kernel<<<flat_grid(n), kT, 0, st>>>(block, inst, gamma, met64, au, av);
    cudaError_t e = cudaGetLastError();
    e = e ?: op_apply(op_xi, 0, 1, 0, au, dxi, ny, nx, 1, n, st);
    e = e ?: op_apply(op_eta, 1, 1, 0, av, deta, ny, nx, 1, n, st);
    if (e != cudaSuccess) return e;
    rinf_kernel<<<flat_grid(n), kT, 0, st>>>(block, met64, dxi, deta, rinf);
    return cudaGetLastError();
}

cudaError_t time_update(InstanceDev* inst, const int* active, int ninst, cudaStream_t st) {
    time_update_kernel<<<(ninst + kT - 1) / kT, kT, 0, st>>>(inst, active, ninst);
    return cudaGetLastError();
}

cudaError_t pack_state(const BlockDev* blocks, const InstanceDev* inst, int nblocks, const int64_t* packed_off,
                       int prec, int dtype, const void* q_hi, const void* q_lo, void* packed, int64_t max_points,
                       cudaStream_t st) {
    pack_kernel<<<per_block_grid(nblocks, max_points), kT, 0, st>>>(blocks, inst, packed_off, prec, dtype, q_hi,
                                                                   q_lo, packed);
    return cudaGetLastError();
}

cudaError_t unpack_state(const BlockDev* blocks, const InstanceDev* inst, int nblocks, const int64_t* packed_off,
                         int prec, int dtype, const void* packed, void* q_hi, void* q_lo, int64_t max_points,
                         cudaStream_t st) {
    unpack_kernel<<<per_block_grid(nblocks, max_points), kT, 0, st>>>(blocks, inst, packed_off, prec, dtype, packed,
                                                                     q_hi, q_lo);
    return cudaGetLastError();
}

}  // namespace sbp
