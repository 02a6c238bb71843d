// Launchers of the system-level kernels (system_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "euler_device.cuh"

namespace sbp {

// Metrics::new combine step (sbp/src/grid.rs:101-130): from the four derivative planes build
// detj, J dxi/dx = y_eta, J dxi/dy = -x_eta, J deta/dx = -y_xi, J deta/dy = x_xi into `out`
// (5 planes spaced `pstride`); sets STATUS_DETJ in *status if detj <= 0 anywhere.
cudaError_t metrics_combine(const double* x_xi, const double* x_eta, const double* y_xi, const double* y_eta,
                            int64_t n, double* out, int64_t pstride, unsigned* status, cudaStream_t st);

// Narrow f64 planes to f32 (n elements).
cudaError_t narrow_f32(const double* in, float* out, int64_t n, cudaStream_t st);
// Plane 0 (J) of every block's f32 metrics replaced by 1 / J, rounded from the f64 quotient.
cudaError_t jacobian_inverse_f32(const BlockDev* blocks, int nblocks, const double* met64, float* met32,
                                 int64_t max_points, cudaStream_t st);

// Vortex initial data for every block whose instance is selected (instance < 0: all).
// f64 state: q_hi only.  f32 state: (hi, lo) split of the f64 value.
cudaError_t vortex_init(const BlockDev* blocks, const InstanceDev* inst, int nblocks, int instance, double gamma,
                        double t, const double* xy, int prec, void* q_hi, void* q_lo, int64_t max_points,
                        cudaStream_t st);

// Partial sums per block of the norm kernels below (the `partials` buffers hold
// kNormParts * nblocks doubles).
constexpr int kNormParts = 128;

// Field::h2_err terms against the vortex at each block's instance time: block_sums[b] = sum of
// (q - vortex)^2 hx hy over the block (euler/src/lib.rs:377-431).  Each CTA writes a partial
// sum and the partials are added in a fixed order, so the result is the same on every run.
cudaError_t error_terms(const BlockDev* blocks, const InstanceDev* inst, int nblocks, double gamma,
                        const double* xy, int prec, const void* q_hi, const void* q_lo, const double* hweights,
                        const int64_t* h_off, int64_t max_points, double* block_sums, double* partials,
                        cudaStream_t st);

// Field::h2_err of one block's state against a dense (4, ny, nx) f64 field: *sum = terms
// (partials: kNormParts doubles).
cudaError_t diff_terms(const BlockDev* block, const InstanceDev* inst, int prec, const void* q_hi, const void* q_lo,
                       const double* dense, const double* hx, const double* hy, int64_t max_points, double* sum,
                       double* partials, cudaStream_t st);

// max |uhat|, max |vhat| per block (multigrid/src/system.rs:555-580), as ordered bit patterns.
cudaError_t max_speeds(const BlockDev* blocks, const InstanceDev* inst, int nblocks, int prec, const void* q_hi,
                       const void* q_lo, const double* met64, int64_t max_points, unsigned long long* out2,
                       cudaStream_t st);

// One explicit Runge-Kutta combination (utils/integrate/src/lib.rs:193-211):
// out = base; out = out + (coef[j] * dt) * k[j] for j = 0 .. nk-1 with coef[j] != 0, in that
// order (Field::scaled_add, euler/src/lib.rs:205-212), dt = the block's instance dt or dt_fixed
// when dt_fixed >= 0.  Over the padded planes of every block; out may be base.
constexpr int kMaxStages = 8;
struct StageCombination {
    double coef[kMaxStages];
    const double* k[kMaxStages];
    int nk;
    double dt_fixed;
};
cudaError_t combine_stages(const BlockDev* blocks, const InstanceDev* inst, int nblocks, const double* base,
                           double* out, const StageCombination& cm, int64_t max_points, cudaStream_t st);

// time[i] += dt[i] for the instances whose flag is set.
cudaError_t time_update(InstanceDev* inst, const int* active, int ninst, cudaStream_t st);

// Packed host layout (blocks concatenated, each (4, ny, nx) dense) <-> padded device planes.
// The packed state is the absolute state; a compensated system's planes hold its deviation from
// each instance's reference state (InstanceDev::qref), converted in f64.
// dtype of the packed buffer: 0 = f64,
//                              1 = f32 hi planes followed by lo planes per block (hi + lo = state).
cudaError_t pack_state(const BlockDev* blocks, const InstanceDev* inst, int nblocks, const int64_t* packed_off,
                       int prec, int dtype, const void* q_hi, const void* q_lo, void* packed, int64_t max_points,
                       cudaStream_t st);
cudaError_t unpack_state(const BlockDev* blocks, const InstanceDev* inst, int nblocks, const int64_t* packed_off,
                         int prec, int dtype, const void* packed, void* q_hi, void* q_lo, int64_t max_points,
                         cudaStream_t st);

// Free-stream dissipation plane of one block of a compensated upwind system:
// rinf = (diss_xi(alpha_u,r) + diss_eta(alpha_v,r)) / detJ in f64, stored as f32 at the block's
// r_off, where alpha_u,r / alpha_v,r are the upwind dissipation coefficients at the instance's
// reference state (euler/src/lib.rs:619-674).  The stage kernels add q_r * rinf to k.
// `work` holds 4 nx ny doubles.
cudaError_t free_stream_dissipation(const BlockDev* block, const InstanceDev* inst, double gamma, int op_xi,
                                    int op_eta, int nx, int ny, const double* met64, double* work, float* rinf,
                                    cudaStream_t st);

}  // namespace sbp
