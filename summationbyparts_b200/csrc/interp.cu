// sbp_interpolate: the interface interpolation operators applied to batches of lines
// (InterpolationOperator::fine2coarse / coarse2fine, sbp/src/operators.rs:108-113).  Built with
// -fmad=false so every product is rounded before its add, as in the reference.
#include <cuda_runtime.h>

#include "common.h"
#include "interp.cuh"

namespace {

template <class T>
__global__ void interp_kernel(int op, bool f2c, const T* __restrict__ in, T* __restrict__ out, int64_t nin,
                              int64_t nout, int64_t nbatch, int64_t in_stride, int64_t out_stride) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nout * nbatch) return;
    const int64_t b = idx / nout, i = idx % nout;
    const sbp::InterpDev<T> I = sbp::interp_dev<T>(op, f2c);
    const T* line = in + b * in_stride;
    out[b * out_stride + i] = sbp::interp_at<T>(I, i, nin, nout, [&](int64_t k) { return line[k]; });
}

}  // namespace

extern "C" sbp_status sbp_interpolate(int op, int fine2coarse, int dtype, const void* d_in, void* d_out, int64_t n_in,
                                      int64_t n_out, int64_t nbatch, int64_t in_stride, int64_t out_stride,
                                      void* stream) {
    using namespace sbp;
    clear_error();
    if (op < 0 || op > 3 || !d_in || !d_out || nbatch < 1 || (dtype != SBP_F64 && dtype != SBP_F32)) {
        set_error("bad interpolation operator, dtype or pointer");
        return SBP_ERR_INVALID_ARGUMENT;
    }
    const bool f2c = fine2coarse != 0;
    if (f2c ? !interp_sizes_ok(op, n_in, n_out) : !interp_sizes_ok(op, n_out, n_in)) {
        set_error("interpolation %s from %lld to %lld points breaks the operator's size relation",
                  f2c ? "fine2coarse" : "coarse2fine", (long long)n_in, (long long)n_out);
        return SBP_ERR_SHAPE;
    }
    if (in_stride < n_in || out_stride < n_out) {
        set_error("strides smaller than the lines");
        return SBP_ERR_SHAPE;
    }
    if (!interp_reads_in_range(op, f2c, n_in, n_out)) {
        set_error("interpolation from %lld to %lld points reads beyond the input line", (long long)n_in,
                  (long long)n_out);
        return SBP_ERR_SHAPE;
    }
    const int64_t total = n_out * nbatch;
    const unsigned blocks = (unsigned)((total + 255) / 256);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (dtype == SBP_F64)
        interp_kernel<double><<<blocks, 256, 0, st>>>(op, f2c, static_cast<const double*>(d_in),
                                                      static_cast<double*>(d_out), n_in, n_out, nbatch, in_stride,
                                                      out_stride);
    else
        interp_kernel<float><<<blocks, 256, 0, st>>>(op, f2c, static_cast<const float*>(d_in),
                                                     static_cast<float*>(d_out), n_in, n_out, nbatch, in_stride,
                                                     out_stride);
    SBP_TRY_CUDA(cudaGetLastError());
    return SBP_OK;
}
