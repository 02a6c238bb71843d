// Grid metrics without any device allocation.
//
// sbp_metrics takes its working memory (the four derivative planes x_xi, x_eta, y_xi, y_eta
// and a status word) from cudaMallocAsync.  Some callers cannot allocate device memory at the
// point where they need metrics: hosts whose device memory belongs to another runtime's pool
// or arena (a Rust or Fortran solver that hands out only its own buffers, a framework whose
// caching allocator must not be bypassed), and time-critical loops that forbid allocator calls
// because an allocation can synchronise the device and has no bounded latency.
// sbp_metrics_noalloc gives them the same results with the working memory taken from a fixed,
// file-scope device array instead, so the call itself allocates nothing.
//
// Cost and limits, stated once here:
//  * The array holds grids of up to kNoAllocMaxPoints points (512 x 512) and occupies
//    8 MiB + 256 B on every GPU that loads this library, until the process exits.
//  * All calls share it and it keeps the last call's contents; the status word is cleared at
//    the start of every call.  Calls whose GPU work overlaps (two host threads, or two streams
//    without ordering between them) race on the array and must not be issued.
//  * The first call on each device looks up the array's device address with
//    cudaGetSymbolAddress while that device is current; make that first call before any
//    stream capture.  The address is kept for the life of the process, so the entry point must
//    not be used on a device after cudaDeviceReset (which unloads the module holding the array).
#include <cuda_runtime.h>

#include <mutex>

#include "common.h"
#include "op_apply.h"
#include "system_kernels.h"

namespace {

constexpr int64_t kNoAllocMaxPoints = 512 * 512;
// four f64 derivative planes, then the status word (padded to 256 bytes)
constexpr int64_t kScratchDoubles = 4 * kNoAllocMaxPoints + 32;

static __device__ __align__(256) double g_metrics_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
double* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once per device).
sbp_status scratch_on_current_device(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return sbp::cuda_status(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) {
        sbp::set_error("device %d beyond the %d devices the scratch table covers", dev, kMaxDevices);
        return SBP_ERR_INVALID_ARGUMENT;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_metrics_scratch);
        if (e != cudaSuccess) return sbp::cuda_status(e, "cudaGetSymbolAddress of the metrics scratch");
        g_scratch_addr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_addr[dev];
    return SBP_OK;
}

}  // namespace

extern "C" sbp_status sbp_metrics_noalloc(int op_xi, int op_eta, const double* d_x, const double* d_y, int64_t ny,
                                          int64_t nx, double* d_metrics, void* stream) {
    using namespace sbp;
    clear_error();
    OpInfo ox, oe;
    if (!op_info(op_xi, ox) || !op_info(op_eta, oe) || !d_x || !d_y || !d_metrics) {
        set_error("bad operator or null pointer");
        return SBP_ERR_INVALID_ARGUMENT;
    }
    if (nx < 2 * ox.M || nx < ox.N || ny < 2 * oe.M || ny < oe.N) {
        set_error("grid %lld x %lld too small for the operators", (long long)ny, (long long)nx);
        return SBP_ERR_SHAPE;
    }
    // each side is bounded before the product is formed, so no shape can overflow it
    if (nx > kNoAllocMaxPoints || ny > kNoAllocMaxPoints / nx) {
        set_error("grid %lld x %lld has more than %lld points, all the fixed scratch of sbp_metrics_noalloc holds "
                  "(use sbp_metrics)",
                  (long long)ny, (long long)nx, (long long)kNoAllocMaxPoints);
        return SBP_ERR_SHAPE;
    }
    double* scratch = nullptr;
    SBP_TRY(scratch_on_current_device(&scratch));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t n = nx * ny;
    double* tmp = scratch;
    unsigned* status = reinterpret_cast<unsigned*>(scratch + 4 * kNoAllocMaxPoints);
    SBP_TRY_CUDA(cudaMemsetAsync(status, 0, sizeof(unsigned), st));
    SBP_TRY_CUDA(op_apply(op_xi, 0, 0, 0, d_x, tmp, ny, nx, 1, n, st));
    SBP_TRY_CUDA(op_apply(op_eta, 1, 0, 0, d_x, tmp + n, ny, nx, 1, n, st));
    SBP_TRY_CUDA(op_apply(op_xi, 0, 0, 0, d_y, tmp + 2 * n, ny, nx, 1, n, st));
    SBP_TRY_CUDA(op_apply(op_eta, 1, 0, 0, d_y, tmp + 3 * n, ny, nx, 1, n, st));
    SBP_TRY_CUDA(metrics_combine(tmp, tmp + n, tmp + 2 * n, tmp + 3 * n, n, d_metrics, n, status, st));
    unsigned hs = 0;
    SBP_TRY_CUDA(cudaMemcpyAsync(&hs, status, sizeof hs, cudaMemcpyDeviceToHost, st));
    SBP_TRY_CUDA(cudaStreamSynchronize(st));
    if (hs) {
        set_error("non-positive Jacobian determinant");
        return SBP_ERR_NONPHYSICAL;
    }
    return SBP_OK;
}
