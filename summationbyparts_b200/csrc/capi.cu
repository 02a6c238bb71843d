// C ABI: library info, operator tables and the standalone operator / metric entry points.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>

#include "common.h"
#include "op_apply.h"
#include "sbp_coefficients.h"
#include "system_kernels.h"

namespace sbp {

namespace {
thread_local std::string g_error;

#define HTAB(TAG)                                                                 \
    static const double h_##TAG##_H[] = {SBPC_##TAG##_H(SBPC_LIT_F64)};            \
    static const double h_##TAG##_DS[] = {SBPC_##TAG##_DIFF_START(SBPC_LIT_F64)};  \
    static const double h_##TAG##_DD[] = {SBPC_##TAG##_DIFF_DIAG(SBPC_LIT_F64)};
#define HTAB_DISS(TAG)                                                            \
    static const double h_##TAG##_SS[] = {SBPC_##TAG##_DISS_START(SBPC_LIT_F64)};  \
    static const double h_##TAG##_SD[] = {SBPC_##TAG##_DISS_DIAG(SBPC_LIT_F64)};
HTAB(UPWIND4)
HTAB(UPWIND4H2)
HTAB(UPWIND9)
HTAB(UPWIND9H2)
HTAB(SBP4)
HTAB(SBP8)
HTAB_DISS(UPWIND4)
HTAB_DISS(UPWIND4H2)
HTAB_DISS(UPWIND9)
HTAB_DISS(UPWIND9H2)

struct HostOp {
    OpInfo info;
    const double *h, *ds, *dd, *ss, *sd;
};

bool host_op(int op, HostOp& o) {
#define HOP(ID, TAG, H2, UPW, SS, SD)                                                             \
    case ID:                                                                                      \
        o = HostOp{{SBPC_##TAG##_M, SBPC_##TAG##_N, SBPC_##TAG##_D, H2, UPW}, h_##TAG##_H,      \
                   h_##TAG##_DS, h_##TAG##_DD, SS, SD};                                           \
        return true;
    switch (op) {
        HOP(SBP_OP_UPWIND4, UPWIND4, false, true, h_UPWIND4_SS, h_UPWIND4_SD)
        HOP(SBP_OP_UPWIND4H2, UPWIND4H2, true, true, h_UPWIND4H2_SS, h_UPWIND4H2_SD)
        HOP(SBP_OP_UPWIND9, UPWIND9, false, true, h_UPWIND9_SS, h_UPWIND9_SD)
        HOP(SBP_OP_UPWIND9H2, UPWIND9H2, true, true, h_UPWIND9H2_SS, h_UPWIND9H2_SD)
        HOP(SBP_OP_SBP4, SBP4, false, false, nullptr, nullptr)
        HOP(SBP_OP_SBP8, SBP8, false, false, nullptr, nullptr)
        default: return false;
    }
#undef HOP
}
}  // namespace

void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_error = buf;
}

void clear_error() { g_error.clear(); }

bool op_info(int op, OpInfo& out) {
    HostOp o;
    if (!host_op(op, o)) return false;
    out = o.info;
    return true;
}

const double* op_h_weights(int op) {
    HostOp o;
    return host_op(op, o) ? o.h : nullptr;
}

// Stage-kernel coefficient table (layout of coef_base in stage_kernel.cuh): for each operator
// and kind, [start M rows][end M rows][diagonal], each row `row` elements (zero padded),
// stride `stride` elements.
// prec 0 writes doubles; prec 1 writes floats rounded from the f32 literals.
#define FTAB(TAG)                                                                 \
    static const float f_##TAG##_DS[] = {SBPC_##TAG##_DIFF_START(SBPC_LIT_F32)};   \
    static const float f_##TAG##_DD[] = {SBPC_##TAG##_DIFF_DIAG(SBPC_LIT_F32)};
#define FTAB_DISS(TAG)                                                            \
    static const float f_##TAG##_SS[] = {SBPC_##TAG##_DISS_START(SBPC_LIT_F32)};   \
    static const float f_##TAG##_SD[] = {SBPC_##TAG##_DISS_DIAG(SBPC_LIT_F32)};
FTAB(UPWIND4)
FTAB(UPWIND4H2)
FTAB(UPWIND9)
FTAB(UPWIND9H2)
FTAB(SBP4)
FTAB(SBP8)
FTAB_DISS(UPWIND4)
FTAB_DISS(UPWIND4H2)
FTAB_DISS(UPWIND9)
FTAB_DISS(UPWIND9H2)

template <class T>
static void fill_one(T* out, const T* st, const T* dg, int M, int N, int D, bool diff, int row) {
    for (int i = 0; i < M; ++i)
        for (int k = 0; k < N; ++k) out[i * row + k] = st[i * N + k];
    for (int i = 0; i < M; ++i)
        for (int k = 0; k < N; ++k) {
            const T v = st[(M - 1 - i) * N + (N - 1 - k)];
            out[(M + i) * row + k] = diff ? -v : v;
        }
    for (int d = 0; d < D; ++d) out[2 * M * row + d] = dg[d];
}

void fill_coef_table(int prec, void* out, int stride, int row) {
    struct F {
        const float *ds, *dd, *ss, *sd;
    };
    const F ft[6] = {{f_UPWIND4_DS, f_UPWIND4_DD, f_UPWIND4_SS, f_UPWIND4_SD},
                     {f_UPWIND4H2_DS, f_UPWIND4H2_DD, f_UPWIND4H2_SS, f_UPWIND4H2_SD},
                     {f_UPWIND9_DS, f_UPWIND9_DD, f_UPWIND9_SS, f_UPWIND9_SD},
                     {f_UPWIND9H2_DS, f_UPWIND9H2_DD, f_UPWIND9H2_SS, f_UPWIND9H2_SD},
                     {f_SBP4_DS, f_SBP4_DD, nullptr, nullptr},
                     {f_SBP8_DS, f_SBP8_DD, nullptr, nullptr}};
    for (int op = 0; op < 6; ++op) {
        HostOp o;
        host_op(op, o);
        const int M = o.info.M, N = o.info.N, D = o.info.D;
        for (int kind = 0; kind < 2; ++kind) {
            const size_t base = (size_t)(2 * op + kind) * stride;
            if (prec == 0) std::fill((double*)out + base, (double*)out + base + stride, 0.0);
            else std::fill((float*)out + base, (float*)out + base + stride, 0.0f);
            if (kind == 1 && !o.info.upwind) continue;
            if (prec == 0)
                fill_one<double>((double*)out + base, kind ? o.ss : o.ds, kind ? o.sd : o.dd, M, N, D, kind == 0, row);
            else
                fill_one<float>((float*)out + base, kind ? ft[op].ss : ft[op].ds, kind ? ft[op].sd : ft[op].dd, M, N,
                                D, kind == 0, row);
        }
    }
}

}  // namespace sbp

using namespace sbp;

namespace {

sbp_status apply_common(int op, int dir, int kind, int dtype, const void* in, void* out, int64_t ny, int64_t nx,
                        int64_t nbatch, int64_t bstride, void* stream) {
    clear_error();
    OpInfo oi;
    if (!op_info(op, oi)) {
        set_error("unknown operator %d", op);
        return SBP_ERR_INVALID_ARGUMENT;
    }
    if (dtype != SBP_F64 && dtype != SBP_F32) {
        set_error("unknown dtype %d", dtype);
        return SBP_ERR_INVALID_ARGUMENT;
    }
    if (kind == 1 && !oi.upwind) {
        set_error("operator %d has no dissipation (not an upwind operator)", op);
        return SBP_ERR_UNSUPPORTED;
    }
    if (!in || !out || ny <= 0 || nx <= 0 || nbatch <= 0) {
        set_error("null pointer or empty shape");
        return SBP_ERR_INVALID_ARGUMENT;
    }
    if (in == out) {
        set_error("prev and fut must not alias");
        return SBP_ERR_INVALID_ARGUMENT;
    }
    const int64_t n = dir == 0 ? nx : ny;
    if (n < 2 * oi.M || n < oi.N) {
        set_error("length %lld along the operator direction is below max(2M, N) = %d", (long long)n,
                  2 * oi.M > oi.N ? 2 * oi.M : oi.N);
        return SBP_ERR_SHAPE;
    }
    if (ny > INT32_MAX || nx > INT32_MAX || ny * nx > bstride && nbatch > 1) {
        set_error("bad shape / batch stride");
        return SBP_ERR_SHAPE;
    }
    cudaError_t e = op_apply(op, dir, kind, dtype, in, out, ny, nx, nbatch, nbatch > 1 ? bstride : ny * nx,
                             static_cast<cudaStream_t>(stream));
    return cuda_status(e, "operator kernel launch");
}

}  // namespace

extern "C" {

const char* sbp_last_error(void) { return sbp::g_error.c_str(); }

const char* sbp_version(void) { return "sbp_b200 0.1.0 (sm_100a)"; }

int sbp_operator_h(int op, double* h, int cap) {
    HostOp o;
    if (!host_op(op, o) || !h) return -1;
    const int m = o.info.M;
    for (int i = 0; i < m && i < cap; ++i) h[i] = o.h[i];
    return m;
}

int sbp_operator_is_h2(int op) {
    OpInfo oi;
    return op_info(op, oi) ? (oi.h2 ? 1 : 0) : -1;
}

int sbp_operator_is_upwind(int op) {
    OpInfo oi;
    return op_info(op, oi) ? (oi.upwind ? 1 : 0) : -1;
}

int sbp_operator_table(int op, int kind, int part, double* out, int cap) {
    HostOp o;
    if (!host_op(op, o) || !out) return -1;
    if (kind == 1 && !o.info.upwind) return -1;
    const double* st = kind == 0 ? o.ds : o.ss;
    const double* dg = kind == 0 ? o.dd : o.sd;
    const int M = o.info.M, N = o.info.N, D = o.info.D;
    if (part == 0) {
        if (cap < M * N) return -1;
        for (int i = 0; i < M * N; ++i) out[i] = st[i];
        return M * N;
    }
    if (part == 1) {
        if (cap < D) return -1;
        for (int i = 0; i < D; ++i) out[i] = dg[i];
        return D;
    }
    if (part == 2) {
        if (cap < M * N) return -1;
        for (int i = 0; i < M; ++i)
            for (int k = 0; k < N; ++k) {
                const double v = st[(M - 1 - i) * N + (N - 1 - k)];
                out[i * N + k] = kind == 0 ? -v : v;
            }
        return M * N;
    }
    return -1;
}

sbp_status sbp_diffxi(int op, int dtype, const void* d_prev, void* d_fut, int64_t ny, int64_t nx, int64_t nbatch,
                      int64_t batch_stride, void* stream) {
    return apply_common(op, 0, 0, dtype, d_prev, d_fut, ny, nx, nbatch, batch_stride, stream);
}

sbp_status sbp_diffeta(int op, int dtype, const void* d_prev, void* d_fut, int64_t ny, int64_t nx, int64_t nbatch,
                       int64_t batch_stride, void* stream) {
    return apply_common(op, 1, 0, dtype, d_prev, d_fut, ny, nx, nbatch, batch_stride, stream);
}

sbp_status sbp_dissxi(int op, int dtype, const void* d_prev, void* d_fut, int64_t ny, int64_t nx, int64_t nbatch,
                      int64_t batch_stride, void* stream) {
    return apply_common(op, 0, 1, dtype, d_prev, d_fut, ny, nx, nbatch, batch_stride, stream);
}

sbp_status sbp_disseta(int op, int dtype, const void* d_prev, void* d_fut, int64_t ny, int64_t nx, int64_t nbatch,
                       int64_t batch_stride, void* stream) {
    return apply_common(op, 1, 1, dtype, d_prev, d_fut, ny, nx, nbatch, batch_stride, stream);
}

sbp_status sbp_metrics(int op_xi, int op_eta, const double* d_x, const double* d_y, int64_t ny, int64_t nx,
                       double* d_metrics, void* stream) {
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
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t n = nx * ny;
    double* tmp = nullptr;
    unsigned* status = nullptr;
    SBP_TRY_CUDA(cudaMallocAsync(&tmp, 4 * n * sizeof(double), st));
    SBP_TRY_CUDA(cudaMallocAsync(&status, sizeof(unsigned), st));
    sbp_status s = SBP_OK;
    do {
        if ((s = cuda_status(cudaMemsetAsync(status, 0, sizeof(unsigned), st), "memset")) != SBP_OK) break;
        if ((s = cuda_status(op_apply(op_xi, 0, 0, 0, d_x, tmp, ny, nx, 1, n, st), "diffxi x")) != SBP_OK) break;
        if ((s = cuda_status(op_apply(op_eta, 1, 0, 0, d_x, tmp + n, ny, nx, 1, n, st), "diffeta x")) != SBP_OK) break;
        if ((s = cuda_status(op_apply(op_xi, 0, 0, 0, d_y, tmp + 2 * n, ny, nx, 1, n, st), "diffxi y")) != SBP_OK) break;
        if ((s = cuda_status(op_apply(op_eta, 1, 0, 0, d_y, tmp + 3 * n, ny, nx, 1, n, st), "diffeta y")) != SBP_OK)
            break;
        if ((s = cuda_status(metrics_combine(tmp, tmp + n, tmp + 2 * n, tmp + 3 * n, n, d_metrics, n, status, st),
                             "metrics")) != SBP_OK)
            break;
        unsigned hs = 0;
        if ((s = cuda_status(cudaMemcpyAsync(&hs, status, sizeof hs, cudaMemcpyDeviceToHost, st), "status")) != SBP_OK)
            break;
        if ((s = cuda_status(cudaStreamSynchronize(st), "sync")) != SBP_OK) break;
        if (hs) {
            set_error("non-positive Jacobian determinant");
            s = SBP_ERR_NONPHYSICAL;
        }
    } while (0);
    cudaFreeAsync(tmp, st);
    cudaFreeAsync(status, st);
    return s;
}

}  // extern "C"
