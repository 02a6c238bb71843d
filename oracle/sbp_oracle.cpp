/*
 * CPU oracle for the SBP-SAT Euler hot path -- TEST INFRASTRUCTURE ONLY.
 * See sbp_oracle.h for scope and parity status ("parity unpinned" against the
 * reference binary; pinned against the reference's known-answer tests).
 *
 * Must be compiled with -ffp-contract=off and without -ffast-math: every
 * product and sum below is rounded separately, as the reference's default
 * x86-64 build does, except where the reference explicitly fuses (std::fma).
 */
#include "sbp_oracle.h"
#include "oracle_coefficients.h"
#include "oracle_interp_coefficients.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <type_traits>
#include <vector>

namespace {

/* ------------------------------------------------------------------------- */
/* Operator tables                                                           */
/* ------------------------------------------------------------------------- */

#define DECL_TABLES(TAG, LIT, SUF, TY)                                        \
    static const TY TAG##_H_##SUF[] = {ORC_##TAG##_H(LIT)};                   \
    static const TY TAG##_DIFF_START_##SUF[] = {ORC_##TAG##_DIFF_START(LIT)}; \
    static const TY TAG##_DIFF_DIAG_##SUF[] = {ORC_##TAG##_DIFF_DIAG(LIT)};
#define DECL_DISS(TAG, LIT, SUF, TY)                                          \
    static const TY TAG##_DISS_START_##SUF[] = {ORC_##TAG##_DISS_START(LIT)}; \
    static const TY TAG##_DISS_DIAG_##SUF[] = {ORC_##TAG##_DISS_DIAG(LIT)};

DECL_TABLES(UPWIND4, ORC_LIT_F64, D, double)
DECL_TABLES(UPWIND4H2, ORC_LIT_F64, D, double)
DECL_TABLES(UPWIND9, ORC_LIT_F64, D, double)
DECL_TABLES(UPWIND9H2, ORC_LIT_F64, D, double)
DECL_TABLES(SBP4, ORC_LIT_F64, D, double)
DECL_TABLES(SBP8, ORC_LIT_F64, D, double)
DECL_DISS(UPWIND4, ORC_LIT_F64, D, double)
DECL_DISS(UPWIND4H2, ORC_LIT_F64, D, double)
DECL_DISS(UPWIND9, ORC_LIT_F64, D, double)
DECL_DISS(UPWIND9H2, ORC_LIT_F64, D, double)
DECL_TABLES(UPWIND4, ORC_LIT_F32, F, float)
DECL_TABLES(UPWIND4H2, ORC_LIT_F32, F, float)
DECL_TABLES(UPWIND9, ORC_LIT_F32, F, float)
DECL_TABLES(UPWIND9H2, ORC_LIT_F32, F, float)
DECL_TABLES(SBP4, ORC_LIT_F32, F, float)
DECL_TABLES(SBP8, ORC_LIT_F32, F, float)
DECL_DISS(UPWIND4, ORC_LIT_F32, F, float)
DECL_DISS(UPWIND4H2, ORC_LIT_F32, F, float)
DECL_DISS(UPWIND9, ORC_LIT_F32, F, float)
DECL_DISS(UPWIND9H2, ORC_LIT_F32, F, float)

/* A BlockMatrix (sbp/src/operators/algos.rs:31-41) plus the H boundary weights. */
template <class T>
struct BlockOp {
    int M = 0, N = 0, D = 0;
    bool h2 = false, upwind = false, valid = false;
    T start[8 * 13] = {};
    T diag[11] = {};
    T end[8 * 13] = {};
    T h[8] = {};
};

template <class T>
struct Raw {
    const T *h, *dstart, *ddiag, *sstart, *sdiag;
};

template <class T>
static bool raw_tables(int op, Raw<T>& r, int& M, int& N, int& D, bool& h2, bool& upw);

#define RAW_CASE(ENUM, TAG, SUF, H2, UPW)                                         \
    case ENUM:                                                                    \
        r.h = TAG##_H_##SUF;                                                      \
        r.dstart = TAG##_DIFF_START_##SUF;                                        \
        r.ddiag = TAG##_DIFF_DIAG_##SUF;                                          \
        M = ORC_##TAG##_M;                                                        \
        N = ORC_##TAG##_N;                                                        \
        D = ORC_##TAG##_D;                                                        \
        h2 = H2;                                                                  \
        upw = UPW;                                                                \
        break;

template <>
bool raw_tables<double>(int op, Raw<double>& r, int& M, int& N, int& D, bool& h2, bool& upw) {
    r = Raw<double>{};
    switch (op) {
        RAW_CASE(ORC_UPWIND4, UPWIND4, D, false, true)
        RAW_CASE(ORC_UPWIND4H2, UPWIND4H2, D, true, true)
        RAW_CASE(ORC_UPWIND9, UPWIND9, D, false, true)
        RAW_CASE(ORC_UPWIND9H2, UPWIND9H2, D, true, true)
        RAW_CASE(ORC_SBP4, SBP4, D, false, false)
        RAW_CASE(ORC_SBP8, SBP8, D, false, false)
        default: return false;
    }
    switch (op) {
        case ORC_UPWIND4: r.sstart = UPWIND4_DISS_START_D; r.sdiag = UPWIND4_DISS_DIAG_D; break;
        case ORC_UPWIND4H2: r.sstart = UPWIND4H2_DISS_START_D; r.sdiag = UPWIND4H2_DISS_DIAG_D; break;
        case ORC_UPWIND9: r.sstart = UPWIND9_DISS_START_D; r.sdiag = UPWIND9_DISS_DIAG_D; break;
        case ORC_UPWIND9H2: r.sstart = UPWIND9H2_DISS_START_D; r.sdiag = UPWIND9H2_DISS_DIAG_D; break;
        default: break;
    }
    return true;
}

template <>
bool raw_tables<float>(int op, Raw<float>& r, int& M, int& N, int& D, bool& h2, bool& upw) {
    r = Raw<float>{};
    switch (op) {
        RAW_CASE(ORC_UPWIND4, UPWIND4, F, false, true)
        RAW_CASE(ORC_UPWIND4H2, UPWIND4H2, F, true, true)
        RAW_CASE(ORC_UPWIND9, UPWIND9, F, false, true)
        RAW_CASE(ORC_UPWIND9H2, UPWIND9H2, F, true, true)
        RAW_CASE(ORC_SBP4, SBP4, F, false, false)
        RAW_CASE(ORC_SBP8, SBP8, F, false, false)
        default: return false;
    }
    switch (op) {
        case ORC_UPWIND4: r.sstart = UPWIND4_DISS_START_F; r.sdiag = UPWIND4_DISS_DIAG_F; break;
        case ORC_UPWIND4H2: r.sstart = UPWIND4H2_DISS_START_F; r.sdiag = UPWIND4H2_DISS_DIAG_F; break;
        case ORC_UPWIND9: r.sstart = UPWIND9_DISS_START_F; r.sdiag = UPWIND9_DISS_DIAG_F; break;
        case ORC_UPWIND9H2: r.sstart = UPWIND9H2_DISS_START_F; r.sdiag = UPWIND9H2_DISS_DIAG_F; break;
        default: break;
    }
    return true;
}

/* End block = flip_lr . flip_ud of the start block, sign-flipped for the first
 * derivative (upwind4.rs:29,46; upwind9.rs:31-35,53-57; constmatrix lib.rs:302-345). */
template <class T>
static BlockOp<T> make_op(int op, int kind) {
    BlockOp<T> b;
    Raw<T> r;
    int M, N, D;
    bool h2, upw;
    if (!raw_tables<T>(op, r, M, N, D, h2, upw)) return b;
    if (kind == ORC_DISS && !upw) return b;
    const T* st = kind == ORC_DIFF ? r.dstart : r.sstart;
    const T* dg = kind == ORC_DIFF ? r.ddiag : r.sdiag;
    b.M = M;
    b.N = N;
    b.D = D;
    b.h2 = h2;
    b.upwind = upw;
    for (int i = 0; i < M * N; ++i) b.start[i] = st[i];
    for (int i = 0; i < D; ++i) b.diag[i] = dg[i];
    for (int i = 0; i < M; ++i)
        for (int j = 0; j < N; ++j) {
            T v = st[(M - 1 - i) * N + (N - 1 - j)];
            b.end[i * N + j] = kind == ORC_DIFF ? -v : v;
        }
    for (int i = 0; i < M; ++i) b.h[i] = r.h[i];
    b.valid = true;
    return b;
}

template <class T>
struct OpCache {
    BlockOp<T> ops[6][2];
    OpCache() {
        for (int o = 0; o < 6; ++o)
            for (int k = 0; k < 2; ++k) ops[o][k] = make_op<T>(o, k);
    }
};

template <class T>
static const BlockOp<T>& get_op(int op, int kind) {
    static const OpCache<T> cache; /* thread-safe one-time initialisation */
    static const BlockOp<T> invalid;
    if (op < 0 || op > 5 || kind < 0 || kind > 1) return invalid;
    return cache.ops[op][kind];
}

/* ------------------------------------------------------------------------- */
/* Stencil application                                                       */
/* ------------------------------------------------------------------------- */

/* idx = 1 / (1 / (n-1)), or 1/(n-2) spacing for h2 operators (algos.rs:125-130). */
template <class T>
static T inv_spacing(const BlockOp<T>& b, int64_t n) {
    T dx = b.h2 ? T(1) / T(n - 2) : T(1) / T(n - 1);
    return T(1) / dx;
}

/* diff_op_1d_slice (algos.rs:101-187).  Every sum is matmul_float_into without
 * fma (utils/constmatrix/src/lib.rs:120-146): t = a0*p0; t = t + ak*pk; then
 * scaled by idx (`*fut *= idx`). */
template <class T>
static void apply_row(const BlockOp<T>& b, const T* p, T* f, int64_t n) {
    const T idx = inv_spacing(b, n);
    const int M = b.M, N = b.N, D = b.D;
    for (int i = 0; i < M; ++i) {
        T t = b.start[i * N] * p[0];
        for (int k = 1; k < N; ++k) t = t + b.start[i * N + k] * p[k];
        f[i] = t * idx;
    }
    const int64_t skip = M - (D - 1) / 2;
    for (int64_t i = 0; i < n - 2 * M; ++i) {
        const T* w = p + skip + i;
        T t = b.diag[0] * w[0];
        for (int d = 1; d < D; ++d) t = t + b.diag[d] * w[d];
        f[M + i] = t * idx;
    }
    const T* pe = p + (n - N);
    for (int i = 0; i < M; ++i) {
        T t = b.end[i * N] * pe[0];
        for (int k = 1; k < N; ++k) t = t + b.end[i * N + k] * pe[k];
        f[n - M + i] = t * idx;
    }
}

/* diffeta/disseta: the operator applied on the transposed view, which the
 * reference dispatches to diff_op_2d_sliceable_y_simd (algos.rs:371-519,
 * 539-555).  Columns j < LANES*floor(nx/LANES) (LANES = 8 for f64x8, 16 for
 * f32x16) accumulate with fused multiply-add from zero, in coefficient order,
 * then multiply by idx (algos.rs:442-447, 492-499); the remaining columns add
 * unfused products to 0.0 (algos.rs:449-455, 501-510). */
template <class T>
static void apply_eta(const BlockOp<T>& b, const T* p, T* f, int64_t ny, int64_t nx) {
    const T idx = inv_spacing(b, ny);
    const int64_t lanes = sizeof(T) == 8 ? 8 : 16;
    const int64_t simd = lanes * (nx / lanes);
    const int M = b.M, N = b.N, D = b.D, half = (D - 1) / 2;
    for (int64_t i = 0; i < ny; ++i) {
        const T* coef;
        int64_t row0;
        int nc;
        bool diag_row = false;
        if (i < M) {
            coef = b.start + i * N;
            row0 = 0;
            nc = N;
        } else if (i >= ny - M) {
            coef = b.end + (i - (ny - M)) * N;
            row0 = ny - N;
            nc = N;
        } else {
            coef = b.diag;
            row0 = i - half;
            nc = D;
            diag_row = true;
        }
        T* out = f + i * nx;
        for (int64_t j = 0; j < simd; ++j) {
            T acc = T(0);
            for (int k = 0; k < nc; ++k) acc = std::fma(p[(row0 + k) * nx + j], coef[k], acc);
            out[j] = acc * idx;
        }
        for (int64_t j = simd; j < nx; ++j) {
            T acc = T(0);
            for (int k = 0; k < nc; ++k) acc += coef[k] * p[(row0 + k) * nx + j];
            out[j] = diag_row ? idx * acc : acc * idx;
        }
    }
}

template <class T>
static int op_apply_t(int op, int dir, int kind, const T* in, T* out, int64_t ny, int64_t nx) {
    const BlockOp<T>& b = get_op<T>(op, kind);
    if (!b.valid) return -1;
    if (dir == ORC_XI) {
        if (nx < 2 * b.M || nx < b.N) return -3;
        for (int64_t r = 0; r < ny; ++r) apply_row(b, in + r * nx, out + r * nx, nx);
    } else {
        if (ny < 2 * b.M || ny < b.N) return -3;
        apply_eta(b, in, out, ny, nx);
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Euler                                                                     */
/* ------------------------------------------------------------------------- */

/* pressure (euler/src/lib.rs:478-480) */
static inline double pressure(double g, double rho, double rhou, double rhov, double e) {
    return (g - 1.0) * (e - (rhou * rhou + rhov * rhov) / (2.0 * rho));
}

struct Metrics {
    std::vector<double> detj, jxx, jxy, jyx, jyy;
};

/* Metrics::new (sbp/src/grid.rs:95-140). */
static int build_metrics(int opx, int ope, const double* x, const double* y, int64_t ny, int64_t nx,
                         Metrics& m) {
    const int64_t n = ny * nx;
    std::vector<double> dx_dxi(n), dx_deta(n), dy_dxi(n), dy_deta(n);
    int rc = 0;
    rc |= op_apply_t<double>(opx, ORC_XI, ORC_DIFF, x, dx_dxi.data(), ny, nx);
    rc |= op_apply_t<double>(ope, ORC_ETA, ORC_DIFF, x, dx_deta.data(), ny, nx);
    rc |= op_apply_t<double>(opx, ORC_XI, ORC_DIFF, y, dy_dxi.data(), ny, nx);
    rc |= op_apply_t<double>(ope, ORC_ETA, ORC_DIFF, y, dy_deta.data(), ny, nx);
    if (rc) return -1;
    m.detj.resize(n);
    m.jxx.resize(n);
    m.jxy.resize(n);
    m.jyx.resize(n);
    m.jyy.resize(n);
    for (int64_t i = 0; i < n; ++i) {
        double d = dx_dxi[i] * dy_deta[i] - dx_deta[i] * dy_dxi[i];
        if (!(d > 0.0)) return -2;
        m.detj[i] = d;
        m.jxx[i] = dy_deta[i];
        m.jxy[i] = -dx_deta[i];
        m.jyx[i] = -dy_dxi[i];
        m.jyy[i] = dx_dxi[i];
    }
    return 0;
}

/* VortexParameters::evaluate (euler/src/vortex.rs:26-113).  With no vortices
 * the reference writes rhou twice and leaves rhov untouched (vortex.rs:56-61);
 * the oracle writes the evident intent, rhou = rho_inf*u_inf and
 * rhov = rho_inf*v_inf, as the library does. */
static void vortex_point(const orc_vortex_params& vp, double gamma, double t, double x, double y, double& rho,
                         double& rhou, double& rhov, double& e) {
    const double PI = 3.14159265358979323846;
    const double m = vp.mach;
    const double p_inf = 1.0 / (gamma * m * m);
    const double rho_inf = 1.0, u_inf = 1.0, v_inf = 0.0;
    const double e_inf = p_inf / (gamma - 1.0) + rho_inf * (u_inf * u_inf + v_inf * v_inf) / 2.0;
    if (vp.nvortices <= 0) {
        rho = rho_inf;
        rhou = rho_inf * u_inf;
        rhov = rho_inf * v_inf;
        e = e_inf;
        return;
    }
    for (int iv = 0; iv < vp.nvortices; ++iv) {
        const double rstar = vp.rstar[iv], eps = vp.eps[iv];
        const double dx = (x - vp.x0[iv]) - t;
        const double dy = y - vp.y0[iv];
        const double f = (1.0 - (dx * dx + dy * dy)) / (rstar * rstar);
        const double r = std::pow(
            1.0 - eps * eps * (gamma - 1.0) * m * m / (8.0 * PI * PI * p_inf * rstar * rstar) * std::exp(f),
            1.0 / (gamma - 1.0));
        const double p = std::pow(r, gamma) * p_inf;
        const double u = 1.0 - eps * dy / (2.0 * PI * std::sqrt(p_inf) * rstar * rstar) * std::exp(f / 2.0);
        const double v = eps * dx / (2.0 * PI * std::sqrt(p_inf) * rstar * rstar) * std::exp(f / 2.0);
        if (iv == 0) {
            rho = r;
            rhou = r * u;
            rhov = r * v;
            e = p / (gamma - 1.0) + r * (u * u + v * v) / 2.0;
        } else {
            rho += r - rho_inf;
            rhou += r * u - rho_inf * u_inf;
            rhov += r * v - rho_inf * v_inf;
            e += (p / (gamma - 1.0) + r * (u * u + v * v) / 2.0) - e_inf;
        }
    }
}

/* SAT_characteristic (euler/src/lib.rs:1150-1252) for one edge point.
 * y = own state at the point, z = boundary data; returns k += hi*tau*T*(...). */
static void sat_point(double gamma, const double y[4], const double z[4], double hi, double sign, double tau,
                      double detj, double detj_d_dx, double detj_d_dy, double k[4]) {
    const double rho = y[0], rhou = y[1], rhov = y[2], e = y[3];
    const double kx_ = detj_d_dx / detj;
    const double ky_ = detj_d_dy / detj;
    const double r = std::hypot(kx_, ky_);
    const double kx = kx_ / r, ky = ky_ / r;
    const double u = rhou / rho, v = rhov / rho;
    const double theta = kx * u + ky * v;
    const double p = pressure(gamma, rho, rhou, rhov, e);
    const double c = std::sqrt(gamma * p / rho);
    const double phi2 = (gamma - 1.0) * (u * u + v * v) / 2.0;
    const double SQRT_2 = 1.41421356237309504880;
    const double alpha = rho / (SQRT_2 * c);
    const double phi2_c2 = (phi2 + c * c) / (gamma - 1.0);
    const double T[4][4] = {
        {1.0, 0.0, alpha, alpha},
        {u, ky, alpha * (u + kx * c), alpha * (u - kx * c)},
        {v, -kx, alpha * (v + ky * c), alpha * (v - ky * c)},
        {phi2 / (gamma - 1.0), rho * (ky * u - kx * v), alpha * (phi2_c2 + c * theta), alpha * (phi2_c2 - c * theta)},
    };
    const double U = kx_ * u + ky_ * v;
    const double L[4] = {U, U, U + c * std::hypot(kx_, ky_), U - c * std::hypot(kx_, ky_)};
    const double beta = 1.0 / (2.0 * c * c);
    const double TI[4][4] = {
        {1.0 - phi2 / (c * c), (gamma - 1.0) * u / (c * c), (gamma - 1.0) * v / (c * c), -(gamma - 1.0) / (c * c)},
        {-(ky * u - kx * v) / rho, ky / rho, -kx / rho, 0.0},
        {beta * (phi2 - c * theta), beta * (kx * c - (gamma - 1.0) * u), beta * (ky * c - (gamma - 1.0) * v),
         beta * (gamma - 1.0)},
        {beta * (phi2 + c * theta), -beta * (kx * c + (gamma - 1.0) * u), -beta * (ky * c + (gamma - 1.0) * v),
         beta * (gamma - 1.0)},
    };
    const double res[4] = {rho - z[0], rhou - z[1], rhov - z[2], e - z[3]};
    double TIres[4] = {0.0, 0.0, 0.0, 0.0};
    for (int row = 0; row < 4; ++row)
        for (int col = 0; col < 4; ++col) TIres[row] += TI[row][col] * res[col];
    double LTIres[4];
    for (int row = 0; row < 4; ++row) LTIres[row] = (L[row] + sign * std::fabs(L[row])) * TIres[row];
    double TLTIres[4] = {0.0, 0.0, 0.0, 0.0};
    for (int row = 0; row < 4; ++row)
        for (int col = 0; col < 4; ++col) TLTIres[row] += T[row][col] * LTIres[col];
    for (int comp = 0; comp < 4; ++comp) k[comp] += hi * tau * TLTIres[comp];
}

struct BlockCtx {
    int64_t nx, ny;
    int opx, ope;
    bool upwind;
    const Metrics* m;
};

/* Work arrays (the reference's WorkBuffers, euler/src/lib.rs:1255-1269). */
struct Work {
    std::vector<double> ehat, fhat, de, df, adxi, adeta, p;
    void ensure(int64_t n) {
        if ((int64_t)p.size() == n) return;
        ehat.assign(4 * n, 0.0);
        fhat.assign(4 * n, 0.0);
        de.assign(4 * n, 0.0);
        df.assign(4 * n, 0.0);
        adxi.assign(4 * n, 0.0);
        adeta.assign(4 * n, 0.0);
        p.assign(n, 0.0);
    }
};

/* fluxes (euler/src/lib.rs:680-735) */
static void fluxes(const BlockCtx& B, double gamma, const double* q, Work& w) {
    const int64_t n = B.nx * B.ny;
    const double *rho = q, *rhou = q + n, *rhov = q + 2 * n, *e = q + 3 * n;
    for (int64_t i = 0; i < n; ++i) w.p[i] = pressure(gamma, rho[i], rhou[i], rhov[i], e[i]);
    double* E = w.ehat.data();
    double* F = w.fhat.data();
    for (int64_t i = 0; i < n; ++i) {
        const double p = w.p[i];
        E[i] = rhou[i];
        E[n + i] = rhou[i] * rhou[i] / rho[i] + p;
        E[2 * n + i] = rhou[i] * rhov[i] / rho[i];
        E[3 * n + i] = rhou[i] * (e[i] + p) / rho[i];
        F[i] = rhov[i];
        F[n + i] = E[2 * n + i];
        F[2 * n + i] = rhov[i] * rhov[i] / rho[i] + p;
        F[3 * n + i] = rhov[i] * (e[i] + p) / rho[i];
    }
    const Metrics& m = *B.m;
    for (int c = 0; c < 4; ++c)
        for (int64_t i = 0; i < n; ++i) {
            const double ef = E[c * n + i], ff = F[c * n + i];
            E[c * n + i] = m.jxx[i] * ef + m.jxy[i] * ff;
            F[c * n + i] = m.jyx[i] * ef + m.jyy[i] * ff;
        }
}

/* upwind_dissipation (euler/src/lib.rs:619-674); writes ad_xi, ad_eta.
 * Uses ehat/fhat as the alpha*q temporaries, as the reference does. */
static int upwind_dissipation(const BlockCtx& B, double gamma, const double* q, Work& w) {
    const int64_t n = B.nx * B.ny;
    const double *rho = q, *rhou = q + n, *rhov = q + 2 * n, *e = q + 3 * n;
    const Metrics& m = *B.m;
    double* t0 = w.ehat.data();
    double* t1 = w.fhat.data();
    int bad = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (!(rho[i] > 0.0)) bad = 1;
        const double u = rhou[i] / rho[i];
        const double v = rhov[i] / rho[i];
        const double uhat = m.jxx[i] * u + m.jxy[i] * v;
        const double vhat = m.jyx[i] * u + m.jyy[i] * v;
        const double p = pressure(gamma, rho[i], rhou[i], rhov[i], e[i]);
        if (!(p > 0.0)) bad = 1;
        const double c = std::sqrt(gamma * p / rho[i]);
        const double au = std::fabs(uhat) + c * std::sqrt(m.jxx[i] * m.jxx[i] + m.jxy[i] * m.jxy[i]);
        const double av = std::fabs(vhat) + c * std::sqrt(m.jyx[i] * m.jyx[i] + m.jyy[i] * m.jyy[i]);
        t0[i] = au * rho[i];
        t1[i] = av * rho[i];
        t0[n + i] = au * rhou[i];
        t1[n + i] = av * rhou[i];
        t0[2 * n + i] = au * rhov[i];
        t1[2 * n + i] = av * rhov[i];
        t0[3 * n + i] = au * e[i];
        t1[3 * n + i] = av * e[i];
    }
    for (int c = 0; c < 4; ++c) {
        op_apply_t<double>(B.opx, ORC_XI, ORC_DISS, t0 + c * n, w.adxi.data() + c * n, B.ny, B.nx);
        op_apply_t<double>(B.ope, ORC_ETA, ORC_DISS, t1 + c * n, w.adeta.data() + c * n, B.ny, B.nx);
    }
    return bad;
}

/* SAT_north/south/east/west (euler/src/lib.rs:1025-1144) applied in the order of
 * SAT_characteristics (euler/src/lib.rs:1002-1013). z[d] holds 4 x edge-length values. */
static void sat_all(const BlockCtx& B, double gamma, const double* q, const double* const z[4], double* k) {
    const int64_t nx = B.nx, ny = B.ny, n = nx * ny;
    const Metrics& m = *B.m;
    const BlockOp<double>& ox = get_op<double>(B.opx, ORC_DIFF);
    const BlockOp<double>& oe = get_op<double>(B.ope, ORC_DIFF);
    const double hi_eta = (oe.h2 ? double(ny - 2) : double(ny - 1)) / oe.h[0];
    const double hi_xi = (ox.h2 ? double(nx - 2) : double(nx - 1)) / ox.h[0];
    for (int d = 0; d < 4; ++d) {
        if (!z[d]) continue;
        const bool ns = d == ORC_NORTH || d == ORC_SOUTH;
        const int64_t len = ns ? nx : ny;
        const double sign = (d == ORC_NORTH || d == ORC_EAST) ? -1.0 : 1.0;
        const double tau = (d == ORC_NORTH || d == ORC_EAST) ? 1.0 : -1.0;
        const double hi = ns ? hi_eta : hi_xi;
        for (int64_t i = 0; i < len; ++i) {
            int64_t pt;
            if (d == ORC_NORTH) pt = (ny - 1) * nx + i;
            else if (d == ORC_SOUTH) pt = i;
            else if (d == ORC_EAST) pt = i * nx + (nx - 1);
            else pt = i * nx;
            double yv[4], zv[4], kv[4];
            for (int c = 0; c < 4; ++c) {
                yv[c] = q[c * n + pt];
                zv[c] = z[d][c * len + i];
                kv[c] = k[c * n + pt];
            }
            const double ddx = ns ? m.jyx[pt] : m.jxx[pt];
            const double ddy = ns ? m.jyy[pt] : m.jxy[pt];
            sat_point(gamma, yv, zv, hi, sign, tau, m.detj[pt], ddx, ddy, kv);
            for (int c = 0; c < 4; ++c) k[c * n + pt] = kv[c];
        }
    }
}

/* RHS_upwind (euler/src/lib.rs:571-616) or RHS_trad (483-515). */
static int rhs(const BlockCtx& B, double gamma, const double* q, const double* const z[4], bool force_trad,
               double* k, Work& w) {
    const int64_t n = B.nx * B.ny;
    w.ensure(n);
    fluxes(B, gamma, q, w);
    for (int c = 0; c < 4; ++c) {
        op_apply_t<double>(B.opx, ORC_XI, ORC_DIFF, w.ehat.data() + c * n, w.de.data() + c * n, B.ny, B.nx);
        op_apply_t<double>(B.ope, ORC_ETA, ORC_DIFF, w.fhat.data() + c * n, w.df.data() + c * n, B.ny, B.nx);
    }
    const Metrics& m = *B.m;
    int bad = 0;
    if (B.upwind && !force_trad) {
        bad = upwind_dissipation(B, gamma, q, w);
        for (int c = 0; c < 4; ++c)
            for (int64_t i = 0; i < n; ++i) {
                const int64_t j = c * n + i;
                k[j] = (-w.de[j] - w.df[j] + w.adxi[j] + w.adeta[j]) / m.detj[i];
            }
    } else {
        for (int c = 0; c < 4; ++c)
            for (int64_t i = 0; i < n; ++i) {
                const int64_t j = c * n + i;
                k[j] = (-w.de[j] - w.df[j]) / m.detj[i];
            }
    }
    sat_all(B, gamma, q, z, k);
    return bad;
}

/* h2_err (euler/src/lib.rs:377-431) */
static double h2_err(int opx, int ope, const double* a, const double* b, int64_t ny, int64_t nx) {
    const BlockOp<double>& ox = get_op<double>(opx, ORC_DIFF);
    const BlockOp<double>& oe = get_op<double>(ope, ORC_DIFF);
    auto weights = [](const BlockOp<double>& o, int64_t n) {
        std::vector<double> h(n, 1.0);
        for (int i = 0; i < o.M; ++i) {
            h[i] = o.h[i];
            h[n - 1 - i] = o.h[i];
        }
        const double factor = o.h2 ? 1.0 / double(n - 2) : 1.0 / double(n - 1);
        for (auto& v : h) v = v * factor;
        return h;
    };
    std::vector<double> hx = weights(ox, nx), hy = weights(oe, ny);
    double s = 0.0;
    const int64_t n = nx * ny;
    for (int c = 0; c < 4; ++c)
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 0; i < nx; ++i) {
                const double d = a[c * n + j * nx + i] - b[c * n + j * nx + i];
                s += d * d * hx[i] * hy[j];
            }
    return std::sqrt(s);
}

}  // namespace

/* ------------------------------------------------------------------------- */
/* Multi-block system (multigrid/src/system.rs:456-636)                      */
/* ------------------------------------------------------------------------- */

struct orc_system {
    std::vector<std::vector<int>> mg[4];  // copies of the MultiGrid triples per block and side
    double gamma = 1.4;
    double time = 0.0;
    std::vector<orc_block_desc> desc;
    std::vector<std::vector<double>> x, y;
    std::vector<Metrics> metrics;
    std::vector<BlockCtx> ctx;
    std::vector<std::vector<double>> now, fut;
    std::vector<std::vector<double>> k[8];
    std::vector<Work> work;
    std::vector<std::vector<double>> ebuf[4];
    orc_vortex_params vp{};
};

namespace {

/* Interpolation operator tables (oracle_interp_coefficients.h, transcribed from the reference:
 * f64 values and the reference's f32-build values). */
template <class T>
struct InterpTable {
    int brows, bcols, drows, dcols, jump0, jump1;
    const T* block;
    const T* diag;
};
#define ORC_INTERP_TABLES(P)                                                                                   \
    static const double kI##P##_F2C_B[] = {ORCI_##P##_F2C_BLOCK}, kI##P##_F2C_D[] = {ORCI_##P##_F2C_DIAG};     \
    static const double kI##P##_C2F_B[] = {ORCI_##P##_C2F_BLOCK}, kI##P##_C2F_D[] = {ORCI_##P##_C2F_DIAG};     \
    static const float kJ##P##_F2C_B[] = {ORCI_##P##_F2C_BLOCK_F32}, kJ##P##_F2C_D[] = {ORCI_##P##_F2C_DIAG_F32}; \
    static const float kJ##P##_C2F_B[] = {ORCI_##P##_C2F_BLOCK_F32}, kJ##P##_C2F_D[] = {ORCI_##P##_C2F_DIAG_F32};
ORC_INTERP_TABLES(4)
ORC_INTERP_TABLES(8)
ORC_INTERP_TABLES(9)
ORC_INTERP_TABLES(9H2)
#undef ORC_INTERP_TABLES
#define ORC_INTERP_ENTRY(T, K, P, D)                                                                           \
    InterpTable<T> {                                                                                           \
        ORCI_##P##_##D##_BROWS, ORCI_##P##_##D##_BCOLS, ORCI_##P##_##D##_DROWS, ORCI_##P##_##D##_DCOLS,       \
            ORCI_##P##_##D##_JUMP0, ORCI_##P##_##D##_JUMP1, K##P##_##D##_B, K##P##_##D##_D                    \
    }
#define ORC_INTERP_ROWS(T, K)                                                                                  \
    {{ORC_INTERP_ENTRY(T, K, 4, C2F), ORC_INTERP_ENTRY(T, K, 4, F2C)},                                         \
     {ORC_INTERP_ENTRY(T, K, 8, C2F), ORC_INTERP_ENTRY(T, K, 8, F2C)},                                         \
     {ORC_INTERP_ENTRY(T, K, 9, C2F), ORC_INTERP_ENTRY(T, K, 9, F2C)},                                         \
     {ORC_INTERP_ENTRY(T, K, 9H2, C2F), ORC_INTERP_ENTRY(T, K, 9H2, F2C)}}
static const InterpTable<double> kInterp[4][2] = ORC_INTERP_ROWS(double, kI);
static const InterpTable<float> kInterp32[4][2] = ORC_INTERP_ROWS(float, kJ);
#undef ORC_INTERP_ROWS
#undef ORC_INTERP_ENTRY
static const bool kInterpFineOdd[4] = {ORCI_4_FINE_ODD != 0, ORCI_8_FINE_ODD != 0, ORCI_9_FINE_ODD != 0,
                                       ORCI_9H2_FINE_ODD != 0};

/* interpolate (sbp/src/operators/interpolation.rs:15-50): every output starts at 0 and
 * accumulates out += in * c over all columns of its row (zeros included), unfused, in T. */
template <class T>
static void interpolate(const T* in, int64_t nin, T* out, int64_t nout, const InterpTable<T>& I) {
    for (int64_t i = 0; i < nout; ++i) {
        T t = T(0);
        if (i < I.brows) {
            for (int k = 0; k < I.bcols; ++k) t = t + in[k] * I.block[i * I.bcols + k];
        } else if (nout - i <= I.brows) {
            const int64_t row = nout - i - 1;
            const int64_t index = nin - I.bcols;
            for (int k = 0; k < I.bcols; ++k) {
                const int col = I.bcols - k - 1;
                t = t + in[index + k] * I.block[row * I.bcols + col];
            }
        } else {
            const int64_t n = i - I.brows;
            const int64_t index = I.jump0 + I.jump1 * (n / I.drows);
            const int64_t row = n % I.drows;
            for (int k = 0; k < I.dcols; ++k) t = t + in[index + k] * I.diag[row * I.dcols + k];
        }
        out[i] = t;
    }
}

/* the size relation the operator asserts (fine = 2 coarse - 1, or 2 (coarse - 1) for 9h2) */
static bool interp_sizes_ok(int op, int64_t fine, int64_t coarse) {
    return kInterpFineOdd[op] ? fine == 2 * coarse - 1 : fine == 2 * (coarse - 1);
}

/* Edge extraction of a field: north = last row, south = row 0, east = last column, west = column 0. */
static void edge_of(const std::vector<double>& q, int64_t ny, int64_t nx, int d, std::vector<double>& out) {
    const int64_t n = nx * ny;
    const bool ns = d == ORC_NORTH || d == ORC_SOUTH;
    const int64_t len = ns ? nx : ny;
    out.resize(4 * len);
    for (int c = 0; c < 4; ++c)
        for (int64_t i = 0; i < len; ++i) {
            int64_t pt;
            if (d == ORC_NORTH) pt = (ny - 1) * nx + i;
            else if (d == ORC_SOUTH) pt = i;
            else if (d == ORC_EAST) pt = i * nx + (nx - 1);
            else pt = i * nx;
            out[c * len + i] = q[c * n + pt];
        }
}

static int opposite(int d) {
    return d == ORC_NORTH ? ORC_SOUTH : d == ORC_SOUTH ? ORC_NORTH : d == ORC_EAST ? ORC_WEST : ORC_EAST;
}

/* boundary_extracts (euler/src/lib.rs:869-930): This -> own opposite edge, Grid(g) -> block g's
 * opposite edge, Vortex -> the vortex at the edge coordinates at `time`. */
static int extract(orc_system* s, const std::vector<std::vector<double>>& fields, int b, double time,
                   const double* z[4]) {
    const orc_block_desc& D = s->desc[b];
    for (int d = 0; d < 4; ++d) {
        std::vector<double>& buf = s->ebuf[d][b];
        const int kind = D.bc_kind[d];
        if (kind == ORC_BC_THIS) {
            edge_of(fields[b], D.ny, D.nx, opposite(d), buf);
        } else if (kind == ORC_BC_GRID) {
            const int g = D.bc_neighbour[d];
            const orc_block_desc& G = s->desc[g];
            edge_of(fields[g], G.ny, G.nx, opposite(d), buf);
            const int64_t len = (d == ORC_NORTH || d == ORC_SOUTH) ? D.nx : D.ny;
            if ((int64_t)buf.size() != 4 * len) return -3;
        } else if (kind == ORC_BC_INTERPOLATE) {
            // euler/src/lib.rs:816-827: fine2coarse when this block's nx is the smaller one
            const int g = D.bc_neighbour[d];
            const int op = D.bc_interp_op[d];
            if (op < 0 || op > 3) return -1;
            const orc_block_desc& G = s->desc[g];
            std::vector<double> from;
            edge_of(fields[g], G.ny, G.nx, opposite(d), from);
            const bool f2c = D.nx < G.nx;
            const int64_t len = (d == ORC_NORTH || d == ORC_SOUTH) ? D.nx : D.ny;
            const int64_t lg = (int64_t)from.size() / 4;
            if (f2c ? !interp_sizes_ok(op, lg, len) : !interp_sizes_ok(op, len, lg)) return -3;
            buf.assign(4 * len, 0.0);
            for (int c = 0; c < 4; ++c) interpolate(from.data() + c * lg, lg, buf.data() + c * len, len, kInterp[op][f2c]);
        } else if (kind == ORC_BC_MULTIGRID) {
            // euler/src/lib.rs:829-846, as written: each segment (g, start, end) of the
            // neighbours' opposite edges is copied in turn, the next one starting on the last
            // point of the previous; the first point of every segment but the last is halved.
            const int64_t len = (d == ORC_NORTH || d == ORC_SOUTH) ? D.nx : D.ny;
            const std::vector<int>& mg = s->mg[d][b];
            buf.assign(4 * len, 0.0);
            int64_t i = 0;
            int remaining = (int)mg.size() / 3;
            if (remaining == 0) return -3;
            for (size_t sgi = 0; sgi + 2 < mg.size(); sgi += 3) {
                const int g = mg[sgi], start = mg[sgi + 1], end = mg[sgi + 2];
                const orc_block_desc& G = s->desc[g];
                std::vector<double> from;
                edge_of(fields[g], G.ny, G.nx, opposite(d), from);
                const int64_t lg = (int64_t)from.size() / 4;
                const int64_t n = end - start;
                if (start < 0 || end > lg || n <= 0 || i + n > len) return -3;
                for (int c = 0; c < 4; ++c)
                    for (int64_t j = 0; j < n; ++j) buf[c * len + i + j] = from[c * lg + start + j];
                remaining -= 1;
                if (remaining == 0) {
                    i += n;
                    if (i != len) return -3;
                } else {
                    for (int c = 0; c < 4; ++c) buf[c * len + i] /= 2.0;
                    i += n - 1;
                }
            }
        } else if (kind == ORC_BC_VORTEX) {
            const bool ns = d == ORC_NORTH || d == ORC_SOUTH;
            const int64_t len = ns ? D.nx : D.ny;
            buf.resize(4 * len);
            for (int64_t i = 0; i < len; ++i) {
                int64_t pt;
                if (d == ORC_NORTH) pt = (D.ny - 1) * D.nx + i;
                else if (d == ORC_SOUTH) pt = i;
                else if (d == ORC_EAST) pt = i * D.nx + (D.nx - 1);
                else pt = i * D.nx;
                vortex_point(s->vp, s->gamma, time, s->x[b][pt], s->y[b][pt], buf[i], buf[len + i], buf[2 * len + i],
                             buf[3 * len + i]);
            }
        } else {
            return -1;
        }
        z[d] = buf.data();
    }
    return 0;
}

/* integrate::<Rk4> (utils/integrate/src/lib.rs:30-35,176-222) over all blocks, with the state update
 * x = x + (c*dt)*k of Field::scaled_add (euler/src/lib.rs:205-212). */
static int advance_step(orc_system* s, double dt, bool force_trad) {
    static const double A[3][3] = {{0.5, 0.0, 0.0}, {0.0, 0.5, 0.0}, {0.0, 0.0, 1.0}};
    static const double Bw[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
    static const double C[3] = {0.5, 0.5, 1.0};
    const size_t nb = s->desc.size();
    int bad = 0;
    for (int i = 0; i < 4; ++i) {
        double simtime;
        for (size_t b = 0; b < nb; ++b) {
            s->fut[b] = s->now[b];
            if (i > 0)
                for (int j = 0; j < i; ++j) {
                    const double a = A[i - 1][j];
                    if (a == 0.0) continue;
                    const double sc = a * dt;
                    std::vector<double>& f = s->fut[b];
                    const std::vector<double>& kk = s->k[j][b];
                    for (size_t q = 0; q < f.size(); ++q) f[q] = f[q] + sc * kk[q];
                }
        }
        simtime = i == 0 ? s->time : s->time + dt * C[i - 1];
        for (size_t b = 0; b < nb; ++b) {
            const double* z[4];
            int rc = extract(s, s->fut, (int)b, simtime, z);
            if (rc) return rc;
            bad |= rhs(s->ctx[b], s->gamma, s->fut[b].data(), z, force_trad, s->k[i][b].data(), s->work[b]);
        }
    }
    for (size_t b = 0; b < nb; ++b) {
        std::vector<double>& f = s->fut[b];
        f = s->now[b];
        for (int j = 0; j < 4; ++j) {
            const double sc = Bw[j] * dt;
            const std::vector<double>& kk = s->k[j][b];
            for (size_t q = 0; q < f.size(); ++q) f[q] = f[q] + sc * kk[q];
        }
    }
    s->time += dt;
    std::swap(s->now, s->fut);
    return bad ? -4 : 0;
}

/* The Butcher tableaus of utils/integrate/src/lib.rs:30-152 (A by rows of stages 2..S). */
struct OrcTableau {
    int s;
    double a[8][8];
    double b[8], c[8], bstar[8];
};
static std::vector<OrcTableau> orc_tableaus() {
    const double R5 = 2.236067977499789696409173668731276235440618359611525724270897245410520925637804899414414408378782275;
    std::vector<OrcTableau> t(7);
    for (auto& x : t) std::memset(&x, 0, sizeof x);
    // 0 Rk4
    t[0].s = 4;
    t[0].a[0][0] = 0.5;
    t[0].a[1][1] = 0.5;
    t[0].a[2][2] = 1.0;
    t[0].b[0] = 1.0 / 6.0; t[0].b[1] = 1.0 / 3.0; t[0].b[2] = 1.0 / 3.0; t[0].b[3] = 1.0 / 6.0;
    t[0].c[0] = 0.5; t[0].c[1] = 0.5; t[0].c[2] = 1.0;
    // 1 Rk4_38
    t[1].s = 4;
    t[1].a[0][0] = 1.0 / 3.0;
    t[1].a[1][0] = -1.0 / 3.0; t[1].a[1][1] = 1.0;
    t[1].a[2][0] = 1.0; t[1].a[2][1] = -1.0; t[1].a[2][2] = 1.0;
    t[1].b[0] = 1.0 / 8.0; t[1].b[1] = 3.0 / 8.0; t[1].b[2] = 3.0 / 8.0; t[1].b[3] = 1.0 / 8.0;
    t[1].c[0] = 1.0 / 3.0; t[1].c[1] = 2.0 / 3.0; t[1].c[2] = 1.0;
    // 2 EulerMethod
    t[2].s = 1;
    t[2].b[0] = 1.0;
    // 3 MidpointMethod
    t[3].s = 2;
    t[3].a[0][0] = 0.5;
    t[3].b[1] = 1.0;
    t[3].c[0] = 1.0 / 2.0;
    // 4 Rk6
    t[4].s = 7;
    t[4].a[0][0] = 4.0 / 7.0;
    t[4].a[1][0] = 115.0 / 112.0; t[4].a[1][1] = -5.0 / 16.0;
    t[4].a[2][0] = 589.0 / 630.0; t[4].a[2][1] = 5.0 / 18.0; t[4].a[2][2] = -16.0 / 45.0;
    t[4].a[3][0] = 229.0 / 1200.0 - 29.0 / 6000.0 * R5;
    t[4].a[3][1] = 119.0 / 240.0 - 187.0 / 1200.0 * R5;
    t[4].a[3][2] = -14.0 / 75.0 + 34.0 / 375.0 * R5;
    t[4].a[3][3] = -3.0 / 100.0 * R5;
    t[4].a[4][0] = 71.0 / 2400.0 - 587.0 / 12000.0 * R5;
    t[4].a[4][1] = 187.0 / 480.0 - 391.0 / 2400.0 * R5;
    t[4].a[4][2] = -38.0 / 75.0 + 26.0 / 375.0 * R5;
    t[4].a[4][3] = 27.0 / 80.0 - 3.0 / 400.0 * R5;
    t[4].a[4][4] = (1.0 + R5) / 4.0;
    t[4].a[5][0] = -49.0 / 480.0 + 43.0 / 160.0 * R5;
    t[4].a[5][1] = -425.0 / 96.0 + 51.0 / 32.0 * R5;
    t[4].a[5][2] = 52.0 / 15.0 - 4.0 / 5.0 * R5;
    t[4].a[5][3] = -27.0 / 16.0 + 3.0 / 16.0 * R5;
    t[4].a[5][4] = 5.0 / 4.0 - 3.0 / 4.0 * R5;
    t[4].a[5][5] = 5.0 / 2.0 - 1.0 / 2.0 * R5;
    t[4].b[0] = 1.0 / 12.0; t[4].b[4] = 5.0 / 12.0; t[4].b[5] = 5.0 / 12.0; t[4].b[6] = 1.0 / 12.0;
    t[4].c[0] = 4.0 / 7.0; t[4].c[1] = 5.0 / 7.0; t[4].c[2] = 6.0 / 7.0;
    t[4].c[3] = (5.0 - R5) / 10.0; t[4].c[4] = (5.0 + R5) / 10.0; t[4].c[5] = 1.0;
    // 5 Fehlberg
    t[5].s = 6;
    t[5].a[0][0] = 1.0 / 4.0;
    t[5].a[1][0] = 3.0 / 32.0; t[5].a[1][1] = 9.0 / 32.0;
    t[5].a[2][0] = 1932.0 / 2197.0; t[5].a[2][1] = -7200.0 / 2197.0; t[5].a[2][2] = 7296.0 / 2197.0;
    t[5].a[3][0] = 439.0 / 216.0; t[5].a[3][1] = -8.0; t[5].a[3][2] = 3680.0 / 513.0; t[5].a[3][3] = -845.0 / 4104.0;
    t[5].a[4][0] = -8.0 / 27.0; t[5].a[4][1] = 2.0; t[5].a[4][2] = -3544.0 / 2565.0; t[5].a[4][3] = 1859.0 / 4104.0;
    t[5].a[4][4] = -11.0 / 40.0;
    t[5].b[0] = 16.0 / 135.0; t[5].b[2] = 6656.0 / 12825.0; t[5].b[3] = 28561.0 / 56430.0; t[5].b[4] = -9.0 / 50.0;
    t[5].b[5] = 2.0 / 55.0;
    t[5].c[1] = 1.0 / 4.0; t[5].c[2] = 3.0 / 8.0; t[5].c[3] = 12.0 / 13.0; t[5].c[4] = 1.0; t[5].c[5] = 1.0 / 2.0;
    t[5].bstar[0] = 25.0 / 216.0; t[5].bstar[2] = 1408.0 / 2565.0; t[5].bstar[3] = 2197.0 / 4104.0;
    t[5].bstar[4] = -1.0 / 5.0;
    // 6 BogackiShampine
    t[6].s = 4;
    t[6].a[0][0] = 1.0 / 2.0;
    t[6].a[1][1] = 3.0 / 4.0;
    t[6].a[2][0] = 2.0 / 9.0; t[6].a[2][1] = 1.0 / 3.0; t[6].a[2][2] = 4.0 / 9.0;
    t[6].b[0] = 2.0 / 9.0; t[6].b[1] = 1.0 / 3.0; t[6].b[2] = 4.0 / 9.0;
    t[6].c[1] = 1.0 / 2.0; t[6].c[2] = 3.0 / 4.0; t[6].c[3] = 1.0;
    t[6].bstar[0] = 7.0 / 24.0; t[6].bstar[1] = 1.0 / 4.0; t[6].bstar[2] = 1.0 / 3.0; t[6].bstar[3] = 1.0 / 8.0;
    return t;
}

/* integrate (utils/integrate/src/lib.rs:176-222) and, when fut2 is given,
 * integrate_embedded_rk's second combination (:237-251); the result goes to s->fut. */
static int integrate_general(orc_system* s, const OrcTableau& T, double dt, bool force_trad, double& time,
                             std::vector<std::vector<double>>* fut2) {
    const size_t nb = s->desc.size();
    int bad = 0;
    for (int i = 0; i < T.s; ++i) {
        for (size_t b = 0; b < nb; ++b) {
            s->fut[b] = s->now[b];
            for (int j = 0; j < i; ++j) {
                const double a = T.a[i - 1][j];
                if (a == 0.0) continue;
                const double sc = a * dt;
                std::vector<double>& f = s->fut[b];
                const std::vector<double>& kk = s->k[j][b];
                for (size_t q = 0; q < f.size(); ++q) f[q] = f[q] + sc * kk[q];
            }
        }
        const double simtime = i == 0 ? time : time + dt * T.c[i - 1];
        for (size_t b = 0; b < nb; ++b) {
            const double* z[4];
            int rc = extract(s, s->fut, (int)b, simtime, z);
            if (rc) return rc;
            bad |= rhs(s->ctx[b], s->gamma, s->fut[b].data(), z, force_trad, s->k[i][b].data(), s->work[b]);
        }
    }
    for (size_t b = 0; b < nb; ++b) {
        std::vector<double>& f = s->fut[b];
        f = s->now[b];
        for (int j = 0; j < T.s; ++j) {
            if (T.b[j] == 0.0) continue;
            const double sc = T.b[j] * dt;
            const std::vector<double>& kk = s->k[j][b];
            for (size_t q = 0; q < f.size(); ++q) f[q] = f[q] + sc * kk[q];
        }
    }
    time += dt;
    if (fut2) {
        fut2->resize(nb);
        for (size_t b = 0; b < nb; ++b) {
            std::vector<double>& f = (*fut2)[b];
            f = s->now[b];
            for (int j = 0; j < T.s; ++j) {
                if (T.bstar[j] == 0.0) continue;
                const double sc = T.bstar[j] * dt;
                const std::vector<double>& kk = s->k[j][b];
                for (size_t q = 0; q < f.size(); ++q) f[q] = f[q] + sc * kk[q];
            }
        }
    }
    return bad ? -4 : 0;
}

}  // namespace

/* ------------------------------------------------------------------------- */
/* C API                                                                      */
/* ------------------------------------------------------------------------- */

extern "C" {

int orc_op_shape(int op, int* m, int* n, int* d, int* is_h2, int* is_upwind) {
    const BlockOp<double>& b = get_op<double>(op, ORC_DIFF);
    if (!b.valid) return -1;
    *m = b.M;
    *n = b.N;
    *d = b.D;
    *is_h2 = b.h2;
    *is_upwind = b.upwind;
    return 0;
}

int orc_op_table(int op, int kind, int part, int dtype, void* out) {
    auto put = [&](auto const& b) -> int {
        using T = std::remove_cv_t<std::remove_reference_t<decltype(b.start[0])>>;
        if (!b.valid) return -1;
        T* o = static_cast<T*>(out);
        int cnt = 0;
        if (part == 0) for (int i = 0; i < b.M * b.N; ++i) o[cnt++] = b.start[i];
        else if (part == 1) for (int i = 0; i < b.D; ++i) o[cnt++] = b.diag[i];
        else if (part == 2) for (int i = 0; i < b.M * b.N; ++i) o[cnt++] = b.end[i];
        else if (part == 3) for (int i = 0; i < b.M; ++i) o[cnt++] = b.h[i];
        else return -1;
        return cnt;
    };
    if (dtype == ORC_F64) return put(get_op<double>(op, kind));
    if (dtype == ORC_F32) return put(get_op<float>(op, kind));
    return -1;
}

int orc_op_apply(int op, int dir, int kind, int dtype, const void* in, void* out, int64_t ny, int64_t nx) {
    if (dtype == ORC_F64)
        return op_apply_t<double>(op, dir, kind, static_cast<const double*>(in), static_cast<double*>(out), ny, nx);
    if (dtype == ORC_F32)
        return op_apply_t<float>(op, dir, kind, static_cast<const float*>(in), static_cast<float*>(out), ny, nx);
    return -1;
}

int orc_metrics(int op_xi, int op_eta, const double* x, const double* y, int64_t ny, int64_t nx, double* out) {
    Metrics m;
    int rc = build_metrics(op_xi, op_eta, x, y, ny, nx, m);
    if (rc) return rc;
    const int64_t n = nx * ny;
    std::memcpy(out, m.detj.data(), n * 8);
    std::memcpy(out + n, m.jxx.data(), n * 8);
    std::memcpy(out + 2 * n, m.jxy.data(), n * 8);
    std::memcpy(out + 3 * n, m.jyx.data(), n * 8);
    std::memcpy(out + 4 * n, m.jyy.data(), n * 8);
    return 0;
}

int orc_vortex(const orc_vortex_params* vp, double gamma, double t, const double* x, const double* y, int64_t n,
               double* q) {
    for (int64_t i = 0; i < n; ++i) vortex_point(*vp, gamma, t, x[i], y[i], q[i], q[n + i], q[2 * n + i], q[3 * n + i]);
    return 0;
}

int orc_rhs(int op_xi, int op_eta, double gamma, const double* q, const double* metrics, const double* zn,
            const double* zs, const double* ze, const double* zw, int64_t ny, int64_t nx, int force_trad,
            double* k) {
    const int64_t n = nx * ny;
    Metrics m;
    m.detj.assign(metrics, metrics + n);
    m.jxx.assign(metrics + n, metrics + 2 * n);
    m.jxy.assign(metrics + 2 * n, metrics + 3 * n);
    m.jyx.assign(metrics + 3 * n, metrics + 4 * n);
    m.jyy.assign(metrics + 4 * n, metrics + 5 * n);
    const BlockOp<double>& ox = get_op<double>(op_xi, ORC_DIFF);
    const BlockOp<double>& oe = get_op<double>(op_eta, ORC_DIFF);
    if (!ox.valid || !oe.valid) return -1;
    BlockCtx B{nx, ny, op_xi, op_eta, ox.upwind && oe.upwind, &m};
    Work w;
    const double* z[4] = {zn, zs, ze, zw};
    return rhs(B, gamma, q, z, force_trad != 0, k, w) ? -4 : 0;
}

double orc_h2_err(int op_xi, int op_eta, const double* a, const double* b, int64_t ny, int64_t nx) {
    return h2_err(op_xi, op_eta, a, b, ny, nx);
}

int orc_interpolate(int op, int fine2coarse, int dtype, const void* in, int64_t n_in, void* out, int64_t n_out) {
    if (op < 0 || op > 3 || !in || !out || (dtype != ORC_F64 && dtype != ORC_F32)) return -1;
    const bool f2c = fine2coarse != 0;
    if (f2c ? !interp_sizes_ok(op, n_in, n_out) : !interp_sizes_ok(op, n_out, n_in)) return -1;
    if (dtype == ORC_F64)
        interpolate(static_cast<const double*>(in), n_in, static_cast<double*>(out), n_out, kInterp[op][f2c]);
    else
        interpolate(static_cast<const float*>(in), n_in, static_cast<float*>(out), n_out, kInterp32[op][f2c]);
    return 0;
}

orc_system* orc_system_create(const orc_block_desc* blocks, int nblocks, double gamma) {
    orc_system* s = new orc_system();
    s->gamma = gamma;
    s->desc.assign(blocks, blocks + nblocks);
    for (int d = 0; d < 4; ++d) {
        s->mg[d].resize(nblocks);
        for (int b = 0; b < nblocks; ++b) {
            if (blocks[b].bc_kind[d] == ORC_BC_MULTIGRID && blocks[b].bc_mg[d] && blocks[b].bc_mg_count[d] > 0)
                s->mg[d][b].assign(blocks[b].bc_mg[d], blocks[b].bc_mg[d] + 3 * blocks[b].bc_mg_count[d]);
            s->desc[b].bc_mg[d] = nullptr;
        }
    }
    s->x.resize(nblocks);
    s->y.resize(nblocks);
    s->metrics.resize(nblocks);
    s->ctx.resize(nblocks);
    s->now.resize(nblocks);
    s->fut.resize(nblocks);
    for (auto& kk : s->k) kk.resize(nblocks);
    for (auto& e : s->ebuf) e.resize(nblocks);
    s->work.resize(nblocks);
    for (int b = 0; b < nblocks; ++b) {
        const orc_block_desc& D = blocks[b];
        const int64_t n = D.nx * D.ny;
        s->x[b].assign(D.x, D.x + n);
        s->y[b].assign(D.y, D.y + n);
        if (build_metrics(D.op_xi, D.op_eta, D.x, D.y, D.ny, D.nx, s->metrics[b])) {
            delete s;
            return nullptr;
        }
        const bool upw = get_op<double>(D.op_xi, ORC_DIFF).upwind && get_op<double>(D.op_eta, ORC_DIFF).upwind;
        s->ctx[b] = BlockCtx{D.nx, D.ny, D.op_xi, D.op_eta, upw, &s->metrics[b]};
        s->now[b].assign(4 * n, 0.0);
        s->fut[b].assign(4 * n, 0.0);
        for (auto& kk : s->k) kk[b].assign(4 * n, 0.0);
        s->desc[b].x = s->x[b].data();
        s->desc[b].y = s->y[b].data();
    }
    return s;
}

void orc_system_destroy(orc_system* s) { delete s; }

int orc_system_set_vortex(orc_system* s, const orc_vortex_params* vp) {
    s->vp = *vp;
    return 0;
}

int orc_system_init_vortex(orc_system* s, double t) {
    for (size_t b = 0; b < s->desc.size(); ++b) {
        const int64_t n = s->desc[b].nx * s->desc[b].ny;
        orc_vortex(&s->vp, s->gamma, t, s->x[b].data(), s->y[b].data(), n, s->now[b].data());
    }
    return 0;
}

int orc_system_set_state(orc_system* s, int block, const double* q) {
    if (block < 0 || block >= (int)s->desc.size()) return -1;
    std::memcpy(s->now[block].data(), q, s->now[block].size() * 8);
    return 0;
}

int orc_system_get_state(const orc_system* s, int block, double* q) {
    if (block < 0 || block >= (int)s->desc.size()) return -1;
    std::memcpy(q, s->now[block].data(), s->now[block].size() * 8);
    return 0;
}

int orc_system_get_metrics(const orc_system* s, int block, double* out) {
    if (block < 0 || block >= (int)s->desc.size()) return -1;
    const Metrics& m = s->metrics[block];
    const int64_t n = (int64_t)m.detj.size();
    std::memcpy(out, m.detj.data(), n * 8);
    std::memcpy(out + n, m.jxx.data(), n * 8);
    std::memcpy(out + 2 * n, m.jxy.data(), n * 8);
    std::memcpy(out + 3 * n, m.jyx.data(), n * 8);
    std::memcpy(out + 4 * n, m.jyy.data(), n * 8);
    return 0;
}

int orc_system_advance(orc_system* s, int64_t nsteps, double dt, int force_trad) {
    for (int64_t i = 0; i < nsteps; ++i) {
        int rc = advance_step(s, dt, force_trad != 0);
        if (rc) return rc;
    }
    return 0;
}

int orc_system_advance_tableau(orc_system* s, int tableau, int64_t nsteps, double dt, int force_trad) {
    static const std::vector<OrcTableau> tabs = orc_tableaus();
    if (tableau < 0 || tableau >= (int)tabs.size()) return -1;
    for (int64_t i = 0; i < nsteps; ++i) {
        int rc = integrate_general(s, tabs[tableau], dt, force_trad != 0, s->time, nullptr);
        if (rc) return rc;
        std::swap(s->now, s->fut);
    }
    return 0;
}

/* euler::System::advance_adaptive (euler/src/lib.rs:149-186), as written: a local time starting
 * at 0 that integrate advances by the step and an accepted step advances once more; the error
 * is h2_err of the previous state against the low-order result.  Single block. */
int orc_system_advance_adaptive(orc_system* s, double dt, double* guess_dt, double maxerr) {
    static const std::vector<OrcTableau> tabs = orc_tableaus();
    if (s->desc.size() != 1) return -1;
    const orc_block_desc& D = s->desc[0];
    std::vector<std::vector<double>> sys2;
    double time = 0.0;
    while (time < dt) {
        int rc = integrate_general(s, tabs[6], *guess_dt, false, time, &sys2);
        if (rc) return rc;
        const double err = orc_h2_err(D.op_xi, D.op_eta, s->now[0].data(), sys2[0].data(), D.ny, D.nx);
        if (err < maxerr) {
            time += *guess_dt;
            std::swap(s->now, s->fut);
            *guess_dt *= 1.05;
        } else {
            *guess_dt *= 0.8;
        }
    }
    return 0;
}

double orc_system_time(const orc_system* s) { return s->time; }
void orc_system_set_time(orc_system* s, double t) { s->time = t; }

/* SingleThreadedSystem::max_dt (multigrid/src/system.rs:542-589) */
double orc_system_max_dt(const orc_system* s) {
    bool is_h2 = false;
    for (auto& D : s->desc)
        is_h2 = is_h2 || get_op<double>(D.op_xi, ORC_DIFF).h2 || get_op<double>(D.op_eta, ORC_DIFF).h2;
    const double c_max = is_h2 ? 0.5 : 1.0;
    double max_dt = INFINITY;
    for (size_t b = 0; b < s->desc.size(); ++b) {
        const int64_t nx = s->desc[b].nx, ny = s->desc[b].ny, n = nx * ny;
        const double* q = s->now[b].data();
        const Metrics& m = s->metrics[b];
        double max_u = 0.0, max_v = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            const double u = q[n + i] / q[i];
            const double v = q[2 * n + i] / q[i];
            const double uhat = m.jxx[i] * u + m.jxy[i] * v;
            const double vhat = m.jyx[i] * u + m.jyy[i] * v;
            max_u = std::fmax(max_u, std::fabs(uhat));
            max_v = std::fmax(max_v, std::fabs(vhat));
        }
        const double dx = 1.0 / double(nx), dy = 1.0 / double(ny);
        const double c_dt = std::fmax(max_u / dx, max_v / dy);
        max_dt = std::fmin(max_dt, c_max / c_dt);
    }
    return max_dt;
}

/* SingleThreadedSystem::error (multigrid/src/system.rs:618-635): sum over blocks of h2_err
 * against the vortex at the current time. */
double orc_system_error(const orc_system* s) {
    double e = 0.0;
    for (size_t b = 0; b < s->desc.size(); ++b) {
        const orc_block_desc& D = s->desc[b];
        const int64_t n = D.nx * D.ny;
        std::vector<double> v(4 * n);
        orc_vortex(&s->vp, s->gamma, s->time, s->x[b].data(), s->y[b].data(), n, v.data());
        e += h2_err(D.op_xi, D.op_eta, s->now[b].data(), v.data(), D.ny, D.nx);
    }
    return e;
}

int orc_systems_advance(orc_system** systems, int n, const int64_t* nsteps, const double* dt, int nthreads) {
    if (nthreads < 1) nthreads = 1;
    std::atomic<int> next{0};
    std::atomic<int> err{0};
    auto worker = [&]() {
        for (;;) {
            int i = next.fetch_add(1);
            if (i >= n) break;
            int rc = orc_system_advance(systems[i], nsteps[i], dt[i], 0);
            if (rc) err.store(rc);
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nthreads; ++t) th.emplace_back(worker);
    worker();
    for (auto& t : th) t.join();
    return err.load();
}

}  // extern "C"
