// Device-side data layout and pointwise physics of the Euler hot path.
//
// HBM layout of a system (all arrays element-indexed, every plane padded to a multiple of
// 64 elements so each plane starts 256-byte aligned):
//   state planes   : block b owns 4 planes (rho, rhou, rhov, e) at q_off[b] + c*npad[b]
//   metric planes  : 5 planes (detj, J dxi/dx, J dxi/dy, J deta/dx, J deta/dy) at m_off[b]
//   coordinates    : 2 planes (x, y) at x_off[b]
// A plane is C-order (ny, nx) with x contiguous, the reference's Field layout
// (euler/src/lib.rs:190-219).
#pragma once

#include <cstdint>

namespace sbp {

enum { BC_THIS = 0, BC_GRID = 1, BC_VORTEX = 2, BC_INTERPOLATE = 3, BC_MULTIGRID = 4, BC_EVAL = 5 };
enum { NORTH = 0, SOUTH = 1, EAST = 2, WEST = 3 };
// Device status bits (one word per system, read by the host after steps).  STATUS_BAD_LAUNCH:
// a stage kernel specialised for one RK stage class was launched for another, or given a tile
// holding closure outputs of both ends of a line (host bugs).
enum : unsigned { STATUS_RHO = 1u, STATUS_P = 2u, STATUS_DETJ = 4u, STATUS_NAN = 8u, STATUS_BAD_LAUNCH = 16u };

struct BlockDev {
    int nx, ny, npad;
    int op_xi, op_eta;
    int instance;
    int simd_f64;  // columns j < simd_f64 use fused column sums (f64x8 lanes)
    int simd_f32;  // same for f32x16 lanes
    int bc_kind[4];
    int bc_nb[4];
    int bc_aux[4];   // BC_INTERPOLATE: interpolation operator; BC_MULTIGRID: first segment in the table
    int bc_aux2[4];  // BC_MULTIGRID: number of segments
    int64_t q_off, m_off, x_off;
    int64_t e_off;  // slot of this block's first edge point in the edge-k buffer (see edge_index)
    int64_t r_off;  // compensated f32: this block's free-stream dissipation plane (see InstanceDev)
    double idx_xi, idx_eta;  // 1/(1/(n-1)) per direction, f64
    float idx_xi_f, idx_eta_f;
    double hi_xi, hi_eta;  // SAT penalty (n-1)/H_0 (euler/src/lib.rs:1033-1037)
};

// Position of edge point (row, col) among a block's 2 nx + 2 ny - 4 edge points: the first row,
// the last row, then the first and the last column without their corner points.
__host__ __device__ __forceinline__ int edge_index(int row, int col, int nx, int ny) {
    if (row == 0) return col;
    if (row == ny - 1) return nx + col;
    if (col == 0) return 2 * nx + row - 1;
    return 2 * nx + ny - 2 + row - 1;  // col == nx - 1
}
__host__ __device__ constexpr int64_t edge_count(int64_t nx, int64_t ny) { return 2 * nx + 2 * ny - 4; }

// Reference state of the compensated-f32 form, as f32 constants of the deviation arithmetic:
// the conserved state q_r = (rho_r, m_r, n_r, e_r), velocity (u_r, v_r), pressure p_r,
// total enthalpy H_r = e_r + p_r, sound speed c_r and c_r^2, gamma / rho_r.  It is always the
// reference's vortex free stream (rho_r = 1, u_r = 1, v_r = 0), which the stage kernels use.
struct RefState {
    float q[4];
    float u, v, p, h, c, c2, g_rho;
};

struct InstanceDev {
    double dt, time;
    double ca[3];  // A-tableau entries times dt for stages 2..4 (0.5dt, 0.5dt, 1.0dt)
    double cb[4];  // B-tableau entries times dt (dt/6, dt/3, dt/3, dt/6)
    int nvort;
    double x0[5], y0[5], rstar[5], eps[5];
    double mach;
    // Compensated-f32 systems store the state of every block of the instance as its deviation
    // from qref, the free stream of the instance's vortex parameters (rho 1, u 1, v 0,
    // p 1/(gamma M^2)); f64 systems store the state itself.
    double qref[4];
    RefState ref;
    // Per-vortex constants of vortex_point_fast (set with the reference state): the factor of
    // e^f in 1 - K e^f, the factor of dx e^(f/2) and dy e^(f/2) in the velocity, 1 / r*^2; and
    // the free-stream pressure and 1 / (gamma - 1).
    double vk_b[5], vk_u[5], vk_f[5];
    double v_pinf, v_igm1;
};

// pressure (euler/src/lib.rs:478-480)
template <class T>
__device__ __forceinline__ T pressure(T g, T rho, T rhou, T rhov, T e) {
    return (g - T(1)) * (e - (rhou * rhou + rhov * rhov) / (T(2) * rho));
}

// VortexParameters::evaluate (euler/src/vortex.rs:26-113) at one point, f64.  With
// POW_FREE and gamma == 1.4 the powers are formed from square roots and products: with
// b = 1 - K e^f, rho = b^(1/(gamma-1)) = b^2.5 = b^2 sqrt(b) and rho^gamma = b^3.5 = b^3 sqrt(b),
// and e^(f/2) = sqrt(e^f); each is correctly rounded, so the values differ from pow and exp in
// the last bits only.  The SAT boundary data use that form (it removes the two f64 pow and one
// exp of every vortex edge point at every stage); initial data and the error norms use pow.
template <bool POW_FREE = false>
__device__ inline void vortex_point(const InstanceDev& I, double gamma, double t, double x, double y, double q[4]) {
    const double PI = 3.14159265358979323846;
    const double m = I.mach;
    const double p_inf = 1.0 / (gamma * m * m);
    const double rho_inf = 1.0, u_inf = 1.0, v_inf = 0.0;
    const double e_inf = p_inf / (gamma - 1.0) + rho_inf * (u_inf * u_inf + v_inf * v_inf) / 2.0;
    if (I.nvort <= 0) {
        // The reference writes rhou twice here and leaves rhov untouched (vortex.rs:56-61);
        // the evident intent is the free stream, which is what is written.
        q[0] = rho_inf;
        q[1] = rho_inf * u_inf;
        q[2] = rho_inf * v_inf;
        q[3] = e_inf;
        return;
    }
    for (int iv = 0; iv < I.nvort; ++iv) {
        const double rstar = I.rstar[iv], eps = I.eps[iv];
        const double dx = (x - I.x0[iv]) - t;
        const double dy = y - I.y0[iv];
        const double f = (1.0 - (dx * dx + dy * dy)) / (rstar * rstar);
        double r, p, ef2;
        if (POW_FREE && gamma == 1.4) {
            const double ef = exp(f);
            const double b = 1.0 - eps * eps * (gamma - 1.0) * m * m / (8.0 * PI * PI * p_inf * rstar * rstar) * ef;
            const double sb = sqrt(b);
            r = b * b * sb;
            p = b * b * b * sb * p_inf;
            ef2 = sqrt(ef);
        } else {
            r = pow(1.0 - eps * eps * (gamma - 1.0) * m * m / (8.0 * PI * PI * p_inf * rstar * rstar) * exp(f),
                    1.0 / (gamma - 1.0));
            p = pow(r, gamma) * p_inf;
            ef2 = exp(f / 2.0);
        }
        const double u = 1.0 - eps * dy / (2.0 * PI * sqrt(p_inf) * rstar * rstar) * ef2;
        const double v = eps * dx / (2.0 * PI * sqrt(p_inf) * rstar * rstar) * ef2;
        if (iv == 0) {
            q[0] = r;
            q[1] = r * u;
            q[2] = r * v;
            q[3] = p / (gamma - 1.0) + r * (u * u + v * v) / 2.0;
        } else {
            q[0] += r - rho_inf;
            q[1] += r * u - rho_inf * u_inf;
            q[2] += r * v - rho_inf * v_inf;
            q[3] += (p / (gamma - 1.0) + r * (u * u + v * v) / 2.0) - e_inf;
        }
    }
}

// vortex_point<true> for gamma = 1.4 with the instance constants precomputed on the host
// (InstanceDev::vk_*) and no division: the boundary data of compensated-f32 systems, whose f64
// SAT terms need not follow the reference's operation order (values differ in the last bits).
__device__ inline void vortex_point_fast(const InstanceDev& I, double t, double x, double y, double q[4]) {
    const double p_inf = I.v_pinf, igm1 = I.v_igm1;
    const double e_inf = p_inf * igm1 + 0.5;  // rho_inf = u_inf = 1, v_inf = 0
    if (I.nvort <= 0) {
        q[0] = 1.0;
        q[1] = 1.0;
        q[2] = 0.0;
        q[3] = e_inf;
        return;
    }
    for (int iv = 0; iv < I.nvort; ++iv) {
        const double dx = (x - I.x0[iv]) - t;
        const double dy = y - I.y0[iv];
        const double ef = exp((1.0 - (dx * dx + dy * dy)) * I.vk_f[iv]);
        const double b = 1.0 - I.vk_b[iv] * ef;
        const double sb = sqrt(b);
        const double r = b * b * sb;
        const double p = b * r * p_inf;
        const double w = I.vk_u[iv] * sqrt(ef);
        const double u = 1.0 - w * dy, v = w * dx;
        const double en = p * igm1 + 0.5 * r * (u * u + v * v);
        if (iv == 0) {
            q[0] = r;
            q[1] = r * u;
            q[2] = r * v;
            q[3] = en;
        } else {
            q[0] += r - 1.0;
            q[1] += r * u - 1.0;
            q[2] += r * v;
            q[3] += en - e_inf;
        }
    }
}

// SAT_characteristic (euler/src/lib.rs:1150-1252) at one edge point, f64:
// k += hi*tau * T * ((L + sign|L|) o (T^-1 (y - z))).
__device__ inline void sat_point(double gamma, const double y[4], const double z[4], double hi, double sign,
                                 double tau, double detj, double detj_d_dx, double detj_d_dy, double k[4]) {
    const double rho = y[0], rhou = y[1], rhov = y[2], e = y[3];
    const double kx_ = detj_d_dx / detj;
    const double ky_ = detj_d_dy / detj;
    const double r = hypot(kx_, ky_);
    const double kx = kx_ / r, ky = ky_ / r;
    const double u = rhou / rho, v = rhov / rho;
    const double theta = kx * u + ky * v;
    const double p = pressure<double>(gamma, rho, rhou, rhov, e);
    const double c = sqrt(gamma * p / rho);
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
    const double hyp = hypot(kx_, ky_);
    const double L[4] = {U, U, U + c * hyp, U - c * hyp};
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
#pragma unroll
    for (int row = 0; row < 4; ++row)
#pragma unroll
        for (int col = 0; col < 4; ++col) TIres[row] += TI[row][col] * res[col];
    double LTIres[4];
#pragma unroll
    for (int row = 0; row < 4; ++row) LTIres[row] = (L[row] + sign * fabs(L[row])) * TIres[row];
    double TLTIres[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int row = 0; row < 4; ++row)
#pragma unroll
        for (int col = 0; col < 4; ++col) TLTIres[row] += T[row][col] * LTIres[col];
#pragma unroll
    for (int comp = 0; comp < 4; ++comp) k[comp] += hi * tau * TLTIres[comp];
}

// Knuth's TwoSum: s + e == a + b exactly (round-to-nearest, no FMA involved).
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
    s = __fadd_rn(a, b);
    const float bb = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}

// Dekker's FastTwoSum (|a| >= |b|).
__device__ __forceinline__ void fast_two_sum(float a, float b, float& s, float& e) {
    s = __fadd_rn(a, b);
    e = __fsub_rn(b, __fsub_rn(s, a));
}

// (hi, lo) += inc, keeping hi + lo as an unevaluated sum with |lo| <= ulp(hi)/2.
__device__ __forceinline__ void comp_add(float& hi, float& lo, float inc) {
    float s, e;
    two_sum(hi, inc, s, e);
    const float t = __fadd_rn(lo, e);
    fast_two_sum(s, t, hi, lo);
}

}  // namespace sbp
