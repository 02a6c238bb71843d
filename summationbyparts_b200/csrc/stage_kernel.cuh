// Fused RK4 stage kernel.
//
// One launch computes, for every point of every scheduled tile, the Euler right-hand side
//   k = ((-dE/dxi - dF/deta) + diss_xi(alpha_u q) + diss_eta(alpha_v q)) / detJ
// (RHS_upwind, euler/src/lib.rs:571-616; RHS_trad 483-515 without the dissipation terms) and
// performs this stage's share of the RK4 update (integrate::<Rk4>,
// utils/integrate/src/lib.rs:176-222):
//   stage 0: acc  = prev + (b0 dt) k ; next = prev + (a dt) k
//   stage 1: acc += (b1 dt) k        ; next = prev + (a dt) k
//   stage 2: acc += (b2 dt) k        ; next = prev + (a dt) k
//   stage 3: new  = acc + (b3 dt) k
// which is the reference's sequence fut = prev; fut += b_j dt k_j (j = 0..3) evaluated
// incrementally, so the k_j of interior points never go to memory.  Points on a block edge
// store their k in the edge-k buffer instead; the edge kernel (sat_kernel, launched right after
// on the same stream) adds the characteristic SATs in the order north, south, east, west
// (SAT_characteristics, euler/src/lib.rs:1002-1013) and does their update.  The SAT of one
// point is a long dependent f64 chain (vortex data, two hypot, a dozen divisions); evaluated by
// a few threads of a tile it held the whole CTA at the next barrier, in a launch of its own it
// runs one thread per edge point.
//
// Work decomposition.  A persistent grid of 256-thread CTAs walks a list of (block, y0, x0)
// output tiles of TY rows x 32 columns.  Lane = column, warp w owns rows w*R .. w*R+R-1
// (R = TY/8).  Phase 1 evaluates the pointwise quantities once per point of the
// cross-shaped region the stencils read -- Ehat and alpha_u q on the tile rows widened by the
// xi halo, Fhat and alpha_v q on the tile columns widened by the eta halo (boundary closures
// widen it to the M x N block) -- into shared memory.  Phase 2 applies the 8 xi and 8 eta
// stencils from shared memory: the eta sums of a thread's R rows share one register window
// (R + D - 1 loads for R outputs); interior rows and columns take branch-free paths and only
// the warps on a block edge run the closure code.
//
// Precision: T = double reproduces the reference's f64 arithmetic operation by operation
// (compile with -fmad=false).  T = float with COMP = true runs fluxes, dissipation and
// stencils in f32 and keeps the RK4 state as a (hi, lo) f32 pair; the step's increment
// sum_j (b_j dt) k_j is accumulated in f32 and added to the pair once per step with TwoSum;
// the f32 metrics hold 1 / J (rounded from f64), so the flux divergence is scaled by a product.
// The SAT terms are computed in f64 from f64 metrics.
#pragma once

#include <type_traits>

#include "euler_device.cuh"
#include "eval_program.cuh"
#include "interp.cuh"
#include "sbp_ops.cuh"

namespace sbp {

constexpr int kStageThreads = 256;
constexpr int kStageWarps = kStageThreads / 32;
constexpr int kTileX = 32;

template <class T>
struct StageArgs {
    const BlockDev* __restrict__ blocks;
    const InstanceDev* __restrict__ inst;
    const int4* __restrict__ tiles;
    int ntiles;
    int stage;               // 0..3 (RK4), or kStageK: write k to u_out (other tableaus)
    double ctime;            // kStageK: the stage's C coefficient (SAT data at time + dt * ctime)
    const T* u_in;           // stage input state, all blocks
    const T* prev_hi;        // state at the start of the step
    const T* prev_lo;        // low part of the state (compensated precision only)
    T* acc_hi;               // RK4 accumulator (compensated form: the step's f32 increment)
    T* u_out;                // next stage input (stages 0..2)
    T* new_hi;               // new state (stage 3)
    T* new_lo;
    T* kedge;                // k of block-edge points, 4 per point (edge_index order per block)
    const double* egeo;      // compensated f32: edge geometry, kEdgeGeo per point (edge_geo_kernel)
    const int4* mg;          // MultiGrid segments (block, start, end, -) of all block sides
    const EvalDev* eval;     // expression programs of SBP_BC_EVAL sides
    double* evz;             // SBP_BC_EVAL data of the launch's edge points (eval_kernel), 4 per point
    const T* met;            // metric planes in T
    const double* met64;     // metric planes in f64 (SAT terms)
    const float* rinf;       // compensated f32, upwind: free-stream dissipation planes (BlockDev::r_off)
    const double* xy;        // coordinates
    const T* coef;           // operator tables, see coef_base
    double gamma;
    unsigned* status;
};

// Stage index of the k-only mode: the launch computes k = RHS(u_in) (SATs included) into u_out
// and updates nothing else; explicit tableaus other than RK4 combine the k on the host side.
constexpr int kStageK = 4;

// Device coefficient table (one per precision): for operator o and kind k the rows
// [start block M rows][end block M rows][interior diagonal], each row padded to kCoefRow
// elements (16-byte aligned rows), at coef_base(o, k).
constexpr int kCoefRow = 16;
constexpr int kCoefStride = (2 * 8 + 1) * kCoefRow;
__host__ __device__ constexpr int coef_base(int op, int kind) { return (2 * op + kind) * kCoefStride; }

// Tiles along a line of n outputs (tile_starts in system.cu) start at multiples of T, except that
// the last tile starts at e = n - M rounded down to even whenever a multiple of T would fall in
// (e, n): so the first tile holds every start-closure output, the last every end-closure output,
// and no tile holds outputs of both ends (n >= 2 M).  The input region of a tile is then at most
// T + 2 H wide (interior tiles and the first one: H on each side, [0, max(T + H, N)) for the
// first; the tile before the last ends at e <= n - M, so its region stops H after it), or
// max(N, M + H + 1) for the last tile, which reads from min(e - H, n - N) to n.
constexpr int region_extent(int T, int H, int M, int N) {
    const int a = T + 2 * H, b = N > M + H + 1 ? N : M + H + 1;
    return a > b ? a : b;
}

// Output rows and columns of a tile: the tile list holds (block, y0, x0, th << 16 | tw).
__device__ __forceinline__ int tile_rows(const int4& td) { return td.w >> 16; }
__device__ __forceinline__ int tile_cols(const int4& td) { return td.w & 0xffff; }

// Shared-memory geometry of one tile: xi arrays are TY rows x XP columns, eta arrays HYP rows
// x 32 columns.
template <int OPX, int OPY, int TY>
struct StageGeom {
    static constexpr int XP = region_extent(kTileX, OpShape<OPX>::H, OpShape<OPX>::M, OpShape<OPX>::N);
    static constexpr int HYP = region_extent(TY, OpShape<OPY>::H, OpShape<OPY>::M, OpShape<OPY>::N);
    static constexpr int XA = TY * XP;       // elements of one xi array
    static constexpr int YA = HYP * kTileX;  // elements of one eta array
};

// Phase-2 operands staged in shared memory by cp.async while phase 1 runs (compensated-f32
// kernel): slot 0 plane 0 of the f32 metrics (1 / J), then up to three state arrays x 4
// components (see stage_operands).
constexpr int kStageSlots = 13;
__host__ __device__ constexpr int staged_elems(bool comp, int TY) { return comp ? kStageSlots * TY * kTileX : 0; }

template <int OPX, int OPY, int TY, class T>
constexpr size_t stage_smem(bool upw, bool comp) {
    using G = StageGeom<OPX, OPY, TY>;
    return sizeof(T) * ((size_t)(4 * G::XA + 4 * G::YA) * (upw ? 2 : 1) + staged_elems(comp, TY));
}

// Characteristic SAT of one edge point (euler/src/lib.rs:1150-1252), f64, written row by row
// so no 4x4 matrix is ever live.  Same operations in the same order as the reference.
__device__ __forceinline__ void sat_point_rows(double gamma, const double y[4], const double z[4], double hi,
                                               double sign, double tau, double detj, double detj_d_dx,
                                               double detj_d_dy, double k[4]) {
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
    const double alpha = rho / (1.41421356237309504880 * c);
    const double phi2_c2 = (phi2 + c * c) / (gamma - 1.0);
    const double U = kx_ * u + ky_ * v;
    const double hyp = hypot(kx_, ky_);
    const double beta = 1.0 / (2.0 * c * c);
    const double cc = c * c, gm1 = gamma - 1.0;
    const double r0 = rho - z[0], r1 = rhou - z[1], r2 = rhov - z[2], r3 = e - z[3];
    double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
    t0 += (1.0 - phi2 / cc) * r0;
    t0 += (gm1 * u / cc) * r1;
    t0 += (gm1 * v / cc) * r2;
    t0 += (-gm1 / cc) * r3;
    t1 += (-(ky * u - kx * v) / rho) * r0;
    t1 += (ky / rho) * r1;
    t1 += (-kx / rho) * r2;
    t1 += 0.0 * r3;
    t2 += (beta * (phi2 - c * theta)) * r0;
    t2 += (beta * (kx * c - gm1 * u)) * r1;
    t2 += (beta * (ky * c - gm1 * v)) * r2;
    t2 += (beta * gm1) * r3;
    t3 += (beta * (phi2 + c * theta)) * r0;
    t3 += (-beta * (kx * c + gm1 * u)) * r1;
    t3 += (-beta * (ky * c + gm1 * v)) * r2;
    t3 += (beta * gm1) * r3;
    const double L0 = U, L2 = U + c * hyp, L3 = U - c * hyp;
    const double l0 = (L0 + sign * fabs(L0)) * t0;
    const double l1 = (L0 + sign * fabs(L0)) * t1;
    const double l2 = (L2 + sign * fabs(L2)) * t2;
    const double l3 = (L3 + sign * fabs(L3)) * t3;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    s0 += 1.0 * l0;
    s0 += 0.0 * l1;
    s0 += alpha * l2;
    s0 += alpha * l3;
    s1 += u * l0;
    s1 += ky * l1;
    s1 += (alpha * (u + kx * c)) * l2;
    s1 += (alpha * (u - kx * c)) * l3;
    s2 += v * l0;
    s2 += (-kx) * l1;
    s2 += (alpha * (v + ky * c)) * l2;
    s2 += (alpha * (v - ky * c)) * l3;
    s3 += (phi2 / gm1) * l0;
    s3 += (rho * (ky * u - kx * v)) * l1;
    s3 += (alpha * (phi2_c2 + c * theta)) * l2;
    s3 += (alpha * (phi2_c2 - c * theta)) * l3;
    const double ht = hi * tau;
    k[0] += ht * s0;
    k[1] += ht * s1;
    k[2] += ht * s2;
    k[3] += ht * s3;
}

// sat_point_rows with five reciprocals in place of its divisions and sqrt(kx^2 + ky^2) in place
// of hypot (no overflow at these magnitudes): the SAT of compensated-f32 systems, still f64, whose
// last bits need not follow the reference's operation order.
__device__ __forceinline__ void sat_point_fast(double gamma, const double y[4], const double z[4], double hi,
                                               double sign, double tau, double detj, double detj_d_dx,
                                               double detj_d_dy, double igm1, double k[4]) {
    const double rho = y[0], rhou = y[1], rhov = y[2], e = y[3];
    const double ij = 1.0 / detj;
    const double kx_ = detj_d_dx * ij, ky_ = detj_d_dy * ij;
    const double hyp = sqrt(kx_ * kx_ + ky_ * ky_);
    const double ih = 1.0 / hyp;
    const double kx = kx_ * ih, ky = ky_ * ih;
    const double irho = 1.0 / rho;
    const double u = rhou * irho, v = rhov * irho;
    const double gm1 = gamma - 1.0;
    const double q2 = u * u + v * v;
    const double p = gm1 * (e - 0.5 * (rhou * u + rhov * v));
    const double cc = gamma * p * irho;
    const double c = sqrt(cc);
    const double icc = 1.0 / cc;
    const double theta = kx * u + ky * v;
    const double phi2 = 0.5 * gm1 * q2;
    const double alpha = 0.70710678118654752440 * rho * c * icc;  // rho / (sqrt(2) c)
    const double phi2_c2 = (phi2 + cc) * igm1;
    const double U = kx_ * u + ky_ * v;
    const double beta = 0.5 * icc;
    const double r0 = rho - z[0], r1 = rhou - z[1], r2 = rhov - z[2], r3 = e - z[3];
    const double gc = gm1 * icc;
    const double t0 = (1.0 - phi2 * icc) * r0 + gc * (u * r1 + v * r2 - r3);
    const double w = ky * u - kx * v;
    const double t1 = irho * (-w * r0 + ky * r1 - kx * r2);
    const double t2 = beta * ((phi2 - c * theta) * r0 + (kx * c - gm1 * u) * r1 + (ky * c - gm1 * v) * r2 + gm1 * r3);
    const double t3 = beta * ((phi2 + c * theta) * r0 - (kx * c + gm1 * u) * r1 - (ky * c + gm1 * v) * r2 + gm1 * r3);
    const double L2 = U + c * hyp, L3 = U - c * hyp;
    const double f0 = U + sign * fabs(U);
    const double l0 = f0 * t0, l1 = f0 * t1;
    const double l2 = (L2 + sign * fabs(L2)) * t2;
    const double l3 = (L3 + sign * fabs(L3)) * t3;
    const double a2 = alpha * l2, a3 = alpha * l3;
    const double ht = hi * tau;
    k[0] += ht * (l0 + a2 + a3);
    k[1] += ht * (u * l0 + ky * l1 + (u + kx * c) * a2 + (u - kx * c) * a3);
    k[2] += ht * (v * l0 - kx * l1 + (v + ky * c) * a2 + (v - ky * c) * a3);
    k[3] += ht * (phi2 * igm1 * l0 + rho * w * l1 + (phi2_c2 + c * theta) * a2 + (phi2_c2 - c * theta) * a3);
}

// Pointwise quantities of one point (fluxes, euler/src/lib.rs:680-735; upwind_dissipation
// 619-674) from its state qv and metrics m = (dxi/dx, dxi/dy, deta/dx, deta/dy), each times
// detJ.  Writes the xi-direction values (Ehat, alpha_u q) and/or eta-direction values (Fhat,
// alpha_v q) into shared memory at the given slots.
template <class T, bool UPW, bool EXACT>
__device__ __forceinline__ void pointwise(const T qv[4], const T m[4], T gamma, T* sxi, int xa, T* seta, int ya,
                                          bool want_xi, bool want_eta, unsigned& bad) {
    const T rho = qv[0], rhou = qv[1], rhov = qv[2], e = qv[3];
    T E[4], F[4];
    T p_, u = T(0), v = T(0), c = T(0);
    if constexpr (EXACT) {
        // the reference's operations, each division rounded on its own
        p_ = pressure<T>(gamma, rho, rhou, rhov, e);
        E[1] = rhou * rhou / rho + p_;
        E[2] = rhou * rhov / rho;
        E[3] = rhou * (e + p_) / rho;
        F[2] = rhov * rhov / rho + p_;
        F[3] = rhov * (e + p_) / rho;
        if constexpr (UPW) {
            u = rhou / rho;
            v = rhov / rho;
            c = sqrt(gamma * p_ / rho);
        }
    } else {
        // f32 bulk: one reciprocal of rho shared by every quotient
        const T ri = T(1) / rho;
        u = rhou * ri;
        v = rhov * ri;
        p_ = (gamma - T(1)) * (e - T(0.5) * (rhou * u + rhov * v));
        E[1] = rhou * u + p_;
        E[2] = rhou * v;
        E[3] = u * (e + p_);
        F[2] = rhov * v + p_;
        F[3] = v * (e + p_);
        if constexpr (UPW) c = sqrt(gamma * p_ * ri);
    }
    E[0] = rhou;
    F[0] = rhov;
    F[1] = E[2];
    if constexpr (UPW) {
        if (!(rho > T(0))) bad |= STATUS_RHO;
        if (!(p_ > T(0))) bad |= STATUS_P;
    }
    if (want_xi) {
        const T jxx = m[0], jxy = m[1];
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) sxi[cc * xa] = jxx * E[cc] + jxy * F[cc];
        if constexpr (UPW) {
            const T uhat = jxx * u + jxy * v;
            const T au = fabs(uhat) + c * sqrt(jxx * jxx + jxy * jxy);
            T* d = sxi + 4 * xa;
            d[0] = au * rho;
            d[xa] = au * rhou;
            d[2 * xa] = au * rhov;
            d[3 * xa] = au * e;
        }
    }
    if (want_eta) {
        const T jyx = m[2], jyy = m[3];
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) seta[cc * ya] = jyx * E[cc] + jyy * F[cc];
        if constexpr (UPW) {
            const T vhat = jyx * u + jyy * v;
            const T av = fabs(vhat) + c * sqrt(jyx * jyx + jyy * jyy);
            T* d = seta + 4 * ya;
            d[0] = av * rho;
            d[ya] = av * rhou;
            d[2 * ya] = av * rhov;
            d[3 * ya] = av * e;
        }
    }
}

// Pointwise quantities of the compensated-f32 form, on deviations.  The state is stored as its
// deviation d = q - q_r from the instance's reference state (its free stream), and every
// quantity the stencils read is formed as its own deviation from the value at q_r:
//   Ehat' = Jxi_x (E(q) - E(q_r)) + Jxi_y (F(q) - F(q_r)),   Fhat' likewise with Jeta,
//   (alpha q)' = alpha_u q - alpha_u,r q_r = alpha_u d + (alpha_u - alpha_u,r) q_r,
// where alpha_u,r is alpha_u at q_r on the point's metrics.  Each deviation is evaluated from d
// with algebra that subtracts no two large numbers (below), so its f32 rounding error is
// relative to the deviation, not to the state: for the vortex runs that is two to three orders
// of magnitude smaller.  The parts dropped from the stencil inputs are restored exactly or
// vanish: the fluxes of q_r are constants times the metrics, whose discrete divergence is the
// metric identity d/dxi(Jxi) + d/deta(Jeta) = 0 (the metrics are built by the same operators,
// which commute), and the dissipation of alpha_r q_r is q_r times a time-independent field that
// the system computes once in f64 (BlockDev::r_off) and the stage kernels add to k.
//   rho = rho_r + d0,  u - u_r = (d1 - u_r d0) / rho,  v - v_r = (d2 - v_r d0) / rho,
//   m u - m_r u_r = m_r du + d1 u,  n v - n_r v_r = n_r dv + d2 v,  m v - m_r v_r = m_r dv + d1 v,
//   p - p_r = (gamma - 1) (d3 - (dmu + dnv) / 2),  H - H_r = d3 + dp,
//   u H - u_r H_r = du H_r + u dH,  c^2 - c_r^2 = (gamma / rho_r) (dp rho_r - p_r d0) / rho,
//   c - c_r = (c^2 - c_r^2) / (c + c_r),  |uhat| - |uhat_r| = sign(uhat_r) duhat when both have
//   one sign (else the plain difference, whose operands are then no larger than duhat).
// The reference state is the free stream of the reference's vortex (rho_r = 1, u_r = 1,
// v_r = 0, so m_r = 1 and n_r = 0; only e_r, p_r and c_r vary with the Mach number), which
// removes the terms of m_r, n_r and v_r from the algebra above.
template <bool UPW>
__device__ __forceinline__ void pointwise_dev(const float d[4], const float m[4], float gamma, const RefState& R,
                                              float* sxi, int xa, float* seta, int ya, bool want_xi, bool want_eta,
                                              unsigned& bad) {
    const float rho = 1.0f + d[0];
    const float ri = 1.0f / rho;
    const float du = (d[1] - d[0]) * ri, v = d[2] * ri;  // u - 1 and v
    const float u = 1.0f + du;
    const float dmu = du + d[1] * u;  // m u - 1
    const float dnv = d[2] * v;       // n v
    const float mv = v + d[1] * v;    // m v
    const float dp = (gamma - 1.0f) * (d[3] - 0.5f * (dmu + dnv));
    const float dh = d[3] + dp;
    float E[4], F[4];
    E[0] = d[1];
    E[1] = dmu + dp;
    E[2] = mv;
    E[3] = du * R.h + u * dh;
    F[0] = d[2];
    F[1] = mv;
    F[2] = dnv + dp;
    F[3] = v * (R.h + dh);
    float c = 0.0f, dc = 0.0f;
    if constexpr (UPW) {
        if (!(rho > 0.0f)) bad |= STATUS_RHO;
        if (!(R.p + dp > 0.0f)) bad |= STATUS_P;
        const float dc2 = gamma * (dp - R.p * d[0]) * ri;  // c^2 - c_r^2 with rho_r = 1
        c = sqrtf(R.c2 + dc2);
        dc = dc2 / (c + R.c);
    }
    auto store = [&](float jx, float jy, float* dst, int stride) {
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) dst[cc * stride] = jx * E[cc] + jy * F[cc];
        if constexpr (UPW) {
            const float dhat = jx * du + jy * v;  // uhat - uhat_r, uhat_r = jx
            const float hat = jx + dhat;
            const float dabs = hat * jx > 0.0f ? (jx > 0.0f ? dhat : -dhat) : fabsf(hat) - fabsf(jx);
            const float s = sqrtf(jx * jx + jy * jy);
            const float a = fabsf(hat) + c * s;
            const float da = dabs + dc * s;
            float* o = dst + 4 * stride;
            o[0] = a * d[0] + da;  // q_r = (1, 1, 0, e_r)
            o[stride] = a * d[1] + da;
            o[2 * stride] = a * d[2];
            o[3 * stride] = a * d[3] + da * R.q[3];
        }
    };
    if (want_xi) store(m[0], m[1], sxi, xa);
    if (want_eta) store(m[2], m[3], seta, ya);
}

// Eta sums of R consecutive rows r0.. of one column from a shared column (stride 32), into
// out[R], scaled by idx.  `interior` (warp-uniform): every row in [M, ny-M).  EXACT selects the
// reference's lane split (fma chain for fused columns, unfused sum otherwise); without it the
// sum is a plain fma chain.  Warps holding closure rows run one N-tap loop per row with the
// row's coefficients from the table (interior rows predicate off the padding).
template <int OP, int KIND, class T, int R, bool EXACT>
__device__ __forceinline__ void eta_rows(const T* __restrict__ col, int ly0, int r0, int nrows, int ny, bool interior,
                                         bool fused, T idx, const T* __restrict__ ctab, T out[R]) {
    constexpr int M = OpShape<OP>::M, N = OpShape<OP>::N, D = OpShape<OP>::D, H = OpShape<OP>::H;
    using C = Coef<OP, KIND, T>;
    if (interior) {
        T w[R + D - 1];
#pragma unroll
        for (int j = 0; j < R + D - 1; ++j) w[j] = col[(r0 - H + j - ly0) * kTileX];
#pragma unroll
        for (int u = 0; u < R; ++u) {
            T f = T(0);
            if (!EXACT || fused) {
#pragma unroll
                for (int d = 0; d < D; ++d) f = fma_rn(w[u + d], C::diag(d), f);
            } else {
#pragma unroll
                for (int d = 0; d < D; ++d) f = f + C::diag(d) * w[u + d];
            }
            out[u] = f * idx;
        }
        return;
    }
    const T* tab = ctab + coef_base(OP, KIND);
#pragma unroll
    for (int u = 0; u < R; ++u) {
        T f = T(0);
        if (u < nrows) {
            const int r = r0 + u;
            const T* crow;
            int base, ntaps;
            if (r < M) {
                crow = tab + r * kCoefRow;
                base = 0;
                ntaps = N;
            } else if (r >= ny - M) {
                crow = tab + (M + r - (ny - M)) * kCoefRow;
                base = ny - N;
                ntaps = N;
            } else {
                crow = tab + 2 * M * kCoefRow;
                base = r - H;
                ntaps = D;
            }
            const T* w = col + (base - ly0) * kTileX;
            if (!EXACT || fused) {
#pragma unroll
                for (int k = 0; k < N; ++k)
                    if (k < ntaps) f = fma_rn(w[k * kTileX], __ldg(crow + k), f);
            } else {
#pragma unroll
                for (int k = 0; k < N; ++k)
                    if (k < ntaps) f = f + __ldg(crow + k) * w[k * kTileX];
            }
        }
        out[u] = f * idx;
    }
}

// Xi sums of one kind for the thread's rows: out[c][u] for component c and row ty0 + u of the
// tile, from the shared xi arrays `sb` (4 component arrays of XA elements, rows of XP, element 0
// = column lx0).  EXACT: the reference's unfused row order; otherwise an fma chain.  In a tile
// holding closure columns (`closure_tile`, tile-uniform) every lane loads its own coefficient
// row once (16-byte vector loads) and runs the same N-tap loop for all 4R sums, so the warp
// does not diverge; interior lanes predicate off the padding taps.
template <int OP, int KIND, class T, int R, bool EXACT, int XA, int XP>
__device__ __forceinline__ void xi_rows(const T* __restrict__ sb, int ty0, int nrows, int lx0, int col, int nx, T idx,
                                        bool closure_tile, const T* __restrict__ ctab, T out[4][R]) {
    constexpr int M = OpShape<OP>::M, N = OpShape<OP>::N, D = OpShape<OP>::D, H = OpShape<OP>::H;
    using C = Coef<OP, KIND, T>;
    if (!closure_tile) {
#pragma unroll
        for (int cc = 0; cc < 4; ++cc)
#pragma unroll
            for (int u = 0; u < R; ++u) {
                T t = T(0);
                if (u < nrows) {
                    const T* w = sb + cc * XA + (ty0 + u) * XP + (col - H - lx0);
                    if constexpr (EXACT) {
                        t = diag_unfused<OP, KIND, T>([&](int d) { return w[d]; });
                    } else {
#pragma unroll
                        for (int d = 0; d < D; ++d) t = fma_rn(w[d], C::diag(d), t);
                    }
                }
                out[cc][u] = t * idx;
            }
        return;
    }
    const T* crow;
    int base, ntaps;
    {
        const T* tab = ctab + coef_base(OP, KIND);
        if (col < M) {
            crow = tab + col * kCoefRow;
            base = 0;
            ntaps = N;
        } else if (col >= nx - M) {
            crow = tab + (M + col - (nx - M)) * kCoefRow;
            base = nx - N;
            ntaps = N;
        } else {
            crow = tab + 2 * M * kCoefRow;
            base = col - H;
            ntaps = D;
        }
    }
    constexpr int V = 16 / sizeof(T), NV = (N + V - 1) / V;
    T cf[NV * V];
    using VT = typename std::conditional<sizeof(T) == 8, double2, float4>::type;
#pragma unroll
    for (int v = 0; v < NV; ++v) *reinterpret_cast<VT*>(cf + v * V) = __ldg(reinterpret_cast<const VT*>(crow) + v);
#pragma unroll
    for (int cc = 0; cc < 4; ++cc)
#pragma unroll
        for (int u = 0; u < R; ++u) {
            T t = T(0);
            if (u < nrows) {
                const T* w = sb + cc * XA + (ty0 + u) * XP + (base - lx0);
                t = cf[0] * w[0];
#pragma unroll
                for (int k = 1; k < N; ++k)
                    if (k < ntaps) {
                        if constexpr (EXACT) t = t + cf[k] * w[k];
                        else t = fma_rn(cf[k], w[k], t);
                    }
            }
            out[cc][u] = t * idx;
        }
}

// Asynchronous global -> shared copy of one element (cp.async, sm_80+), and the wait for all
// of this thread's copies.
template <class T>
__device__ __forceinline__ void cp_async_elem(T* smem, const T* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    if constexpr (sizeof(T) == 4) asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(sa), "l"(gmem));
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// The state arrays this stage's RK update reads (compensated form), in slot order:
// stage 0: u_in (= prev_hi); stages 1, 2: delta (acc_hi), prev_hi; stage 3: delta, prev_hi, prev_lo.
template <class T>
__device__ __forceinline__ int stage_operands(const StageArgs<T>& A, const T* src[3]) {
    if (A.stage == 0) {
        src[0] = A.u_in;
        return 1;
    }
    src[0] = A.acc_hi;
    src[1] = A.prev_hi;
    src[2] = A.prev_lo;
    return A.stage < 3 ? 2 : 3;
}

// Compensated RK update of one component at element e with its operands taken from the
// staging slots (sop(a) = operand array a of this component at this point); same arithmetic
// as rk_update.  cb, ca: this stage's B and A tableau entries times dt, already in f32.
// The step's increment delta = sum_j (b_j dt) k_j is accumulated in f32 (acc_hi) and added to
// the (hi, lo) state once, in stage 3, with TwoSum.
template <class T, class SOP>
__device__ __forceinline__ void rk_update_staged(const StageArgs<T>& A, int64_t e, float cb, float ca, T kc, SOP sop) {
    if (A.stage == kStageK) {
        A.u_out[e] = kc;
        return;
    }
    const float kf = float(kc);
    if (A.stage == 0) {
        A.u_out[e] = T(float(sop(0)) + ca * kf);
        A.acc_hi[e] = T(cb * kf);
    } else if (A.stage < 3) {
        A.u_out[e] = T(float(sop(1)) + ca * kf);
        A.acc_hi[e] = T(float(sop(0)) + cb * kf);
    } else {
        const float d = float(sop(0)) + cb * kf;
        float hi = float(sop(1));
        float lo = float(sop(2));
        comp_add(hi, lo, d);
        A.new_hi[e] = T(hi);
        A.new_lo[e] = T(lo);
    }
}

// This stage's RK4 update of one component at element e (see the header comment), operands
// read from global memory.  `qv` is the stage input at the point (the step-start state in
// stage 0); cb, ca: this stage's B and A tableau entries times dt (ca unused in stage 3).
template <class T, bool COMP>
__device__ __forceinline__ void rk_update(const StageArgs<T>& A, int64_t e, T qv, T kc, double cb, double ca) {
    if (A.stage == kStageK) {
        A.u_out[e] = kc;
        return;
    }
    if constexpr (!COMP) {
        const T cbt = T(cb);
        if (A.stage == 0) {
            A.acc_hi[e] = qv + cbt * kc;
            A.u_out[e] = qv + T(ca) * kc;
        } else if (A.stage < 3) {
            const T av = A.acc_hi[e];
            const T pv = __ldg(A.prev_hi + e);
            A.acc_hi[e] = av + cbt * kc;
            A.u_out[e] = pv + T(ca) * kc;
        } else {
            A.new_hi[e] = A.acc_hi[e] + cbt * kc;
        }
    } else {
        // compensated form: see rk_update_staged
        const float cbf = float(cb);
        const float kf = float(kc);
        if (A.stage == 0) {
            A.u_out[e] = T(float(qv) + float(ca) * kf);
            A.acc_hi[e] = T(cbf * kf);
        } else if (A.stage < 3) {
            const float pv = float(__ldg(A.prev_hi + e));
            A.u_out[e] = T(pv + float(ca) * kf);
            A.acc_hi[e] = T(float(A.acc_hi[e]) + cbf * kf);
        } else {
            const float d = float(A.acc_hi[e]) + cbf * kf;
            float hi = float(A.prev_hi[e]);
            float lo = float(A.prev_lo[e]);
            comp_add(hi, lo, d);
            A.new_hi[e] = T(hi);
            A.new_lo[e] = T(lo);
        }
    }
}

// Element of a block's edge opposite to side d (north -> the block's south row, ...) at position
// k along that edge: the point whose state a neighbour's side-d SAT reads.
__device__ __forceinline__ int opposite_edge_point(int d, int k, int gnx, int gny) {
    if (d == NORTH) return k;                      // south row
    if (d == SOUTH) return (gny - 1) * gnx + k;    // north row
    if (d == EAST) return k * gnx;                 // west column
    return k * gnx + (gnx - 1);                    // east column
}

// Value of component cc of a state stored in T at a point of block Gb, as the absolute state:
// the compensated-f32 form stores deviations from the instance's reference state.
template <class T>
__device__ __forceinline__ double absolute_state(const StageArgs<T>& A, const BlockDev& Gb, int cc, T v) {
    if constexpr (sizeof(T) == 4) return double(v) + A.inst[Gb.instance].qref[cc];
    else return double(v);
}

// The time-independent data of one block-edge point the SATs read: coordinates, the f64
// metrics (detJ, J dxi/dx, J dxi/dy, J deta/dx, J deta/dy).
struct EdgeGeo {
    double x, y, m[5];
};
// Compensated-f32 systems gather the geometry of their block-edge points once into one contiguous
// 64-byte record per point (slot e_off + edge_index: x, y, detJ, the 4 metric terms, padding;
// edge_geo_kernel), which the edge kernel reads instead of seven scattered sectors (the first and
// last columns of a block are nx elements apart).
constexpr int kEdgeGeo = 8;
template <class T>
__device__ __forceinline__ EdgeGeo edge_geo(const StageArgs<T>& A, const BlockDev& B, int pt) {
    const int64_t np = B.npad;
    const double* m64 = A.met64 + B.m_off;
    const double* xy = A.xy + B.x_off;
    EdgeGeo g;
    g.x = xy[pt];
    g.y = xy[np + pt];
#pragma unroll
    for (int c = 0; c < 5; ++c) g.m[c] = m64[c * np + pt];
    return g;
}

// SATs of one block-edge point in the reference's order N, S, E, W; k updated in place.
template <class T>
__device__ __forceinline__ void sat_edge(const StageArgs<T>& A, const InstanceDev& I, const BlockDev& B, int eidx, int row,
                                      int col, const EdgeGeo& geo, const double yv[4], double kv[4]) {
    const int nx = B.nx, ny = B.ny;
    const bool on[4] = {row == ny - 1, row == 0, col == nx - 1, col == 0};
    // compensated-f32 systems: division-free SAT arithmetic and vortex data (gamma = 1.4)
    constexpr bool FAST = sizeof(T) == 4;
    const double cst = A.stage == kStageK ? A.ctime : (A.stage == 0 ? 0.0 : (A.stage == 3 ? 1.0 : 0.5));
    const double stime = cst == 0.0 ? I.time : I.time + I.dt * cst;
    for (int d = 0; d < 4; ++d) {
        if (!on[d]) continue;
        double zv[4];
        const int kind = B.bc_kind[d];
        if (kind == BC_VORTEX) {
            if (FAST && A.gamma == 1.4)
                vortex_point_fast(I, stime, geo.x, geo.y, zv);
            else
                vortex_point<true>(I, A.gamma, stime, geo.x, geo.y, zv);
        } else if (kind == BC_EVAL) {
            // BoundaryCharacteristic::Eval (euler/src/lib.rs:853-863): the expressions at the stage
            // time, evaluated for this edge point by eval_kernel just before
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) zv[cc] = A.evz[4 * (int64_t)eidx + cc];
        } else if (kind == BC_INTERPOLATE || kind == BC_MULTIGRID) {
            // boundary_extract (euler/src/lib.rs:816-846): data from neighbours' opposite edges
            const bool ns_ = d == NORTH || d == SOUTH;
            const int i = ns_ ? col : row;       // position along this edge
            const int len = ns_ ? nx : ny;
            if (kind == BC_INTERPOLATE) {
                const BlockDev& Gb = A.blocks[B.bc_nb[d]];
                const T* gq = A.u_in + Gb.q_off;
                const int lg = ns_ ? Gb.nx : Gb.ny;
                const bool f2c = nx < Gb.nx;  // fine2coarse when this block's nx is smaller (:818)
                // in f64 for both state precisions (the f32 state widened), as the SAT itself
                const InterpDev<double> ip = interp_dev<double>(B.bc_aux[d], f2c);
#pragma unroll 1
                for (int cc = 0; cc < 4; ++cc) {
                    const T* plane = gq + cc * (int64_t)Gb.npad;
                    zv[cc] = interp_at<double>(ip, i, lg, len, [&](int64_t k) {
                        return absolute_state<T>(A, Gb, cc, plane[opposite_edge_point(d, (int)k, Gb.nx, Gb.ny)]);
                    });
                }
            } else {
                // Segments (g, start, end) are laid end to end, each starting on the previous
                // one's last point; the first point of every segment but the last is halved.
                const int4* sg = A.mg + B.bc_aux[d];
                const int nseg = B.bc_aux2[d];
                int p0 = 0, hit = 0, hp = 0;
                for (int k = 0; k < nseg; ++k) {
                    const int n = sg[k].z - sg[k].y;
                    if (i >= p0 && i < p0 + n) {
                        hit = k;
                        hp = p0;
                    }
                    p0 += n - 1;
                }
                const int4 seg = sg[hit];
                const BlockDev& Gb = A.blocks[seg.x];
                const T* gq = A.u_in + Gb.q_off;
                const int gp = opposite_edge_point(d, seg.y + (i - hp), Gb.nx, Gb.ny);
                const bool halve = i == hp && hit != nseg - 1;
#pragma unroll
                for (int cc = 0; cc < 4; ++cc) {
                    const double v = absolute_state<T>(A, Gb, cc, gq[cc * (int64_t)Gb.npad + gp]);
                    zv[cc] = halve ? v / 2.0 : v;
                }
            }
        } else {
            // This: own opposite edge; Grid(g): neighbour's opposite edge
            // (boundary_extracts, euler/src/lib.rs:869-930).
            const BlockDev& Gb = kind == BC_GRID ? A.blocks[B.bc_nb[d]] : B;
            const T* gq = A.u_in + Gb.q_off;
            const int gp = opposite_edge_point(d, (d == NORTH || d == SOUTH) ? col : row, Gb.nx, Gb.ny);
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) zv[cc] = absolute_state<T>(A, Gb, cc, gq[cc * (int64_t)Gb.npad + gp]);
        }
        const bool ns = d == NORTH || d == SOUTH;
        const double sign = (d == NORTH || d == EAST) ? -1.0 : 1.0;
        const double tau = (d == NORTH || d == EAST) ? 1.0 : -1.0;
        const double hi = ns ? B.hi_eta : B.hi_xi;
        const double ddx = ns ? geo.m[3] : geo.m[1];
        const double ddy = ns ? geo.m[4] : geo.m[2];
        if constexpr (FAST)
            sat_point_fast(A.gamma, yv, zv, hi, sign, tau, geo.m[0], ddx, ddy, I.v_igm1, kv);
        else
            sat_point_rows(A.gamma, yv, zv, hi, sign, tau, geo.m[0], ddx, ddy, kv);
    }
}

template <int OPX, int OPY, class T, bool UPW, bool COMP, int TY>
__global__ void __launch_bounds__(kStageThreads, 2) stage_kernel(const StageArgs<T> A) {
    using G = StageGeom<OPX, OPY, TY>;
    constexpr int R = TY / kStageWarps;
    constexpr int XA = G::XA, YA = G::YA, XP = G::XP;
    constexpr int P1B = sizeof(T) == 4 ? 4 : 2;  // phase-1 points per thread and batch
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sE = reinterpret_cast<T*>(smem_raw);       // [UPW ? 8 : 4][TY][XP]: Ehat (0..3), alpha_u q (4..7)
    T* sF = sE + (UPW ? 8 : 4) * XA;              // [UPW ? 8 : 4][HYP][32]: Fhat (0..3), alpha_v q (4..7)
    T* sR = sF + (UPW ? 8 : 4) * YA;              // [13][TY][32]: staged phase-2 operands (COMP)
    const T gamma = T(A.gamma);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned bad = 0;

    for (int t = blockIdx.x; t < A.ntiles; t += gridDim.x) {
        const int4 td = A.tiles[t];
        const BlockDev& B = A.blocks[td.x];
        const int nx = B.nx, ny = B.ny;
        const int64_t np = B.npad;
        const int y0 = td.y, x0 = td.z;
        const int th = tile_rows(td), tw = tile_cols(td);
        const int y1 = y0 + th, x1 = x0 + tw;
        int lx0, lx1, ly0, ly1;
        region_of<OPX>(x0, x1, nx, lx0, lx1);
        region_of<OPY>(y0, y1, ny, ly0, ly1);
        // Everything later phases need from the block and instance descriptors is read here,
        // once: the global stores of phase 2 would otherwise force the compiler to reload it.
        const int64_t qoff = B.q_off, eoff = B.e_off;
        const T* q = A.u_in + qoff;
        const T* mt = A.met + B.m_off;
        const InstanceDev& I = A.inst[B.instance];
        const double cb = A.stage < 4 ? I.cb[A.stage] : 0.0;
        const double ca = A.stage < 3 ? I.ca[A.stage] : 0.0;

        // ---------------- phase 1: pointwise quantities ----------------
        // Stage this thread's phase-2 operands (1 / J, RK state) into shared memory; the copies
        // run while phase 1 computes.
        if constexpr (COMP) {
            const int pr0 = y0 + warp * R, prn = min(R, y1 - pr0);
            if (lane < tw) {
                const T* src[3];
                const int nsrc = stage_operands<T>(A, src);
#pragma unroll
                for (int u = 0; u < R; ++u)
                    if (u < prn) {
                        const int ty = pr0 - y0 + u;
                        const int pt = (pr0 + u) * nx + x0 + lane;
                        T* slot = sR + ty * kTileX + lane;
                        cp_async_elem(slot, mt + pt);
                        for (int a = 0; a < nsrc; ++a)
#pragma unroll
                            for (int cc = 0; cc < 4; ++cc)
                                cp_async_elem(slot + (1 + 4 * a + cc) * TY * kTileX, src[a] + qoff + cc * np + pt);
                    }
            }
        }

        // One index space over all threads: eta-region points (rows ly0..ly1, 32 slots per row,
        // slots >= tw idle) followed by the xi-halo points (tile rows x hw columns, packed).
        // A thread takes points p = tid, tid + 256, ... in batches of P1B: all loads of a batch
        // are issued before any of its points is evaluated, so a thread waits for memory once
        // per batch rather than once per point.
        const int eh = ly1 - ly0;
        const int hl = x0 - lx0, hw = hl + (lx1 - x1);
        const int n_eta = eh * kTileX, n_all = n_eta + th * hw;
        const unsigned hw_inv = hw ? (65536u + hw - 1) / hw : 0u;  // exact floor(h / hw) for h < 1024
        for (int pb = threadIdx.x; pb < n_all; pb += P1B * kStageThreads) {
            int pt[P1B], oxi[P1B], oeta[P1B];  // point, xi slot (-1: none), eta slot (-1: none)
            T qv[P1B][4], m[P1B][4];
#pragma unroll
            for (int b = 0; b < P1B; ++b) {
                const int p = pb + b * kStageThreads;
                pt[b] = -1;
                oxi[b] = -1;
                oeta[b] = -1;
                if (p < n_eta) {
                    const int row = ly0 + (p >> 5), tx = p & 31;
                    if (tx < tw) {
                        const int col = x0 + tx;
                        pt[b] = row * nx + col;
                        oeta[b] = (row - ly0) * kTileX + tx;
                        if (row >= y0 && row < y1) oxi[b] = (row - y0) * XP + (col - lx0);
                    }
                } else if (p < n_all) {
                    const int h = p - n_eta;
                    const int ty = (int)(((unsigned)h * hw_inv) >> 16);
                    const int hc = h - ty * hw;
                    const int col = hc < hl ? lx0 + hc : x1 + (hc - hl);
                    pt[b] = (y0 + ty) * nx + col;
                    oxi[b] = ty * XP + (col - lx0);
                }
#pragma unroll
                for (int cc = 0; cc < 4; ++cc) {
                    qv[b][cc] = T(1);
                    m[b][cc] = T(0);
                }
                if (pt[b] >= 0) {
#pragma unroll
                    for (int cc = 0; cc < 4; ++cc) qv[b][cc] = __ldg(q + cc * np + pt[b]);
                    if (oxi[b] >= 0) {
                        m[b][0] = __ldg(mt + np + pt[b]);
                        m[b][1] = __ldg(mt + 2 * np + pt[b]);
                    }
                    if (oeta[b] >= 0) {
                        m[b][2] = __ldg(mt + 3 * np + pt[b]);
                        m[b][3] = __ldg(mt + 4 * np + pt[b]);
                    }
                }
            }
#pragma unroll
            for (int b = 0; b < P1B; ++b)
                if (pt[b] >= 0) {
                    if constexpr (COMP)
                        pointwise_dev<UPW>(qv[b], m[b], gamma, I.ref, sE + (oxi[b] >= 0 ? oxi[b] : 0), XA,
                                           sF + (oeta[b] >= 0 ? oeta[b] : 0), YA, oxi[b] >= 0, oeta[b] >= 0, bad);
                    else
                        pointwise<T, UPW, true>(qv[b], m[b], gamma, sE + (oxi[b] >= 0 ? oxi[b] : 0), XA,
                                                sF + (oeta[b] >= 0 ? oeta[b] : 0), YA, oxi[b] >= 0, oeta[b] >= 0,
                                                bad);
                }
        }
        if constexpr (COMP) cp_async_wait_all();
        __syncthreads();

        // ---------------- phase 2: stencils and stage update ----------------
        // Interior points finish component by component (k_c, then the RK update of c); points
        // on a block edge store k_c for the edge kernel.
        const int r0 = y0 + warp * R;  // first global row of this thread
        const int nrows = min(R, y1 - r0);
        if (lane < tw && nrows > 0) {
            const int col = x0 + lane;
            // the compensated form's f32 metrics carry the spacing factors already
            const T idxx = COMP ? T(1) : (sizeof(T) == 8 ? T(B.idx_xi) : T(B.idx_xi_f));
            const T idxy = COMP ? T(1) : (sizeof(T) == 8 ? T(B.idx_eta) : T(B.idx_eta_f));
            const bool fused = col < (sizeof(T) == 8 ? B.simd_f64 : B.simd_f32);
            const bool eta_interior = r0 >= OpShape<OPY>::M && r0 + R <= ny - OpShape<OPY>::M;
            const bool edge_col = col == 0 || col == nx - 1;
            const bool xi_closure = x0 < OpShape<OPX>::M || x1 > nx - OpShape<OPX>::M;
            const float cbf = float(cb), caf = float(ca);
            // metrics plane 0: J in f64 (the reference divides by it), 1 / J in the f32 metrics
            T jac[R];
#pragma unroll
            for (int u = 0; u < R; ++u) {
                if constexpr (COMP) jac[u] = u < nrows ? sR[(r0 - y0 + u) * kTileX + lane] : T(1);
                else jac[u] = u < nrows ? __ldg(mt + (r0 + u) * nx + col) : T(1);
            }
            T ex[4][R], dx[4][R];
            xi_rows<OPX, DIFF, T, R, !COMP, XA, XP>(sE, r0 - y0, nrows, lx0, col, nx, idxx, xi_closure, A.coef, ex);
            if constexpr (UPW)
                xi_rows<OPX, DISS, T, R, !COMP, XA, XP>(sE + 4 * XA, r0 - y0, nrows, lx0, col, nx, idxx, xi_closure,
                                                        A.coef, dx);
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) {
                T dF[R];
                eta_rows<OPY, DIFF, T, R, !COMP>(sF + cc * YA + lane, ly0, r0, nrows, ny, eta_interior, fused, idxy,
                                                 A.coef, dF);
                T ay[R];
                if constexpr (UPW)
                    eta_rows<OPY, DISS, T, R, !COMP>(sF + (4 + cc) * YA + lane, ly0, r0, nrows, ny, eta_interior,
                                                     fused, idxy, A.coef, ay);
#pragma unroll
                for (int u = 0; u < R; ++u) {
                    if (u < nrows) {
                        const int row = r0 + u;
                        T kc;
                        if constexpr (UPW) kc = -ex[cc][u] - dF[u] + dx[cc][u] + ay[u];
                        else kc = -ex[cc][u] - dF[u];
                        if constexpr (COMP) kc = kc * jac[u];
                        else kc = kc / jac[u];
                        if constexpr (COMP && UPW)
                            kc = kc + I.ref.q[cc] * __ldg(A.rinf + B.r_off + (int64_t)row * nx + col);
                        if (edge_col || row == 0 || row == ny - 1)
                            A.kedge[4 * (eoff + edge_index(row, col, nx, ny)) + cc] = kc;
                        else if constexpr (COMP)
                            rk_update_staged<T>(A, qoff + cc * np + row * nx + col, cbf, caf, kc, [&](int a) {
                                return sR[((1 + 4 * a + cc) * TY + row - y0) * kTileX + lane];
                            });
                        else
                            rk_update<T, COMP>(A, qoff + cc * np + row * nx + col, q[cc * np + row * nx + col], kc,
                                               cb, ca);
                    }
                }
            }
        }
        // Every thread is done with this tile's shared arrays before the next tile's phase 1.
        __syncthreads();
    }
    if (bad) atomicOr(A.status, bad);
}

// Edge kernel: one thread per block-edge point of a stage launch's blocks (edges[i] = block,
// row, col).  Adds the SATs to the k the stage kernel stored and does the point's RK update.
constexpr int kSatThreads = 128;
template <class T, bool COMP>
__global__ void __launch_bounds__(kSatThreads, 4) sat_kernel(const StageArgs<T> A, const int4* __restrict__ edges,
                                                          int nedges) {
    const int i = blockIdx.x * kSatThreads + threadIdx.x;
    if (i >= nedges) return;
    const int4 ed = edges[i];
    const BlockDev& B = A.blocks[ed.x];
    const InstanceDev& I = A.inst[B.instance];
    const int row = ed.y, col = ed.z;
    const int nx = B.nx, ny = B.ny;
    const int64_t np = B.npad, qoff = B.q_off;
    const int64_t slot = 4 * (B.e_off + edge_index(row, col, nx, ny));
    const double cb = A.stage < 4 ? I.cb[A.stage] : 0.0;
    const double ca = A.stage < 3 ? I.ca[A.stage] : 0.0;
    const int pt = row * nx + col;
    const T* q = A.u_in + qoff;
    double yv[4], kv[4];
    T qs[4];  // the stored stage input (a deviation in the compensated form)
#pragma unroll
    for (int cc = 0; cc < 4; ++cc) {
        qs[cc] = q[cc * np + pt];
        yv[cc] = absolute_state<T>(A, B, cc, qs[cc]);
        kv[cc] = double(A.kedge[slot + cc]);
    }
    EdgeGeo geo;
    if (sizeof(T) == 4 && A.egeo) {
        const double2* gp = reinterpret_cast<const double2*>(A.egeo + kEdgeGeo * (B.e_off + edge_index(row, col, nx, ny)));
        const double2 g0 = gp[0], g1 = gp[1], g2 = gp[2], g3 = gp[3];
        geo.x = g0.x;
        geo.y = g0.y;
        geo.m[0] = g1.x;
        geo.m[1] = g1.y;
        geo.m[2] = g2.x;
        geo.m[3] = g2.y;
        geo.m[4] = g3.x;
    } else {
        geo = edge_geo(A, B, pt);
    }
    sat_edge<T>(A, I, B, i, row, col, geo, yv, kv);
#pragma unroll
    for (int cc = 0; cc < 4; ++cc) rk_update<T, COMP>(A, qoff + cc * np + pt, qs[cc], T(kv[cc]), cb, ca);
}

// Edge geometry of a group's edge points (edges[i] = block, row, col) at their slots.
template <class T>
__global__ void edge_geo_kernel(const StageArgs<T> A, const int4* __restrict__ edges, int nedges, double* __restrict__ geo) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nedges) return;
    const int4 ed = edges[i];
    const BlockDev& B = A.blocks[ed.x];
    const EdgeGeo g = edge_geo(A, B, ed.y * B.nx + ed.z);
    double* o = geo + kEdgeGeo * (B.e_off + edge_index(ed.y, ed.z, B.nx, B.ny));
    o[0] = g.x;
    o[1] = g.y;
#pragma unroll
    for (int c = 0; c < 5; ++c) o[2 + c] = g.m[c];
    o[7] = 0.0;
}

// Expression boundary data (SBP_BC_EVAL sides) of a stage launch's edge points (edges[i] =
// block, row, col) at the stage time, into evz[4 i ..]; launched before the edge kernel only for
// systems with such sides, so the edge kernel itself stays free of the interpreter.
template <class T>
__global__ void __launch_bounds__(kSatThreads) eval_kernel(const StageArgs<T> A, const int4* __restrict__ edges,
                                                           int nedges) {
    const int i = blockIdx.x * kSatThreads + threadIdx.x;
    if (i >= nedges) return;
    const int4 ed = edges[i];
    const BlockDev& B = A.blocks[ed.x];
    const int row = ed.y, col = ed.z;
    const bool on[4] = {row == B.ny - 1, row == 0, col == B.nx - 1, col == 0};
    bool any = false;
    for (int d = 0; d < 4; ++d) any = any || (on[d] && B.bc_kind[d] == BC_EVAL);
    if (!any) return;
    const InstanceDev& I = A.inst[B.instance];
    const double cst = A.stage == kStageK ? A.ctime : (A.stage == 0 ? 0.0 : (A.stage == 3 ? 1.0 : 0.5));
    const double stime = cst == 0.0 ? I.time : I.time + I.dt * cst;
    const int64_t pt = (int64_t)row * B.nx + col;
    const double* xy = A.xy + B.x_off;
    double z[4];
    eval_state(*A.eval, A.gamma, stime, xy[pt], xy[B.npad + pt], z);
    for (int cc = 0; cc < 4; ++cc) A.evz[4 * (int64_t)i + cc] = z[cc];
}

}  // namespace sbp
