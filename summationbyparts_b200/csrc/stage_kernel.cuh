// Fused RK4 stage kernel.
//
// One launch computes, for every point of every scheduled tile, the Euler right-hand side
//   k = ((-dE/dxi - dF/deta) + diss_xi(alpha_u q) + diss_eta(alpha_v q)) / detJ
// (RHS_upwind, euler/src/lib.rs:571-616; RHS_trad 483-515 without the dissipation terms),
// adds the characteristic SATs on block edges in the order north, south, east, west
// (SAT_characteristics, euler/src/lib.rs:1002-1013), and performs this stage's share of the
// RK4 update (integrate::<Rk4>, utils/integrate/src/lib.rs:176-222):
//   stage 0: acc  = prev + (b0 dt) k ; next = prev + (a dt) k
//   stage 1: acc += (b1 dt) k        ; next = prev + (a dt) k
//   stage 2: acc += (b2 dt) k        ; next = prev + (a dt) k
//   stage 3: new  = acc + (b3 dt) k
// which is the reference's sequence fut = prev; fut += b_j dt k_j (j = 0..3) evaluated
// incrementally, so the k_j never go to memory.
//
// Work decomposition: a persistent grid walks a list of (block, y0, x0) output tiles.  For a
// tile, phase 1 evaluates the pointwise quantities once per point over the cross-shaped
// region the stencils read -- Ehat and alpha_u q on the tile rows widened by the xi halo,
// Fhat and alpha_v q on the tile columns widened by the eta halo (boundary closures widen
// the halo to the M x N block) -- into shared memory; phase 2 applies the 8 xi and 8 eta
// stencils from shared memory and finishes each point.
//
// Precision: T = double reproduces the reference's f64 arithmetic operation by operation
// (compile with -fmad=false).  T = float with COMP = true runs fluxes, dissipation and
// stencils in f32 and keeps the RK4 state as a (hi, lo) f32 pair updated with TwoSum;
// the SAT terms are computed in f64 from f64 metrics.
#pragma once

#include "euler_device.cuh"
#include "sbp_ops.cuh"

namespace sbp {

template <class T>
struct StageArgs {
    const BlockDev* __restrict__ blocks;
    const InstanceDev* __restrict__ inst;
    const int4* __restrict__ tiles;
    int ntiles;
    int stage;               // 0..3
    int TY, TX;              // tile shape
    int WX, HY;              // shared-memory capacities of the xi region width / eta region height
    const T* u_in;           // stage input state, all blocks
    const T* prev_hi;        // state at the start of the step
    const T* prev_lo;        // low part of the state (compensated precision only)
    T* acc_hi;               // RK4 accumulator
    T* acc_lo;
    T* u_out;                // next stage input (stages 0..2)
    T* new_hi;               // new state (stage 3)
    T* new_lo;
    const T* met;            // metric planes in T
    const double* met64;     // metric planes in f64 (SAT terms)
    const double* xy;        // coordinates
    double gamma;
    unsigned* status;
};

template <class T>
__device__ __forceinline__ T ldg(const T* p) {
    return __ldg(p);
}

template <int OPX, int OPY, class T, bool UPW, bool COMP>
__global__ void __launch_bounds__(256) stage_kernel(const StageArgs<T> A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);
    const int TY = A.TY, TX = A.TX, WX = A.WX, HY = A.HY;
    // xi-region arrays: 4 components x TY rows x WX columns; eta-region: 4 x HY x TX.
    T* sE = sm;
    T* sDx = sE + 4 * TY * WX;
    T* sF = UPW ? sDx + 4 * TY * WX : sDx;
    T* sDy = sF + 4 * HY * TX;
    const T gamma = T(A.gamma);
    unsigned bad = 0;

    for (int t = blockIdx.x; t < A.ntiles; t += gridDim.x) {
        const int4 td = A.tiles[t];
        const BlockDev& B = A.blocks[td.x];
        const int nx = B.nx, ny = B.ny;
        const int64_t np = B.npad;
        const int y0 = td.y, x0 = td.z;
        const int y1 = min(y0 + TY, ny), x1 = min(x0 + TX, nx);
        const int tw = x1 - x0, th = y1 - y0;
        int lx0, lx1, ly0, ly1;
        region_of<OPX>(x0, x1, nx, lx0, lx1);
        region_of<OPY>(y0, y1, ny, ly0, ly1);
        const T* q = A.u_in + B.q_off;
        const T* mt = A.met + B.m_off;

        // ---------------- phase 1: pointwise quantities ----------------
        const int eh = ly1 - ly0;
        const int hl = x0 - lx0, hr = lx1 - x1, hw = hl + hr;
        const int nEta = eh * tw, nHalo = th * hw;
        for (int p = threadIdx.x; p < nEta + nHalo; p += blockDim.x) {
            int row, col;
            bool in_eta, in_xi;
            if (p < nEta) {
                const int hy = p / tw;
                row = ly0 + hy;
                col = x0 + (p - hy * tw);
                in_eta = true;
                in_xi = row >= y0 && row < y1;
            } else {
                const int qq = p - nEta;
                const int ty = qq / hw;
                const int kk = qq - ty * hw;
                row = y0 + ty;
                col = kk < hl ? lx0 + kk : x1 + (kk - hl);
                in_eta = false;
                in_xi = true;
            }
            const int64_t pt = (int64_t)row * nx + col;
            const T rho = ldg(q + pt), rhou = ldg(q + np + pt), rhov = ldg(q + 2 * np + pt),
                    e = ldg(q + 3 * np + pt);
            // fluxes (euler/src/lib.rs:680-735)
            const T p_ = pressure<T>(gamma, rho, rhou, rhov, e);
            T E[4], F[4];
            E[0] = rhou;
            E[1] = rhou * rhou / rho + p_;
            E[2] = rhou * rhov / rho;
            E[3] = rhou * (e + p_) / rho;
            F[0] = rhov;
            F[1] = E[2];
            F[2] = rhov * rhov / rho + p_;
            F[3] = rhov * (e + p_) / rho;
            T u = T(0), v = T(0), c = T(0);
            if constexpr (UPW) {
                // upwind_dissipation (euler/src/lib.rs:619-674)
                if (!(rho > T(0))) bad |= STATUS_RHO;
                if (!(p_ > T(0))) bad |= STATUS_P;
                u = rhou / rho;
                v = rhov / rho;
                c = sqrt(gamma * p_ / rho);
            }
            if (in_xi) {
                const T jxx = ldg(mt + np + pt), jxy = ldg(mt + 2 * np + pt);
                const int si = (row - y0) * WX + (col - lx0);
#pragma unroll
                for (int cc = 0; cc < 4; ++cc) sE[cc * TY * WX + si] = jxx * E[cc] + jxy * F[cc];
                if constexpr (UPW) {
                    const T uhat = jxx * u + jxy * v;
                    const T au = fabs(uhat) + c * sqrt(jxx * jxx + jxy * jxy);
                    sDx[si] = au * rho;
                    sDx[TY * WX + si] = au * rhou;
                    sDx[2 * TY * WX + si] = au * rhov;
                    sDx[3 * TY * WX + si] = au * e;
                }
            }
            if (in_eta) {
                const T jyx = ldg(mt + 3 * np + pt), jyy = ldg(mt + 4 * np + pt);
                const int si = (row - ly0) * TX + (col - x0);
#pragma unroll
                for (int cc = 0; cc < 4; ++cc) sF[cc * HY * TX + si] = jyx * E[cc] + jyy * F[cc];
                if constexpr (UPW) {
                    const T vhat = jyx * u + jyy * v;
                    const T av = fabs(vhat) + c * sqrt(jyx * jyx + jyy * jyy);
                    sDy[si] = av * rho;
                    sDy[HY * TX + si] = av * rhou;
                    sDy[2 * HY * TX + si] = av * rhov;
                    sDy[3 * HY * TX + si] = av * e;
                }
            }
        }
        __syncthreads();

        // ---------------- phase 2: stencils, SAT, stage update ----------------
        const T idxx = sizeof(T) == 8 ? T(B.idx_xi) : T(B.idx_xi_f);
        const T idxy = sizeof(T) == 8 ? T(B.idx_eta) : T(B.idx_eta_f);
        const int simd = sizeof(T) == 8 ? B.simd_f64 : B.simd_f32;
        const InstanceDev& I = A.inst[B.instance];
        for (int o = threadIdx.x; o < th * tw; o += blockDim.x) {
            const int ty = o / tw, tx = o - ty * tw;
            const int row = y0 + ty, col = x0 + tx;
            const int64_t pt = (int64_t)row * nx + col;
            const bool fused = col < simd;
            const T detj = ldg(mt + pt);
            T k[4];
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) {
                const T* se = sE + cc * TY * WX + ty * WX - lx0;
                const T* sf = sF + cc * HY * TX + tx - ly0 * TX;
                const T dE = sum_unfused<OPX, DIFF, T>(col, nx, [&](int kk) { return se[kk]; }) * idxx;
                const T dF = sum_column<OPY, DIFF, T>(fused, row, ny, [&](int kk) { return sf[kk * TX]; }) * idxy;
                if constexpr (UPW) {
                    const T* sdx = sDx + cc * TY * WX + ty * WX - lx0;
                    const T* sdy = sDy + cc * HY * TX + tx - ly0 * TX;
                    const T ax = sum_unfused<OPX, DISS, T>(col, nx, [&](int kk) { return sdx[kk]; }) * idxx;
                    const T ay =
                        sum_column<OPY, DISS, T>(fused, row, ny, [&](int kk) { return sdy[kk * TX]; }) * idxy;
                    k[cc] = (-dE - dF + ax + ay) / detj;
                } else {
                    k[cc] = (-dE - dF) / detj;
                }
            }

            // SATs on block edges, in the reference's order N, S, E, W.
            const bool on_n = row == ny - 1, on_s = row == 0, on_e = col == nx - 1, on_w = col == 0;
            if (on_n || on_s || on_e || on_w) {
                const double* m64 = A.met64 + B.m_off;
                double yv[4], kv[4];
#pragma unroll
                for (int cc = 0; cc < 4; ++cc) {
                    yv[cc] = double(q[cc * np + pt]);
                    kv[cc] = double(k[cc]);
                }
                const double C[4] = {0.0, 0.5, 0.5, 1.0};
                const double stime = A.stage == 0 ? I.time : I.time + I.dt * C[A.stage];
#pragma unroll
                for (int d = 0; d < 4; ++d) {
                    const bool on = d == NORTH ? on_n : d == SOUTH ? on_s : d == EAST ? on_e : on_w;
                    if (!on) continue;
                    double zv[4];
                    const int kind = B.bc_kind[d];
                    if (kind == BC_VORTEX) {
                        const double* xy = A.xy + B.x_off;
                        vortex_point(I, A.gamma, stime, xy[pt], xy[np + pt], zv);
                    } else {
                        // This: own opposite edge; Grid(g): neighbour's opposite edge
                        // (boundary_extracts, euler/src/lib.rs:869-930).
                        const BlockDev& G = kind == BC_GRID ? A.blocks[B.bc_nb[d]] : B;
                        const T* gq = A.u_in + G.q_off;
                        int64_t gp;
                        if (d == NORTH) gp = col;                                          // g.south
                        else if (d == SOUTH) gp = (int64_t)(G.ny - 1) * G.nx + col;        // g.north
                        else if (d == EAST) gp = (int64_t)row * G.nx;                      // g.west
                        else gp = (int64_t)row * G.nx + (G.nx - 1);                        // g.east
#pragma unroll
                        for (int cc = 0; cc < 4; ++cc) zv[cc] = double(gq[cc * (int64_t)G.npad + gp]);
                    }
                    const bool ns = d == NORTH || d == SOUTH;
                    const double sign = (d == NORTH || d == EAST) ? -1.0 : 1.0;
                    const double tau = (d == NORTH || d == EAST) ? 1.0 : -1.0;
                    const double hi = ns ? B.hi_eta : B.hi_xi;
                    const double ddx = ns ? m64[3 * np + pt] : m64[np + pt];
                    const double ddy = ns ? m64[4 * np + pt] : m64[2 * np + pt];
                    sat_point(A.gamma, yv, zv, hi, sign, tau, m64[pt], ddx, ddy, kv);
                }
#pragma unroll
                for (int cc = 0; cc < 4; ++cc) k[cc] = T(kv[cc]);
            }

            // RK4 stage update
            const int64_t g = B.q_off + pt;
            if (!COMP) {
                const T cb = T(I.cb[A.stage]);
                if (A.stage == 0) {
                    const T ca = T(I.ca[0]);
#pragma unroll
                    for (int cc = 0; cc < 4; ++cc) {
                        const T pv = q[cc * np + pt];
                        A.acc_hi[g + cc * np] = pv + cb * k[cc];
                        A.u_out[g + cc * np] = pv + ca * k[cc];
                    }
                } else if (A.stage < 3) {
                    const T ca = T(I.ca[A.stage]);
#pragma unroll
                    for (int cc = 0; cc < 4; ++cc) {
                        const T av = A.acc_hi[g + cc * np];
                        const T pv = ldg(A.prev_hi + g + cc * np);
                        A.acc_hi[g + cc * np] = av + cb * k[cc];
                        A.u_out[g + cc * np] = pv + ca * k[cc];
                    }
                } else {
#pragma unroll
                    for (int cc = 0; cc < 4; ++cc) {
                        const T av = A.acc_hi[g + cc * np];
                        A.new_hi[g + cc * np] = av + cb * k[cc];
                    }
                }
            } else {
                const float cb = float(I.cb[A.stage]);
                if (A.stage == 0) {
                    const float ca = float(I.ca[0]);
#pragma unroll
                    for (int cc = 0; cc < 4; ++cc) {
                        float hi = float(q[cc * np + pt]);
                        float lo = float(ldg(A.prev_lo + g + cc * np));
                        const float kk = float(k[cc]);
                        A.u_out[g + cc * np] = T(hi + ca * kk);
                        comp_add(hi, lo, __fmul_rn(cb, kk));
                        A.acc_hi[g + cc * np] = T(hi);
                        A.acc_lo[g + cc * np] = T(lo);
                    }
                } else if (A.stage < 3) {
                    const float ca = float(I.ca[A.stage]);
#pragma unroll
                    for (int cc = 0; cc < 4; ++cc) {
                        float hi = float(A.acc_hi[g + cc * np]);
                        float lo = float(A.acc_lo[g + cc * np]);
                        const float kk = float(k[cc]);
                        const float pv = float(ldg(A.prev_hi + g + cc * np));
                        A.u_out[g + cc * np] = T(pv + ca * kk);
                        comp_add(hi, lo, __fmul_rn(cb, kk));
                        A.acc_hi[g + cc * np] = T(hi);
                        A.acc_lo[g + cc * np] = T(lo);
                    }
                } else {
#pragma unroll
                    for (int cc = 0; cc < 4; ++cc) {
                        float hi = float(A.acc_hi[g + cc * np]);
                        float lo = float(A.acc_lo[g + cc * np]);
                        comp_add(hi, lo, __fmul_rn(cb, float(k[cc])));
                        A.new_hi[g + cc * np] = T(hi);
                        A.new_lo[g + cc * np] = T(lo);
                    }
                }
            }
        }
        __syncthreads();
    }
    if (bad) atomicOr(A.status, bad);
}

// Shared memory bytes of one CTA.
template <class T>
inline size_t stage_smem_bytes(bool upw, int TY, int TX, int WX, int HY) {
    const size_t per = (size_t)4 * TY * WX + (size_t)4 * HY * TX;
    return sizeof(T) * per * (upw ? 2 : 1);
}

}  // namespace sbp
