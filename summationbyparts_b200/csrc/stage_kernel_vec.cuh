// Fused RK4 stage kernel, compensated-f32 form, with 2 x 2 micro-tiles and paired f32 FMAs in
// the stencil phase.
//
// Same right-hand side, same RK4 stage update and same edge-k hand-off as stage_kernel
// (stage_kernel.cuh), with every output's sums taken in the same order, so the two kernels give
// the same numbers.  What changes is the work decomposition of a 32 row x 32 column tile:
//
// * Phase 1 (pointwise fluxes and dissipation coefficients) is stage_kernel's, except where the
//   values go in shared memory: the xi arrays are stored transposed ([column][row], row pitch
//   kVecPitch = 34) with the even local columns first and the odd ones after them, the eta
//   arrays row by row (pitch 32).
// * Phase 2: thread (g, p) produces the 2 x 2 outputs of columns x0 + 2g, x0 + 2g + 1 and rows
//   y0 + 2p, y0 + 2p + 1.  An xi tap is one 8-byte shared load carrying the two rows of one
//   column (transposed layout); an eta tap one 8-byte load carrying the two columns of one row.
//   Both feed __ffma2_rn, two f32 FMAs in one instruction: per output and stencil array
//   (D + 1) / 4 loads and D / 2 paired FMAs in each direction, instead of D (xi) or
//   (R + D - 1) / R (eta) loads and D FMAs.  A half-warp (g = lane & 15, one row pair) reads
//   128 contiguous bytes of an eta row, or 16 consecutive column slots of the transposed xi
//   array -- columns 2g + k share k's parity, so the even/odd split puts them in consecutive
//   slots, and a slot pitch of 17 row pairs (odd) spreads them over all 16 bank pairs: both
//   kinds of load are conflict-free.
// * Closures: the first and the last tile of a block row hold all its closure columns (and the
//   first and last tile of a column all its closure rows; tile_starts in system.cu), and such a
//   tile first computes the closure outputs' xi (eta) terms with all its threads into a small
//   shared buffer (closure_xi, closure_eta: the N inputs of the closure block loaded once,
//   compile-time closure coefficients, first product then an fma chain as the table path of
//   stage_kernel); every thread then runs the interior path, and the owners of closure outputs
//   replace its result from the buffer -- no divergence, no per-thread coefficient tables.
// * The RK operands (1 / J and the stage's state arrays) are read from global memory into
//   registers one component ahead of their use, as 8-byte row pairs, which leaves the shared
//   memory of two 256-thread CTAs per SM to the stencil arrays.
#pragma once

#include "stage_kernel.cuh"

namespace sbp {

constexpr int kVecRows = 32;   // tile rows (256 threads = 16 column pairs x 16 row pairs)
constexpr int kVecPitch = 34;  // row pitch of the transposed xi arrays: 17 row pairs

template <int OPX, int OPY>
struct VecGeom {
    static constexpr int XC = region_extent(kTileX, OpShape<OPX>::H, OpShape<OPX>::M, OpShape<OPX>::N);
    static constexpr int HYP = region_extent(kVecRows, OpShape<OPY>::H, OpShape<OPY>::M, OpShape<OPY>::N);
    static constexpr int XCH = (XC + 1) / 2;   // column slots of each parity
    static constexpr int XA = 2 * XCH * kVecPitch;  // elements of one (transposed) xi array
    static constexpr int YA = HYP * kTileX;         // elements of one eta array
};

// Slot of local column c in a transposed xi array: even columns first, then the odd ones.
template <int XCH>
__device__ __forceinline__ int xslot(int c) { return (c >> 1) + (c & 1) * XCH; }

__device__ __forceinline__ float2 ffma2(float2 a, float c, float2 acc) { return __ffma2_rn(a, make_float2(c, c), acc); }

// Taps I..D of two adjacent outputs of one stencil: ld(i) is the input pair at tap position i of
// the first output (D + 1 positions for the two); output 0 takes coefficient i at position i,
// output 1 coefficient i - 1.  Unrolled at compile time so every coefficient is a constant and
// zero coefficients cost nothing.
template <int OP, int KIND, int I, int D>
struct PairTaps {
    template <class LD>
    __device__ __forceinline__ static void run(const LD& ld, float2& a0, float2& a1) {
        if constexpr (I <= D) {
            const float2 v = ld(I);
            if constexpr (I < D) {
                constexpr float c = CDiag<OP, KIND>::v[I];
                if constexpr (c != 0.0f) a0 = ffma2(v, c, a0);
            }
            if constexpr (I >= 1) {
                constexpr float c = CDiag<OP, KIND>::v[I - 1];
                if constexpr (c != 0.0f) a1 = ffma2(v, c, a1);
            }
            PairTaps<OP, KIND, I + 1, D>::run(ld, a0, a1);
        }
    }
};

// Xi sums of one kind at columns c0, c0 + 1, each over the thread's two rows.  Local column
// c0 - H + i of the transposed array, row r0, is at (i even ? pe : po) + (i / 2) * kVecPitch
// (pe, po: the slots of columns c0 - H and c0 - H + 1; 8-byte aligned).  Interior columns: the
// fma chain of stage_kernel's interior path (its zero taps skipped).
template <int OP, int KIND>
__device__ __forceinline__ void xi_pair(const float* __restrict__ pe, const float* __restrict__ po, float2 out[2]) {
    constexpr int D = OpShape<OP>::D;
    float2 a0 = make_float2(0.0f, 0.0f), a1 = make_float2(0.0f, 0.0f);
    PairTaps<OP, KIND, 0, D>::run(
        [&](int i) { return *reinterpret_cast<const float2*>((i & 1 ? po : pe) + (i >> 1) * kVecPitch); }, a0, a1);
    out[0] = a0;
    out[1] = a1;
}

// Eta sums of one kind at rows r0, r0 + 1, each over the thread's two columns: p points at the
// eta array's row r0 - H, column c0 (8-byte aligned).
template <int OP, int KIND>
__device__ __forceinline__ void eta_pair(const float* __restrict__ p, float2 out[2]) {
    constexpr int D = OpShape<OP>::D;
    float2 a0 = make_float2(0.0f, 0.0f), a1 = make_float2(0.0f, 0.0f);
    PairTaps<OP, KIND, 0, D>::run([&](int i) { return *reinterpret_cast<const float2*>(p + i * kTileX); }, a0, a1);
    out[0] = a0;
    out[1] = a1;
}

// Closure terms of a tile: xi ([component][closure column][row], row pitch 34, closure_xi) and
// eta ([component][closure row][column], closure_eta), one buffer each.
constexpr int kClosurePitch = 34;
__host__ __device__ constexpr int closure_xi_elems(int mx) { return 4 * mx * kClosurePitch; }
__host__ __device__ constexpr int closure_eta_elems(int my) { return 4 * my * kTileX; }

template <int OPX, int OPY>
constexpr size_t vec_stage_smem(bool upw) {
    using G = VecGeom<OPX, OPY>;
    return sizeof(float) * ((size_t)(4 * G::XA + 4 * G::YA) * (upw ? 2 : 1) + closure_xi_elems(OpShape<OPX>::M) +
                            closure_eta_elems(OpShape<OPY>::M));
}

// Closure-block coefficient (row I, input K) of one end of a line: the start block, or the end
// block (row I applies -/+ st[(M - 1 - I) N + (N - 1 - K)], DIFF negated).
template <int OP, int KIND, bool RIGHT, int I, int K>
struct ClosureCoef {
    static constexpr int M = OpShape<OP>::M, N = OpShape<OP>::N;
    static constexpr float value = RIGHT ? (KIND == DIFF ? -1.0f : 1.0f) * CDiag<OP, KIND>::st[(M - 1 - I) * N + (N - 1 - K)]
                                         : CDiag<OP, KIND>::st[I * N + K];
};
// Rows I.. of the closure block: the sum over the N inputs v, first product then an fma chain
// (the table path's order).
template <int OP, int KIND, bool RIGHT, int I, int K = 1>
__device__ __forceinline__ float closure_sum(const float* v, float t) {
    if constexpr (K == 1) t = v[0] * ClosureCoef<OP, KIND, RIGHT, I, 0>::value;
    if constexpr (K < OpShape<OP>::N) {
        constexpr float c = ClosureCoef<OP, KIND, RIGHT, I, K>::value;
        return closure_sum<OP, KIND, RIGHT, I, K + 1>(v, __fmaf_rn(v[K], c, t));
    } else {
        return t;
    }
}

// Writes closure columns I .. I + CNT - 1 of closure_xi.
template <int OP, bool UPW, bool RIGHT, int I, int CNT, int PITCH = kClosurePitch>
__device__ __forceinline__ void closure_out(const float* ve, const float* va, float* cb) {
    if constexpr (CNT > 0) {
        float d = 0.0f;
        if constexpr (UPW) d = closure_sum<OP, DISS, RIGHT, I>(va, 0.0f);
        cb[I * PITCH] = d - closure_sum<OP, DIFF, RIGHT, I>(ve, 0.0f);
        closure_out<OP, UPW, RIGHT, I + 1, CNT - 1, PITCH>(ve, va, cb);
    }
}

// The xi term diss_xi(alpha_u q) - diff_xi(Ehat) of closure columns I0 .. I0 + CNT - 1 at one end
// of a line, for one component and tile row: e / a are the transposed Ehat / alpha_u q arrays at
// the row, `lc` the local column of the block's first input (the inputs carry the spacing
// factor through the metrics), into cb[i * kClosurePitch].
template <int OP, bool UPW, bool RIGHT, int XCH, int I0, int CNT>
__device__ __forceinline__ void closure_xi(const float* __restrict__ e, const float* __restrict__ a, int lc,
                                           float* __restrict__ cb) {
    constexpr int N = OpShape<OP>::N;
    const int se = xslot<XCH>(lc) * kVecPitch, so = xslot<XCH>(lc + 1) * kVecPitch;
    float ve[N], va[N];
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const int o = (k & 1 ? so : se) + (k >> 1) * kVecPitch;
        ve[k] = e[o];
        va[k] = UPW ? a[o] : 0.0f;
    }
    closure_out<OP, UPW, RIGHT, I0, CNT>(ve, va, cb);
}

// The eta term diss_eta(alpha_v q) - diff_eta(Fhat) of closure rows I0 .. I0 + CNT - 1 at one
// end of a column (BOTTOM = false: rows 0 .. M - 1, true: n - M .. n - 1), for one component and
// tile column: f / a are the Fhat / alpha_v q arrays at the column, `lr` the local row of the
// block's first input, into cb[i * kTileX].
template <int OP, bool UPW, bool BOTTOM, int I0, int CNT>
__device__ __forceinline__ void closure_eta(const float* __restrict__ f, const float* __restrict__ a, int lr,
                                            float* __restrict__ cb) {
    constexpr int N = OpShape<OP>::N;
    float ve[N], va[N];
#pragma unroll
    for (int k = 0; k < N; ++k) {
        ve[k] = f[(lr + k) * kTileX];
        va[k] = UPW ? a[(lr + k) * kTileX] : 0.0f;
    }
    closure_out<OP, UPW, BOTTOM, I0, CNT, kTileX>(ve, va, cb);
}

// The two values of a thread's row u at columns c0, c0 + 1 from `p` (the element of (r0, c0)).
// Row r0 starts at an even element (r0 and c0 are even, planes start 256-byte aligned), so its
// pair is one 8-byte load, which stays inside the plane's padded extent even where c0 + 1 is past
// the row (the second value is then not used); row r0 + 1 is one 8-byte load for even nx, else
// two loads.
__device__ __forceinline__ float2 ld_row_pair(const float* __restrict__ p, int u, int nx, bool ok1, bool cok1, float def) {
    if (u == 0) return __ldg(reinterpret_cast<const float2*>(p));
    if (!ok1) return make_float2(def, def);
    if ((nx & 1) == 0) return __ldg(reinterpret_cast<const float2*>(p + nx));
    return make_float2(__ldg(p + nx), cok1 ? __ldg(p + nx + 1) : def);
}

// Stage class of the RK update: 0 = stage 0, 1 = stages 1 and 2, 2 = stage 3.  The micro-tile
// kernel takes it as a template parameter, so the operand arrays it reads and the update it
// writes are fixed at compile time (the k-only stage of other tableaus runs on f64 systems only).
__host__ __device__ constexpr int vec_stage_class(int stage) { return stage == 0 ? 0 : (stage < 3 ? 1 : 2); }

template <int OPX, int OPY, bool UPW, int SC>
__global__ void __launch_bounds__(kStageThreads, 2) stage_kernel_vec(const StageArgs<float> A) {
    static_assert(SC >= 0 && SC <= 2, "stage class");
    using G = VecGeom<OPX, OPY>;
    constexpr int XA = G::XA, YA = G::YA, XCH = G::XCH;
    constexpr int HX = OpShape<OPX>::H, HY = OpShape<OPY>::H;
    // phase-1 points per thread and batch: enough for an interior tile's whole region
    // ((32 + 2 H_eta) rows x 32 + 32 rows x 2 H_xi points) in one batch of loads
    constexpr int P1B = ((kVecRows + 2 * HY) * kTileX + kVecRows * 2 * HX + kStageThreads - 1) / kStageThreads;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* sE = reinterpret_cast<float*>(smem_raw);  // [UPW ? 8 : 4][2 XCH][34]: Ehat, alpha_u q (transposed)
    float* sF = sE + (UPW ? 8 : 4) * XA;             // [UPW ? 8 : 4][HYP][32]: Fhat, alpha_v q
    float* cbuf = sF + (UPW ? 8 : 4) * YA;           // [4][M_xi][34]: closure-column xi terms
    float* cbuf_y = cbuf + closure_xi_elems(OpShape<OPX>::M);  // [4][M_eta][32]: closure-row eta terms
    const float gamma = float(A.gamma);
    const int tid = threadIdx.x;
    const int grp = tid & 15, rpr = tid >> 4;  // column pair, row pair (0..15 each)
    unsigned bad = 0;
    if (A.stage == kStageK || vec_stage_class(A.stage) != SC) {  // launched for another stage class
        if (tid == 0) atomicOr(A.status, STATUS_BAD_LAUNCH);
        return;
    }
    // RK operand arrays (stage_operands): stage 0 u_in; stages 1, 2 acc_hi, prev_hi; stage 3 also prev_lo
    constexpr int NSRC = SC + 1;
    const float* src[3] = {SC == 0 ? A.u_in : A.acc_hi, A.prev_hi, A.prev_lo};

    for (int t = blockIdx.x; t < A.ntiles; t += gridDim.x) {
        const int4 td = A.tiles[t];
        const BlockDev& B = A.blocks[td.x];
        const int nx = B.nx, ny = B.ny;
        const int np = (int)B.npad;  // in-block offsets fit 32 bits (checked when the system is built)
        const int y0 = td.y, x0 = td.z;
        const int th = tile_rows(td), tw = tile_cols(td);
        const int y1 = y0 + th, x1 = x0 + tw;
        int lx0, lx1, ly0, ly1;
        region_of<OPX>(x0, x1, nx, lx0, lx1);
        region_of<OPY>(y0, y1, ny, ly0, ly1);
        const int64_t qoff = B.q_off, eoff = B.e_off;
        const float* q = A.u_in + qoff;
        const float* mt = A.met + B.m_off;
        const InstanceDev& I = A.inst[B.instance];
        const float cbf = float(A.stage < 4 ? I.cb[A.stage] : 0.0);
        const float caf = float(A.stage < 3 ? I.ca[A.stage] : 0.0);

        // ---------------- phase 1: pointwise quantities ----------------
        // One index space over all threads: eta-region points (local rows 0 .. eh - 1, 32 slots per
        // row, slots >= tw idle) followed by the xi-halo points (tile rows x hw columns, packed).
        // A thread takes points p = tid, tid + 256, ... in batches of P1B, all loads of a batch
        // issued before any of its points is evaluated.
        const int eh = ly1 - ly0;
        const int hl = x0 - lx0, hw = hl + (lx1 - x1);
        const int n_eta = eh * kTileX, n_all = n_eta + th * hw;
        const unsigned hw_inv = hw ? (65536u + hw - 1) / hw : 0u;  // exact floor(h / hw) for h < 1024
        for (int pb = tid; pb < n_all; pb += P1B * kStageThreads) {
            int pt[P1B], oxi[P1B], oeta[P1B];
            float qv[P1B][4], m[P1B][4];
#pragma unroll
            for (int b = 0; b < P1B; ++b) {
                const int p = pb + b * kStageThreads;
                pt[b] = -1;
                oxi[b] = -1;
                oeta[b] = -1;
                if (p < n_eta) {
                    const int lr = p >> 5, tx = p & 31, row = ly0 + lr;
                    if (tx < tw) {
                        const int col = x0 + tx;
                        pt[b] = row * nx + col;
                        oeta[b] = lr * kTileX + tx;
                        if (row >= y0 && row < y1) oxi[b] = xslot<XCH>(col - lx0) * kVecPitch + (row - y0);
                    }
                } else if (p < n_all) {
                    const int h = p - n_eta;
                    const int ty = (int)(((unsigned)h * hw_inv) >> 16);
                    const int hc = h - ty * hw;
                    const int col = hc < hl ? lx0 + hc : x1 + (hc - hl);
                    pt[b] = (y0 + ty) * nx + col;
                    oxi[b] = xslot<XCH>(col - lx0) * kVecPitch + ty;
                }
#pragma unroll
                for (int cc = 0; cc < 4; ++cc) {
                    qv[b][cc] = 1.0f;
                    m[b][cc] = 0.0f;
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
                if (pt[b] >= 0)
                    pointwise_dev<UPW>(qv[b], m[b], gamma, I.ref, sE + (oxi[b] >= 0 ? oxi[b] : 0), XA,
                                       sF + (oeta[b] >= 0 ? oeta[b] : 0), YA, oxi[b] >= 0, oeta[b] >= 0, bad);
        }

        // Phase-2 operands of this thread (1 / J and component 0's RK operands), loaded before
        // the barrier so the loads overlap the other warps' phase 1.  Element of point (u, j)
        // of component cc: in-block offset e0 + cc * np + u * nx + j from the block bases.
        const int c0 = x0 + 2 * grp, r0 = y0 + 2 * rpr;
        const bool cok[2] = {2 * grp < tw, 2 * grp + 1 < tw};
        const bool rok[2] = {2 * rpr < th, 2 * rpr + 1 < th};
        const bool active = cok[0] && rok[0];
        const int e0 = r0 * nx + c0;
        const float* srcb[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) srcb[a] = a < NSRC ? src[a] + qoff : nullptr;
        float jinv[2][2], rinf[2][2], opn[3][2][2];  // jinv: plane 0 of the f32 metrics, 1 / J
        const float* rb = UPW ? A.rinf + B.r_off : nullptr;
        if (active) {
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const float2 jv = ld_row_pair(mt + e0, u, nx, rok[1], cok[1], 1.0f);
                jinv[u][0] = jv.x;
                jinv[u][1] = jv.y;
                if constexpr (UPW) {
                    const float2 rv = ld_row_pair(rb + e0, u, nx, rok[1], cok[1], 0.0f);
                    rinf[u][0] = rv.x;
                    rinf[u][1] = rv.y;
                } else {
                    rinf[u][0] = rinf[u][1] = 0.0f;
                }
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    const float2 ov = a < NSRC ? ld_row_pair(srcb[a] + e0, u, nx, rok[1], cok[1], 0.0f) : make_float2(0.0f, 0.0f);
                    opn[a][u][0] = ov.x;
                    opn[a][u][1] = ov.y;
                }
            }
        }
        __syncthreads();

        // Closure outputs.  The tile list gives every closure column of a block row to its first
        // or its last tile and no tile both (tile_starts), and likewise for rows.  A tile holding
        // closure columns first writes their xi terms (diss - diff, scaled) for every row and
        // component into cbuf, a tile holding closure rows their eta terms into cbuf_y (all
        // threads, one barrier for both); in phase 2 every thread runs the interior path and the
        // threads owning closure outputs replace its result from the buffers.
        const bool left_cl = x0 < OpShape<OPX>::M, right_cl = x1 > nx - OpShape<OPX>::M;
        const bool top_cl = y0 < OpShape<OPY>::M, bot_cl = y1 > ny - OpShape<OPY>::M;
        if ((left_cl && right_cl) || (top_cl && bot_cl)) {  // a tile list not made by tile_starts
            if (tid == 0) atomicOr(A.status, STATUS_BAD_LAUNCH);
            return;
        }
        const bool xi_pre = left_cl || right_cl, eta_pre = top_cl || bot_cl;
        if (xi_pre) {
            // thread: component tid / 64, tile row (tid / 2) % 32, half tid % 2 of the M columns
            constexpr int MX = OpShape<OPX>::M;
            const int comp = tid >> 6, r = (tid >> 1) & 31, half = tid & 1;
            if (r < th) {
                const int lc = right_cl ? nx - OpShape<OPX>::N - lx0 : -lx0;
                const float* e = sE + comp * XA + r;
                const float* al = sE + (UPW ? 4 + comp : comp) * XA + r;
                float* cb = cbuf + comp * MX * kClosurePitch + r;
                if (right_cl) {
                    if (half) closure_xi<OPX, UPW, true, XCH, MX / 2, MX / 2>(e, al, lc, cb);
                    else closure_xi<OPX, UPW, true, XCH, 0, MX / 2>(e, al, lc, cb);
                } else {
                    if (half) closure_xi<OPX, UPW, false, XCH, MX / 2, MX / 2>(e, al, lc, cb);
                    else closure_xi<OPX, UPW, false, XCH, 0, MX / 2>(e, al, lc, cb);
                }
            }
        }
        if (eta_pre) {
            // thread: component tid / 64, half (tid / 32) % 2 of the M rows, tile column tid % 32
            constexpr int MY = OpShape<OPY>::M;
            const int comp = tid >> 6, half = (tid >> 5) & 1, col = tid & 31;
            if (col < tw) {
                const int lr = bot_cl ? ny - OpShape<OPY>::N - ly0 : -ly0;
                const float* f = sF + comp * YA + col;
                const float* al = sF + (UPW ? 4 + comp : comp) * YA + col;
                float* cb = cbuf_y + comp * MY * kTileX + col;
                if (bot_cl) {
                    if (half) closure_eta<OPY, UPW, true, MY / 2, MY / 2>(f, al, lr, cb);
                    else closure_eta<OPY, UPW, true, 0, MY / 2>(f, al, lr, cb);
                } else {
                    if (half) closure_eta<OPY, UPW, false, MY / 2, MY / 2>(f, al, lr, cb);
                    else closure_eta<OPY, UPW, false, 0, MY / 2>(f, al, lr, cb);
                }
            }
        }
        if (xi_pre || eta_pre) __syncthreads();

        // ---------------- phase 2: stencils and stage update ----------------
        if (active) {
            const float* xrow = sE + (r0 - y0);                                  // xi arrays at row r0
            // interior-path window from column c0 - H (kept inside the arrays for closure columns,
            // whose interior-path sums are replaced)
            const int cw = min(max(c0 - HX - lx0, 0), G::XC - OpShape<OPX>::D - 1);
            const float* xwe = xrow + xslot<XCH>(cw) * kVecPitch;      // xi arrays at column c0 - H
            const float* xwo = xrow + xslot<XCH>(cw + 1) * kVecPitch;  // ... column c0 - H + 1
            const float* ecol = sF + (c0 - x0);                        // eta arrays at local row 0, column c0
            // interior-path window from row r0 - H (kept inside the arrays for closure rows, whose
            // interior-path sums are replaced)
            const float* ewin = ecol + min(max(r0 - HY - ly0, 0), G::HYP - OpShape<OPY>::D - 1) * kTileX;
            bool edge[2][2];
#pragma unroll
            for (int u = 0; u < 2; ++u)
#pragma unroll
                for (int j = 0; j < 2; ++j)
                    edge[u][j] = r0 + u == 0 || r0 + u == ny - 1 || c0 + j == 0 || c0 + j == nx - 1;
            // outputs: stage 3 the new (hi, lo) state, otherwise the next stage input and the increment
            // per-array pointers at point (r0, c0) of component cc, advanced by one plane per
            // component: the four points are at offsets 0, 1, nx, nx + 1
            float* out1 = (SC == 2 ? A.new_hi : A.u_out) + qoff + e0;
            float* out2 = (SC == 2 ? A.new_lo : A.acc_hi) + qoff + e0;
            const float* ps[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) ps[a] = a < NSRC ? srcb[a] + e0 : nullptr;
            float* kq = A.kedge + 4 * eoff;
#pragma unroll 1
            for (int cc = 0; cc < 4; ++cc) {
                const float qr = I.ref.q[cc];  // reference state (free-stream dissipation term)
                float nxt[3][2][2];
                if (cc < 3) {
#pragma unroll
                    for (int u = 0; u < 2; ++u)
#pragma unroll
                        for (int a = 0; a < 3; ++a) {
                            const float2 v = a < NSRC ? ld_row_pair(ps[a] + np, u, nx, rok[1], cok[1], 0.0f) : make_float2(0.0f, 0.0f);
                            nxt[a][u][0] = v.x;
                            nxt[a][u][1] = v.y;
                        }
                }
                // xi sums: ex[j] / dx[j] = column c0 + j over rows (r0, r0 + 1)
                float2 ex[2], dx[2] = {make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f)};
                float2 ey[2], ay[2] = {make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f)};
                xi_pair<OPX, DIFF>(xwe + cc * XA, xwo + cc * XA, ex);
                if constexpr (UPW) xi_pair<OPX, DISS>(xwe + (4 + cc) * XA, xwo + (4 + cc) * XA, dx);
                // eta sums: ey[u] / ay[u] = row r0 + u over columns (c0, c0 + 1)
                eta_pair<OPY, DIFF>(ewin + cc * YA, ey);
                if constexpr (UPW) eta_pair<OPY, DISS>(ewin + (4 + cc) * YA, ay);
                if (xi_pre) {
#pragma unroll
                    for (int j = 0; j < 2; ++j) {
                        const int ci = left_cl ? c0 + j : c0 + j - (nx - OpShape<OPX>::M);
                        if (ci >= 0 && ci < OpShape<OPX>::M && cok[j]) {
                            // the whole xi term as -ex: (-ex - ey + dx) + ay with dx = 0
                            const float2 t = *reinterpret_cast<const float2*>(
                                cbuf + (cc * OpShape<OPX>::M + ci) * kClosurePitch + (r0 - y0));
                            ex[j] = make_float2(-t.x, -t.y);
                            dx[j] = make_float2(0.0f, 0.0f);
                        }
                    }
                }
                if (eta_pre) {
#pragma unroll
                    for (int u = 0; u < 2; ++u) {
                        const int ri = top_cl ? r0 + u : r0 + u - (ny - OpShape<OPY>::M);
                        if (ri >= 0 && ri < OpShape<OPY>::M && rok[u]) {
                            const float2 t = *reinterpret_cast<const float2*>(
                                cbuf_y + (cc * OpShape<OPY>::M + ri) * kTileX + (c0 - x0));
                            ey[u] = make_float2(-t.x, -t.y);
                            ay[u] = make_float2(0.0f, 0.0f);
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    if (!rok[u]) continue;
                    float v1[2], v2[2];
                    bool st[2];
#pragma unroll
                    for (int j = 0; j < 2; ++j) {
                        const float exv = u == 0 ? ex[j].x : ex[j].y, dxv = u == 0 ? dx[j].x : dx[j].y;
                        const float eyv = j == 0 ? ey[u].x : ey[u].y, ayv = j == 0 ? ay[u].x : ay[u].y;
                        float kc;
                        if constexpr (UPW) kc = (-exv - eyv + dxv + ayv) * jinv[u][j] + qr * rinf[u][j];
                        else kc = (-exv - eyv) * jinv[u][j];
                        st[j] = cok[j] && !edge[u][j];
                        if (cok[j] && edge[u][j]) kq[4 * edge_index(r0 + u, c0 + j, nx, ny) + cc] = kc;
                        if constexpr (SC == 0) {
                            v1[j] = opn[0][u][j] + caf * kc;
                            v2[j] = cbf * kc;
                        } else if constexpr (SC == 1) {
                            v1[j] = opn[1][u][j] + caf * kc;
                            v2[j] = opn[0][u][j] + cbf * kc;
                        } else {
                            float hi = opn[1][u][j], lo = opn[2][u][j];
                            comp_add(hi, lo, opn[0][u][j] + cbf * kc);
                            v1[j] = hi;
                            v2[j] = lo;
                        }
                    }
                    // one 8-byte store per output array where both points are written and the
                    // row's pair is 8-byte aligned (see ld_row_pair), else one store per point
                    float* p1 = out1 + u * nx;
                    float* p2 = out2 + u * nx;
                    if (st[0] && st[1] && (u == 0 || (nx & 1) == 0)) {
                        *reinterpret_cast<float2*>(p1) = make_float2(v1[0], v1[1]);
                        *reinterpret_cast<float2*>(p2) = make_float2(v2[0], v2[1]);
                    } else {
#pragma unroll
                        for (int j = 0; j < 2; ++j)
                            if (st[j]) {
                                p1[j] = v1[j];
                                p2[j] = v2[j];
                            }
                    }
                }
#pragma unroll
                for (int a = 0; a < NSRC; ++a) ps[a] += np;
                out1 += np;
                out2 += np;
                if (cc < 3) {
#pragma unroll
                    for (int a = 0; a < NSRC; ++a)
#pragma unroll
                        for (int u = 0; u < 2; ++u)
#pragma unroll
                            for (int j = 0; j < 2; ++j) opn[a][u][j] = nxt[a][u][j];
                }
            }
        }
        // Every thread is done with this tile's shared arrays before the next tile's phase 1.
        __syncthreads();
    }
    if (bad) atomicOr(A.status, bad);
}

// Entry of the micro-tile kernel for stage class sc (vec_stage_class), for cudaLaunchKernel.
template <int OPX, int OPY, bool UPW>
const void* vec_entry(int sc) {
    if (sc == 0) return reinterpret_cast<const void*>(&stage_kernel_vec<OPX, OPY, UPW, 0>);
    if (sc == 1) return reinterpret_cast<const void*>(&stage_kernel_vec<OPX, OPY, UPW, 1>);
    return reinterpret_cast<const void*>(&stage_kernel_vec<OPX, OPY, UPW, 2>);
}

}  // namespace sbp
