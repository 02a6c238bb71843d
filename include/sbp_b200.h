/*
 * sbp_b200 -- B200-native (sm_100a) SBP-SAT Euler time stepping, C ABI.
 *
 * This is the drop-in boundary for the reference's hot path (mulimoen/
 * SummationByParts): the SbpOperator2d / UpwindOperator2d stencils, the Euler
 * right-hand side with its SATs, and the RK4 stage update, plus the
 * euler::System / multigrid::System driver surface that calls them.  The
 * reference has no FFI of its own; each entry point below names the Rust item
 * it replaces.  A Rust -sys crate binds exactly these symbols, with the same
 * struct layouts.
 *
 * Conventions
 *  - Every function returns sbp_status (0 = SBP_OK) unless noted; on error a
 *    message is available from sbp_last_error() (thread-local).  Nothing in
 *    the library aborts or exits.
 *  - Fields are C-order (4, ny, nx) arrays of (rho, rhou, rhov, e), the
 *    reference's euler::Field layout (euler/src/lib.rs:190-219).  2-D arrays
 *    are (ny, nx) with x (xi) contiguous.
 *  - Pointers named d_* are device pointers; others are host pointers.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *  - Directions are indexed SBP_NORTH, SBP_SOUTH, SBP_EAST, SBP_WEST.
 */
#ifndef SBP_B200_H
#define SBP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum sbp_status {
    SBP_OK = 0,
    SBP_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad enum, bad index */
    SBP_ERR_SHAPE = 2,            /* n < max(2M, N), mismatched interface lengths, ... */
    SBP_ERR_UNSUPPORTED = 3,      /* combination not built (e.g. dissipation of SBP4) */
    SBP_ERR_CUDA = 4,             /* a CUDA runtime call failed */
    SBP_ERR_NONPHYSICAL = 5,      /* rho <= 0, p <= 0, detJ <= 0 or NaN detected on device */
    SBP_ERR_NO_DEVICE = 6,
    SBP_ERR_OUT_OF_MEMORY = 7
} sbp_status;

/* The six operators of sbp/src/operators.rs:152-165. */
typedef enum sbp_operator {
    SBP_OP_UPWIND4 = 0,
    SBP_OP_UPWIND4H2 = 1,
    SBP_OP_UPWIND9 = 2,
    SBP_OP_UPWIND9H2 = 3,
    SBP_OP_SBP4 = 4,
    SBP_OP_SBP8 = 5
} sbp_operator;

typedef enum sbp_dtype { SBP_F64 = 0, SBP_F32 = 1 } sbp_dtype;

/* SBP_PRECISION_F64: the reference's f64 arithmetic, operation for operation.
 * SBP_PRECISION_F32_COMPENSATED: stencils, fluxes and dissipation in f32 on deviations from each
 * instance's free stream (so f32 rounding is relative to the deviation, not to the state), the
 * RK4 state kept as that deviation in a compensated (hi, lo) f32 pair; metrics built in f64,
 * the free-stream dissipation term, SAT terms and norms in f64.  Every state entry point below
 * takes and returns the absolute state. */
typedef enum sbp_precision { SBP_PRECISION_F64 = 0, SBP_PRECISION_F32_COMPENSATED = 1 } sbp_precision;

/* euler::BoundaryCharacteristic (euler/src/lib.rs:737-745): This, Grid(neighbour), Vortex,
 * Interpolate(neighbour, operator) (a 2:1 interface) and MultiGrid(segments). */
typedef enum sbp_boundary_kind {
    SBP_BC_THIS = 0,
    SBP_BC_GRID = 1,
    SBP_BC_VORTEX = 2,
    SBP_BC_INTERPOLATE = 3,
    SBP_BC_MULTIGRID = 4,
    SBP_BC_EVAL = 5
} sbp_boundary_kind;

/* sbp::operators::{Interpolation4, Interpolation8, Interpolation9, Interpolation9h2}
 * (sbp/src/operators/interpolation/interpolation{4,8,9,9h2}.rs).  Fine lines have 2 n - 1 points for a coarse line of
 * n points (2 (n - 1) for Interpolation9h2). */
typedef enum sbp_interpolation {
    SBP_INTERP4 = 0,
    SBP_INTERP8 = 1,
    SBP_INTERP9 = 2,
    SBP_INTERP9H2 = 3
} sbp_interpolation;

enum { SBP_NORTH = 0, SBP_SOUTH = 1, SBP_EAST = 2, SBP_WEST = 3 };

/* euler::VortexParameters (euler/src/vortex.rs:4-21): up to 5 superposed vortices. */
typedef struct sbp_vortex_params {
    int nvortices;
    double x0[5], y0[5], rstar[5], eps[5];
    double mach;
} sbp_vortex_params;

/* One curvilinear block: its grid (sbp::grid::Grid, sbp/src/grid.rs:9-35), its operator pair
 * (the (eta, xi) tuple of sbp/src/operators.rs:115-150), its four boundary kinds and the
 * independent solve ("instance") it belongs to.  Blocks of one instance share dt, time and
 * vortex parameters; instances are independent (an ensemble). */
typedef struct sbp_block_desc {
    int64_t nx, ny;
    int op_xi, op_eta;    /* sbp_operator */
    const double* x;      /* host, (ny, nx) */
    const double* y;      /* host, (ny, nx) */
    int bc_kind[4];       /* sbp_boundary_kind per direction */
    int bc_neighbour[4];  /* block index for SBP_BC_GRID and SBP_BC_INTERPOLATE */
    int instance;         /* 0 .. ninstances-1 */
    int bc_interp_op[4];  /* SBP_BC_INTERPOLATE: sbp_interpolation; fine2coarse when this block's
                             nx is smaller than the neighbour's (euler/src/lib.rs:818) */
    int bc_multigrid_count[4];   /* SBP_BC_MULTIGRID: number of segments */
    const int* bc_multigrid[4];  /* SBP_BC_MULTIGRID: (block, start, end) per segment, host
                                    memory read at creation (euler/src/lib.rs:829-846) */
} sbp_block_desc;

typedef struct sbp_system sbp_system;

/* ---- library ------------------------------------------------------------ */

/* Message of the last failed call on this thread ("" if none). */
const char* sbp_last_error(void);
/* Library version string. */
const char* sbp_version(void);

/* ---- operators: SbpOperator1d / SbpOperator2d / UpwindOperator2d -------- */

/* SbpOperator1d::h (sbp/src/operators.rs:15-16): writes the M boundary weights of H into h
 * (capacity cap) and returns M, or -1 for a bad operator. */
int sbp_operator_h(int op, double* h, int cap);
/* SbpOperator1d::is_h2 (sbp/src/operators.rs:17-20): 1, 0, or -1 for a bad operator. */
int sbp_operator_is_h2(int op);
/* SbpOperator2d::upwind().is_some() (sbp/src/operators.rs:85-87): 1, 0, or -1. */
int sbp_operator_is_upwind(int op);
/* Coefficients as built into the kernels, for verification against the reference tables:
 * kind 0 = first derivative (DIFF), 1 = dissipation (DISS); part 0 = start block (M*N),
 * 1 = interior diagonal (D), 2 = end block (M*N).  Returns the count written, or -1. */
int sbp_operator_table(int op, int kind, int part, double* out, int cap);

/* SbpOperator2d::diffxi (sbp/src/operators.rs:56-61; algos.rs:101-187 row path):
 * for each of nbatch (ny, nx) arrays spaced batch_stride elements apart, differentiate along x.
 * Results are bit-identical to the reference's row path in the same dtype. */
sbp_status sbp_diffxi(int op, int dtype, const void* d_prev, void* d_fut, int64_t ny, int64_t nx,
                      int64_t nbatch, int64_t batch_stride, void* stream);
/* SbpOperator2d::diffeta (sbp/src/operators.rs:62-64; algos.rs:371-519 column path). */
sbp_status sbp_diffeta(int op, int dtype, const void* d_prev, void* d_fut, int64_t ny, int64_t nx,
                       int64_t nbatch, int64_t batch_stride, void* stream);
/* UpwindOperator2d::dissxi (sbp/src/operators.rs:91-96). */
sbp_status sbp_dissxi(int op, int dtype, const void* d_prev, void* d_fut, int64_t ny, int64_t nx,
                      int64_t nbatch, int64_t batch_stride, void* stream);
/* UpwindOperator2d::disseta (sbp/src/operators.rs:98-100). */
sbp_status sbp_disseta(int op, int dtype, const void* d_prev, void* d_fut, int64_t ny, int64_t nx,
                       int64_t nbatch, int64_t batch_stride, void* stream);
/* InterpolationOperator::fine2coarse / coarse2fine (sbp/src/operators.rs:108-113) of nbatch
 * lines: line b of d_in starts at b * in_stride, of d_out at b * out_stride.  fine2coarse != 0:
 * n_in fine points -> n_out coarse points; else coarse -> fine.  The sizes must satisfy the
 * operator's relation.  Bit-identical to the reference's unfused sums in the same dtype. */
sbp_status sbp_interpolate(int op, int fine2coarse, int dtype, const void* d_in, void* d_out, int64_t n_in,
                           int64_t n_out, int64_t nbatch, int64_t in_stride, int64_t out_stride, void* stream);

/* Grid::metrics / Metrics::new (sbp/src/grid.rs:64-140) in f64 on device:
 * d_metrics receives 5 planes (detj, detj*dxi/dx, detj*dxi/dy, detj*deta/dx, detj*deta/dy).
 * Returns SBP_ERR_NONPHYSICAL if detj <= 0 anywhere (the reference asserts). */
sbp_status sbp_metrics(int op_xi, int op_eta, const double* d_x, const double* d_y, int64_t ny, int64_t nx,
                       double* d_metrics, void* stream);

/* Grid metrics like sbp_metrics, with no device allocation.  This entry point has no
 * counterpart in the reference.  It serves callers that cannot allocate device memory where
 * they need metrics (all device memory belongs to another runtime's pool or arena, or a
 * time-critical loop forbids allocator calls, which can synchronise the device): its working
 * memory is a fixed array inside the library (8 MiB + 256 B on every GPU that loads it, kept
 * until exit) instead of cudaMallocAsync.
 * Limits: at most 512 x 512 = 262144 points per call (larger grids return SBP_ERR_SHAPE);
 * calls share the array, so calls whose GPU work overlaps race and must not be issued; the
 * first call on each device looks the array up with cudaGetSymbolAddress and should come
 * before any stream capture; the address is kept until exit, so the entry point must not be
 * used on a device after cudaDeviceReset.  Synchronises `stream` to read the Jacobian check. */
sbp_status sbp_metrics_noalloc(int op_xi, int op_eta, const double* d_x, const double* d_y, int64_t ny,
                               int64_t nx, double* d_metrics, void* stream);

/* ---- systems: euler::System, multigrid::System, ensembles --------------- */

/* Build a system on `device`: copies the grids in, builds the f64 metrics on the device
 * (BaseSystem::create, multigrid/src/system.rs:55-78) and allocates state and stage buffers.
 * State starts at zero; instance dt starts at NaN and time at 0 (system.rs:126-128).
 * A block has at most 2^28 points (larger grids return SBP_ERR_SHAPE). */
sbp_status sbp_system_create(int device, const sbp_block_desc* blocks, int nblocks, int ninstances,
                             int precision, double gamma, sbp_system** out);
sbp_status sbp_system_destroy(sbp_system* sys);

/* Use RHS_trad even for upwind operators (euler::System::advance, euler/src/lib.rs:50-81)
 * when force_trad != 0; otherwise RHS_upwind when both operators are upwind (system.rs:520-526). */
sbp_status sbp_system_set_force_trad(sbp_system* sys, int force_trad);

/* Vortex parameters of one instance (or all when instance < 0); used by vortex initial data,
 * SBP_BC_VORTEX boundaries and sbp_system_error.  Their free stream is the instance's reference
 * state in the compensated precision; a compensated system's state is re-expressed against the
 * new reference, so the state itself is unchanged. */
sbp_status sbp_system_set_vortex(sbp_system* sys, int instance, const sbp_vortex_params* vp);
/* Field::vortex / SingleThreadedSystem::vortex (euler/src/lib.rs:319-328, system.rs:477-481):
 * state of every block of the instance(s) := the vortex at time t.  instance < 0 = all. */
sbp_status sbp_system_init_vortex(sbp_system* sys, int instance, double t);

/* Host <-> device state of one block, (4, ny, nx) f64 (the f32 state is widened / rounded). */
sbp_status sbp_system_set_state(sbp_system* sys, int block, const double* q);
sbp_status sbp_system_get_state(sbp_system* sys, int block, double* q);
/* All blocks at once, concatenated in block order; for a compensated system the state is
 * 2 x (4, ny, nx) f32 per block (hi then lo) when dtype = SBP_F32, else widened f64. */
sbp_status sbp_system_set_state_all(sbp_system* sys, int dtype, const void* q);
sbp_status sbp_system_get_state_all(sbp_system* sys, int dtype, void* q);
/* The same packing into device memory (sbp_system_state_count(dtype) elements of 8 bytes for
 * SBP_F64, 4 for SBP_F32), for callers that keep the result on the GPU. */
sbp_status sbp_system_get_state_all_device(sbp_system* sys, int dtype, void* d_q);
/* Boundary data of SBP_BC_EVAL sides from expressions: BoundaryCharacteristic::Eval with the
 * multigrid driver's evalexpr evaluator (euler/src/lib.rs:853-863, multigrid/src/eval/evalexpr.rs),
 * evaluated on the device at every stage time for each edge point.  `form` SBP_EVAL_CONSERVATION
 * gives programs for rho, rhou, rhov, e (rhou and rhov may read rho; e reads rho, rhou, rhov);
 * SBP_EVAL_PRESSURE gives rho, u, v, p (u and v read rho; p reads rho, u, v), turned into the
 * conserved state as euler/src/eval.rs:72-100 does.  Each program (len[k] <= 512 int32 words) is
 * a stack program over f64: opcode words 1..23 of csrc/eval_program.cuh (EV_CONST k, EV_VAR v with
 * v = x, y, t, rho, rhou, rhov, u, v, EV_LOAD / EV_STORE slot < 16, arithmetic, comparisons,
 * logic, EV_SELECT, EV_FN1 / EV_FN2 function ids) with `nconsts` (<= 256) constants shared by
 * the four programs; every program is checked (operands in range, stack depth <= 32, one value
 * left) and rejected with SBP_ERR_INVALID_ARGUMENT otherwise.  summationbyparts_b200/expr.py
 * compiles the expression text.  A system with SBP_BC_EVAL sides refuses to step until this has
 * been called. */
enum { SBP_EVAL_CONSERVATION = 0, SBP_EVAL_PRESSURE = 1 };
sbp_status sbp_system_set_eval(sbp_system* sys, int form, const int32_t* const code[4], const int32_t len[4],
                               const double* consts, int nconsts);
/* Host state in, `nsteps` RK4 steps, host state out: the result of sbp_system_set_state_all(q_in),
 * sbp_system_advance(nsteps), sbp_system_get_state_all(q_out), bit for bit, in one call that
 * pipelines the work over up to `nchunks` groups of whole instances (<= 0: 16): while one chunk's
 * steps run, the next chunk's state is uploaded and the previous chunk's result downloaded, so
 * the two PCIe directions and the GPU work overlap.  It replaces the reference's per-step
 * `System::advance_upwind(dt)` + `System::field()` pair (euler/src/lib.rs:149-188) for callers
 * whose state lives on the host.  q_in and q_out may be the same buffer; they should be pinned
 * (page-locked) host memory for the copies to overlap.  Instances coupled to another instance
 * (interfaces across instances, MultiGrid sides) run as one chunk.  The chunk step graphs are
 * built on the first call and kept until the tile shape or the equation form changes. */
sbp_status sbp_system_advance_host(sbp_system* sys, int dtype, const void* q_in, void* q_out, int64_t nsteps,
                                   int nchunks);
/* Number of chunks the last sbp_system_advance_host call used (-1 for a null system). */
int sbp_system_advance_host_chunks(sbp_system* sys);
/* Number of state elements of sbp_system_{set,get}_state_all for dtype. */
int64_t sbp_system_state_count(const sbp_system* sys, int dtype);

/* dt / time of one instance (instance < 0 = all).  System::set_dt (system.rs:396-405). */
sbp_status sbp_system_set_dt(sbp_system* sys, int instance, double dt);
sbp_status sbp_system_set_time(sbp_system* sys, int instance, double t);
sbp_status sbp_system_get_time(sbp_system* sys, int instance, double* t);

/* SingleThreadedSystem::max_dt (multigrid/src/system.rs:542-589) over the blocks of one instance. */
sbp_status sbp_system_max_dt(sbp_system* sys, int instance, double* dt);

/* SingleThreadedSystem::advance (system.rs:491-498): nsteps RK4 steps of every instance, each
 * with its own dt; four fused stage launches per step, replayed as one CUDA graph. */
sbp_status sbp_system_advance(sbp_system* sys, int64_t nsteps);
/* Ragged ensemble advance: instance i takes nsteps[i] steps; finished instances drop out of the
 * launch schedule.  Blocks until done. */
sbp_status sbp_system_advance_instances(sbp_system* sys, const int64_t* nsteps);

/* SingleThreadedSystem::error (system.rs:618-635): sum over the instance's blocks of
 * Field::h2_err against the vortex at the instance time.  per_instance has ninstances entries. */
sbp_status sbp_system_error(sbp_system* sys, double* per_instance);
/* Field::h2_err (euler/src/lib.rs:377-431) of one block's state against a host field q. */
sbp_status sbp_system_h2_err(sbp_system* sys, int block, const double* q, double* err);

/* Tile schedule: output tiles of ty x tx points per CTA, `threads` threads per CTA
 * (0 = keep), for every operator group; clears the autotuner's per-group choices.
 * sbp_system_autotune searches, per operator group, the tile rows (16, 32) and the width of the
 * stage kernel's grid (as many persistent CTAs per SM as fit, one per SM, or one CTA per tile),
 * timing whole RK4 steps on the current state (state and time are restored) by coordinate
 * descent over the groups, and keeps the fastest; it returns the tile shape of the group with
 * the most points. */
sbp_status sbp_system_set_tiles(sbp_system* sys, int ty, int tx, int threads);
sbp_status sbp_system_autotune(sbp_system* sys, int* ty, int* tx, int* threads);
/* Schedule of one operator group: tile rows, persistent CTAs per SM (-1 = as many as fit,
 * 0 = one CTA per tile) and the resulting grid size of its stage kernel. */
sbp_status sbp_system_group_tiles(sbp_system* sys, int group, int* ty, int* ctas_per_sm, int* grid);

/* Stream the system launches on (cudaStream_t as void*; NULL = a stream owned by the system). */
sbp_status sbp_system_set_stream(sbp_system* sys, void* stream);
/* Device pointer to one block's current state plane set, for zero-copy use: the state in an f64
 * system; in a compensated system the f32 hi planes of the state's deviation from the
 * instance's free stream (sbp_system_get_state_all_device gives the state itself). */
sbp_status sbp_system_device_state(sbp_system* sys, int block, void** d_q);
/* Explicit Runge-Kutta tableaus of utils/integrate/src/lib.rs:30-152. */
typedef enum sbp_tableau {
    SBP_RK4 = 0,
    SBP_RK4_38 = 1,
    SBP_EULER_METHOD = 2,
    SBP_MIDPOINT_METHOD = 3,
    SBP_RK6 = 4,
    SBP_FEHLBERG = 5,
    SBP_BOGACKI_SHAMPINE = 6
} sbp_tableau;
/* nsteps steps of integrate::<tableau> (utils/integrate/src/lib.rs:176-222) with each instance's
 * dt: k_i = RHS(prev + sum_j (a_ij dt) k_j) for every stage (the stage and edge kernels in a
 * k-only mode, SATs at time + dt c_i), then prev + sum_j (b_j dt) k_j, all in the reference's
 * order of operations; time += dt.  f64 systems only (SBP_ERR_UNSUPPORTED otherwise); every
 * instance takes part.  sbp_system_advance remains the fused RK4 path. */
sbp_status sbp_system_advance_tableau(sbp_system* sys, int tableau, int64_t nsteps);
/* euler::System::advance_adaptive (euler/src/lib.rs:149-186) for a single-block f64 system
 * whose four sides are SBP_BC_THIS: embedded Bogacki-Shampine steps of *guess_dt until the
 * local time reaches dt; a step is kept when h2_err(prev, low-order result) < maxerr, and
 * *guess_dt grows by 1.05 after a kept step and shrinks by 0.8 after a rejected one (the time
 * bookkeeping and the compared states are the reference's, as written).  The instance time is
 * not advanced (the reference's euler::System has none). */
sbp_status sbp_system_advance_adaptive(sbp_system* sys, double dt, double* guess_dt, double maxerr);

/* Kernel launches per RK4 step: per operator pair and stage a stage kernel and an edge (SAT)
 * kernel, plus the time update. */
int sbp_system_launches_per_step(const sbp_system* sys);

/* Per-kernel measurement.  A system's blocks are scheduled in groups, one per operator pair
 * (xi, eta); each group has one stage-kernel launch per RK4 stage.  No counterpart in the
 * reference (its RHS is a sequence of CPU sweeps); these exist so a caller can time one kernel
 * with events on the system's stream. */
/* Number of groups (builds the schedule if needed); -1 on error. */
int sbp_system_group_count(sbp_system* sys);
/* Operator pair and grid points of one group. */
sbp_status sbp_system_group_info(sbp_system* sys, int group, int* op_xi, int* op_eta, int64_t* points);
/* Enqueue one group's stage kernel for RK4 stage 0..3 on the system's stream, followed by its
 * edge (SAT) kernel when with_edges != 0.  This advances no time and checks no status: it runs
 * the stage on whatever the stage buffers hold, so a system used for it must be re-initialised
 * before its results mean anything. */
sbp_status sbp_system_launch_stage(sbp_system* sys, int group, int stage, int with_edges);

/* ---------------------------------------------------------------------------------------
 * Learned correction of a coarse solve (configuration 4).  No counterpart in the reference.
 * A 5-layer 3x3 convolutional network (4 -> 32 -> 32 -> 32 -> 32 -> 4 channels, GELU between
 * layers, zero padding) on the 64 x 64 coarse grid maps the coarse state at the end time to a
 * correction toward the restriction of a fine-grid solve.  Activations BF16, accumulation FP32
 * on the tensor cores, parameters and gradients FP32, Adam.  States are device arrays of
 * images [n][4][64][64] (component planes), consecutive images img_stride elements apart.
 * The network input is (state - in_mean) / in_scale per component, its output y the
 * correction divided by out_scale; the loss is the mean squared error of y against
 * (fine_restricted - coarse) / out_scale.
 * ------------------------------------------------------------------------------------- */
typedef struct sbp_cnn sbp_cnn;
/* Network with activation buffers for up to max_batch images; parameters from seed. */
sbp_status sbp_cnn_create(int device, int max_batch, unsigned long long seed, sbp_cnn** out);
sbp_status sbp_cnn_destroy(sbp_cnn* net);
/* Stream for all later work of the network (cudaStream_t; NULL = the legacy default stream).
 * Until it is called the network uses a stream of its own. */
sbp_status sbp_cnn_set_stream(sbp_cnn* net, void* stream);
sbp_status sbp_cnn_synchronize(sbp_cnn* net);
/* Number of FP32 parameters (padded layout: per layer weights [cout][9][cin], then biases). */
int64_t sbp_cnn_param_count(const sbp_cnn* net);
sbp_status sbp_cnn_get_params(sbp_cnn* net, float* host_params);
/* Also resets the optimiser state. */
sbp_status sbp_cnn_set_params(sbp_cnn* net, const float* host_params);
sbp_status sbp_cnn_set_normalisation(sbp_cnn* net, const float* in_mean4, const float* in_scale4,
                                     const float* out_scale4);
/* Forward pass of n images (dtype SBP_F32 or SBP_F64 state); sbp_cnn_output copies y
 * ([n][64*64][8] FP32, channels 0..3 used) to a device buffer. */
sbp_status sbp_cnn_forward(sbp_cnn* net, int n, const void* d_coarse, int dtype, int64_t img_stride);
sbp_status sbp_cnn_output(sbp_cnn* net, int n, float* d_y);
/* Forward and backward; loss (optional, synchronises) and the gradient of every parameter
 * (optional host copy, sbp_cnn_param_count floats).  d_fine_r: [n][4][64][64] FP64. */
sbp_status sbp_cnn_gradients(sbp_cnn* net, int n, const void* d_coarse, int dtype, int64_t img_stride,
                             const double* d_fine_r, float* loss, float* host_grads);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) on the gradients of this batch. */
sbp_status sbp_cnn_train_step(sbp_cnn* net, int n, const void* d_coarse, int dtype, int64_t img_stride,
                              const double* d_fine_r, float lr, float* loss);
/* corrected = coarse + y * out_scale, FP64 [n][4][64][64] into d_out. */
sbp_status sbp_cnn_apply(sbp_cnn* net, int n, const void* d_coarse, int dtype, int64_t img_stride, double* d_out);
/* Restriction of n fine images [n][4][nf][nf] (FP64, on linspace nodes) to [n][4][nc][nc] by
 * tensor-product 6-point Lagrange interpolation at the coarse linspace nodes (exact for
 * polynomials of degree 5 in each direction; one-sided stencils at the ends). */
sbp_status sbp_restrict_linspace(int n, int nf, int nc, const double* d_fine, double* d_coarse, void* stream);
/* Per image relative L2 difference |a - b| / |b| over 4 planes of `points` points each. */
sbp_status sbp_rel_l2_images(int n, int64_t points, const void* d_a, int dtype_a, int64_t stride_a,
                             const void* d_b, int dtype_b, int64_t stride_b, double* d_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SBP_B200_H */
