"""GPU systems of curvilinear blocks (the sbp_system_* C ABI).

`BlockSystem` is the common engine behind the reference-shaped front ends:
euler.System (one periodic block, euler/src/lib.rs:20-188), multigrid.System (many blocks
coupled by SATs, multigrid/src/system.rs:368-636) and ensemble.Ensemble (independent
solves).  A system holds, per block, the grid, its f64 metrics and the RK4 buffers in GPU
memory; stepping runs fused stage kernels replayed as a CUDA graph.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _capi
from ._capi import BC_EVAL, BC_GRID, BC_INTERPOLATE, BC_MULTIGRID, BC_THIS, BC_VORTEX, F32, F64, check  # noqa: F401
from .operators import SbpOperator2d

PRECISIONS = {"f64": _capi.PRECISION_F64, "f32c": _capi.PRECISION_F32_COMPENSATED}


@dataclass
class Vortice:
    """euler::Vortice (euler/src/vortex.rs:4-10)."""
    x0: float
    y0: float
    rstar: float
    eps: float


@dataclass
class VortexParameters:
    """euler::VortexParameters (euler/src/vortex.rs:15-21): up to 5 superposed vortices."""
    vortices: list = field(default_factory=list)
    mach: float = 0.5

    def to_c(self) -> _capi.VortexParams:
        if len(self.vortices) > 5:
            raise ValueError("at most 5 vortices")
        vp = _capi.VortexParams()
        vp.nvortices = len(self.vortices)
        for i, v in enumerate(self.vortices):
            vp.x0[i], vp.y0[i], vp.rstar[i], vp.eps[i] = v.x0, v.y0, v.rstar, v.eps
        vp.mach = self.mach
        return vp


@dataclass
class BlockSpec:
    """One block: grid (ny, nx), operator, boundary kinds (N, S, E, W) and instance."""
    x: np.ndarray
    y: np.ndarray
    op: SbpOperator2d
    bc: list  # 4 x (kind, neighbour)
    instance: int = 0


def _set_bc(desc, d: int, bc) -> list:
    """One side's boundary: (kind, neighbour) for This / Grid / Vortex, (BC_INTERPOLATE,
    neighbour, operator) for a 2:1 interface, (BC_MULTIGRID, [(block, start, end), ...])."""
    kind = bc[0]
    desc.bc_kind[d] = kind
    desc.bc_neighbour[d] = 0
    if kind == BC_MULTIGRID:
        tri = np.ascontiguousarray(np.array(bc[1], dtype=np.int32).reshape(-1))
        desc.bc_multigrid_count[d] = tri.size // 3
        desc.bc_multigrid[d] = tri.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        return [tri]
    desc.bc_neighbour[d] = bc[1]
    if kind == _capi.BC_INTERPOLATE:
        desc.bc_interp_op[d] = bc[2]
    return []


class BlockSystem:
    def __init__(self, blocks: list[BlockSpec], ninstances: int = 1, precision: str = "f64", gamma: float = 1.4,
                 device: int = 0):
        self.precision = precision
        self.gamma = gamma
        self.shapes = []
        self._keep = []
        arr = (_capi.BlockDesc * len(blocks))()
        for i, b in enumerate(blocks):
            x = np.ascontiguousarray(b.x, dtype=np.float64)
            y = np.ascontiguousarray(b.y, dtype=np.float64)
            if x.shape != y.shape or x.ndim != 2:
                raise ValueError("x and y must be 2-D arrays of the same shape")
            self._keep += [x, y]
            arr[i].ny, arr[i].nx = x.shape
            arr[i].op_xi, arr[i].op_eta = b.op.ids
            arr[i].x = x.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            arr[i].y = y.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            for d in range(4):
                self._keep += _set_bc(arr[i], d, b.bc[d])
            arr[i].instance = b.instance
            self.shapes.append(x.shape)
        self.ninstances = ninstances
        self.nblocks = len(blocks)
        self.block_instance = [b.instance for b in blocks]
        h = ctypes.c_void_p()
        check(_capi.lib.sbp_system_create(device, arr, len(blocks), ninstances, PRECISIONS[precision], gamma,
                                          ctypes.byref(h)))
        self.h = h
        self._keep = []

    # -- lifecycle
    def close(self) -> None:
        if getattr(self, "h", None):
            _capi.lib.sbp_system_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- configuration
    def set_force_trad(self, on: bool) -> None:
        check(_capi.lib.sbp_system_set_force_trad(self.h, int(on)))

    def set_eval(self, expressions) -> None:
        """Boundary data of BC_EVAL sides from an expr.Expressions evaluator, compiled to the
        device programs of sbp_system_set_eval."""
        from .expr import compile_program
        form, codes, consts = compile_program(expressions)
        arrs = [np.ascontiguousarray(np.array(c, dtype=np.int32)) for c in codes]
        ptrs = (ctypes.POINTER(ctypes.c_int32) * 4)(*[a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)) for a in arrs])
        lens = (ctypes.c_int32 * 4)(*[len(c) for c in codes])
        cv = np.ascontiguousarray(np.array(consts if consts else [0.0], dtype=np.float64))
        check(_capi.lib.sbp_system_set_eval(self.h, form, ptrs, lens, cv.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                            len(consts)))

    def set_vortex(self, params: VortexParameters, instance: int = -1) -> None:
        vp = params.to_c()
        check(_capi.lib.sbp_system_set_vortex(self.h, instance, ctypes.byref(vp)))

    def init_vortex(self, t: float = 0.0, instance: int = -1) -> None:
        check(_capi.lib.sbp_system_init_vortex(self.h, instance, t))

    def set_dt(self, dt: float, instance: int = -1) -> None:
        check(_capi.lib.sbp_system_set_dt(self.h, instance, dt))

    def set_time(self, t: float, instance: int = -1) -> None:
        check(_capi.lib.sbp_system_set_time(self.h, instance, t))

    def time(self, instance: int = 0) -> float:
        t = ctypes.c_double()
        check(_capi.lib.sbp_system_get_time(self.h, instance, ctypes.byref(t)))
        return t.value

    def set_tiles(self, ty: int, tx: int, threads: int = 0) -> None:
        check(_capi.lib.sbp_system_set_tiles(self.h, ty, tx, threads))

    def autotune(self) -> tuple[int, int, int]:
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(_capi.lib.sbp_system_autotune(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def set_stream(self, stream_handle: int) -> None:
        check(_capi.lib.sbp_system_set_stream(self.h, ctypes.c_void_p(stream_handle)))

    def launches_per_step(self) -> int:
        return _capi.lib.sbp_system_launches_per_step(self.h)

    # -- per-kernel measurement (sbp_system_group_* / sbp_system_launch_stage)
    def groups(self) -> list[tuple[int, int, int]]:
        """(op_xi, op_eta, points) of each stage-kernel group."""
        n = _capi.lib.sbp_system_group_count(self.h)
        if n < 0:
            raise _capi.SbpError(1, _capi.lib.sbp_last_error().decode(errors='replace'))
        out = []
        for g in range(n):
            ox, oy, pts = ctypes.c_int(), ctypes.c_int(), ctypes.c_int64()
            check(_capi.lib.sbp_system_group_info(self.h, g, ctypes.byref(ox), ctypes.byref(oy), ctypes.byref(pts)))
            out.append((ox.value, oy.value, pts.value))
        return out

    def group_tiles(self, group: int) -> tuple[int, int, int]:
        """(tile rows, persistent CTAs per SM (-1 = as many as fit, 0 = one CTA per tile), grid
        size) of one stage-kernel group's schedule."""
        ty, cps, grid = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(_capi.lib.sbp_system_group_tiles(self.h, group, ctypes.byref(ty), ctypes.byref(cps), ctypes.byref(grid)))
        return ty.value, cps.value, grid.value

    def launch_stage(self, group: int, stage: int, with_edges: bool = False) -> None:
        """Enqueue one group's stage kernel (and optionally its edge kernel) on the system's
        stream.  Advances no time; the stage buffers are left as the launch leaves them."""
        check(_capi.lib.sbp_system_launch_stage(self.h, group, stage, int(with_edges)))

    # -- state
    def set_state(self, block: int, q: np.ndarray) -> None:
        q = np.ascontiguousarray(q, dtype=np.float64)
        if q.shape != (4,) + tuple(self.shapes[block]):
            raise ValueError(f"state of block {block} must be (4, {self.shapes[block][0]}, {self.shapes[block][1]})")
        check(_capi.lib.sbp_system_set_state(self.h, block, q.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))

    def state(self, block: int) -> np.ndarray:
        q = np.zeros((4,) + tuple(self.shapes[block]))
        check(_capi.lib.sbp_system_get_state(self.h, block, q.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return q

    def state_count(self, dtype: int = F64) -> int:
        return _capi.lib.sbp_system_state_count(self.h, dtype)

    def set_state_all(self, buf, dtype: int = F64) -> None:
        """buf: host buffer (numpy array or pinned torch tensor) holding every block's state."""
        ptr = buf.ctypes.data if isinstance(buf, np.ndarray) else buf.data_ptr()
        check(_capi.lib.sbp_system_set_state_all(self.h, dtype, ctypes.c_void_p(ptr)))

    def get_state_all(self, buf, dtype: int = F64) -> None:
        ptr = buf.ctypes.data if isinstance(buf, np.ndarray) else buf.data_ptr()
        check(_capi.lib.sbp_system_get_state_all(self.h, dtype, ctypes.c_void_p(ptr)))

    def get_state_all_device(self, d_ptr: int, dtype: int = F64) -> None:
        """Pack every block's state into device memory at d_ptr (state_count(dtype) elements)."""
        check(_capi.lib.sbp_system_get_state_all_device(self.h, dtype, ctypes.c_void_p(d_ptr)))

    def advance_host(self, buf_in, buf_out, nsteps: int, dtype: int = F64, nchunks: int = 0) -> int:
        """set_state_all(buf_in); advance(nsteps); get_state_all(buf_out) in one call, pipelined over
        up to nchunks groups of whole instances (0: the library's default).  Returns the number of
        chunks used.  Pinned host buffers let the copies overlap the steps."""
        pi = buf_in.ctypes.data if isinstance(buf_in, np.ndarray) else buf_in.data_ptr()
        po = buf_out.ctypes.data if isinstance(buf_out, np.ndarray) else buf_out.data_ptr()
        check(_capi.lib.sbp_system_advance_host(self.h, dtype, ctypes.c_void_p(pi), ctypes.c_void_p(po), int(nsteps),
                                                int(nchunks)))
        return _capi.lib.sbp_system_advance_host_chunks(self.h)

    # -- stepping and diagnostics
    def max_dt(self, instance: int = 0) -> float:
        dt = ctypes.c_double()
        check(_capi.lib.sbp_system_max_dt(self.h, instance, ctypes.byref(dt)))
        return dt.value

    def advance(self, nsteps: int) -> None:
        check(_capi.lib.sbp_system_advance(self.h, int(nsteps)))

    def advance_tableau(self, tableau: str, nsteps: int) -> None:
        """nsteps steps of integrate::<tableau> (rk4, rk4_38, euler, midpoint, rk6, fehlberg,
        bogacki_shampine) with each instance's dt; f64 systems."""
        check(_capi.lib.sbp_system_advance_tableau(self.h, _capi.TABLEAUS[tableau], int(nsteps)))

    def advance_adaptive(self, dt: float, guess_dt: float, maxerr: float) -> float:
        """euler::System::advance_adaptive on a single-block periodic (This) f64 system; returns
        the updated guess_dt."""
        g = ctypes.c_double(guess_dt)
        check(_capi.lib.sbp_system_advance_adaptive(self.h, dt, ctypes.byref(g), maxerr))
        return g.value

    def advance_instances(self, nsteps) -> None:
        arr = (ctypes.c_int64 * self.ninstances)(*[int(n) for n in nsteps])
        check(_capi.lib.sbp_system_advance_instances(self.h, arr))

    def errors(self) -> np.ndarray:
        out = np.zeros(self.ninstances)
        check(_capi.lib.sbp_system_error(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def h2_err(self, block: int, q: np.ndarray) -> float:
        q = np.ascontiguousarray(q, dtype=np.float64)
        e = ctypes.c_double()
        check(_capi.lib.sbp_system_h2_err(self.h, block, q.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                          ctypes.byref(e)))
        return e.value
