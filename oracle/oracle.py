"""ctypes binding of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

The oracle is a C++ restatement of the reference's arithmetic (see
sbp_oracle.h for scope and parity status).  Only the tests, the smoke entry
point and the CPU-baseline leg of the benchmark import this module; the
library under test never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")

UPWIND4, UPWIND4H2, UPWIND9, UPWIND9H2, SBP4, SBP8 = range(6)
OPERATORS = {"upwind4": UPWIND4, "upwind4h2": UPWIND4H2, "upwind9": UPWIND9,
             "upwind9h2": UPWIND9H2, "sbp4": SBP4, "sbp8": SBP8}
DIFF, DISS = 0, 1
XI, ETA = 0, 1
F64, F32 = 0, 1
BC_THIS, BC_GRID, BC_VORTEX, BC_INTERPOLATE, BC_MULTIGRID = 0, 1, 2, 3, 4
INTERP4, INTERP8, INTERP9, INTERP9H2 = 0, 1, 2, 3
NORTH, SOUTH, EAST, WEST = 0, 1, 2, 3


class VortexParams(ctypes.Structure):
    _fields_ = [("nvortices", ctypes.c_int), ("x0", ctypes.c_double * 5), ("y0", ctypes.c_double * 5),
                ("rstar", ctypes.c_double * 5), ("eps", ctypes.c_double * 5), ("mach", ctypes.c_double)]


class BlockDesc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int64), ("ny", ctypes.c_int64), ("op_xi", ctypes.c_int), ("op_eta", ctypes.c_int),
                ("x", ctypes.POINTER(ctypes.c_double)), ("y", ctypes.POINTER(ctypes.c_double)),
                ("bc_kind", ctypes.c_int * 4), ("bc_neighbour", ctypes.c_int * 4),
                ("bc_interp_op", ctypes.c_int * 4), ("bc_mg_count", ctypes.c_int * 4),
                ("bc_mg", ctypes.POINTER(ctypes.c_int) * 4)]


def build() -> None:
    """Compile the oracle libraries (make in this directory)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _host_has_v3() -> bool:
    try:
        flags = open("/proc/cpuinfo").read()
    except OSError:
        return False
    return all(f in flags for f in (" avx2", " fma", " bmi2"))


_LIB = None


def lib(fast: bool = False) -> ctypes.CDLL:
    """Load the oracle.  fast=True selects the x86-64-v3 build when the host supports it (identical
    results: the source is compiled without FP contraction either way)."""
    global _LIB
    name = "liborc_v3.so" if fast and _host_has_v3() else "liborc_generic.so"
    path = os.path.join(BUILD, name)
    if not os.path.exists(path):
        build()
    if _LIB is not None and _LIB[0] == path:
        return _LIB[1]
    L = ctypes.CDLL(path)
    dp = ctypes.POINTER(ctypes.c_double)
    L.orc_op_table.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    L.orc_op_shape.argtypes = [ctypes.c_int] + [ctypes.POINTER(ctypes.c_int)] * 5
    L.orc_op_apply.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                               ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64]
    L.orc_metrics.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, ctypes.c_int64, ctypes.c_int64, dp]
    L.orc_vortex.argtypes = [ctypes.POINTER(VortexParams), ctypes.c_double, ctypes.c_double, dp, dp,
                             ctypes.c_int64, dp]
    L.orc_rhs.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, dp, dp, dp, dp, dp, dp,
                          ctypes.c_int64, ctypes.c_int64, ctypes.c_int, dp]
    L.orc_h2_err.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, ctypes.c_int64, ctypes.c_int64]
    L.orc_h2_err.restype = ctypes.c_double
    L.orc_interpolate.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64,
                                  ctypes.c_void_p, ctypes.c_int64]
    L.orc_system_create.argtypes = [ctypes.POINTER(BlockDesc), ctypes.c_int, ctypes.c_double]
    L.orc_system_create.restype = ctypes.c_void_p
    L.orc_system_destroy.argtypes = [ctypes.c_void_p]
    L.orc_system_set_vortex.argtypes = [ctypes.c_void_p, ctypes.POINTER(VortexParams)]
    L.orc_system_init_vortex.argtypes = [ctypes.c_void_p, ctypes.c_double]
    L.orc_system_set_state.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
    L.orc_system_get_state.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
    L.orc_system_get_metrics.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
    L.orc_system_advance.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.c_int]
    L.orc_system_advance_tableau.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double,
                                             ctypes.c_int]
    L.orc_system_advance_adaptive.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.POINTER(ctypes.c_double),
                                              ctypes.c_double]
    L.orc_system_time.argtypes = [ctypes.c_void_p]
    L.orc_system_time.restype = ctypes.c_double
    L.orc_system_set_time.argtypes = [ctypes.c_void_p, ctypes.c_double]
    L.orc_system_max_dt.argtypes = [ctypes.c_void_p]
    L.orc_system_max_dt.restype = ctypes.c_double
    L.orc_system_error.argtypes = [ctypes.c_void_p]
    L.orc_system_error.restype = ctypes.c_double
    L.orc_systems_advance.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_int64), dp, ctypes.c_int]
    _LIB = (path, L)
    return L


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def op_shape(op: int):
    v = [ctypes.c_int() for _ in range(5)]
    rc = lib().orc_op_shape(op, *[ctypes.byref(x) for x in v])
    if rc:
        raise ValueError(op)
    m, n, d, h2, upw = (x.value for x in v)
    return m, n, d, bool(h2), bool(upw)


def op_table(op: int, kind: int, part: int, dtype=np.float64) -> np.ndarray:
    out = np.zeros(8 * 13, dtype=dtype)
    cnt = lib().orc_op_table(op, kind, part, F64 if dtype == np.float64 else F32, out.ctypes.data)
    if cnt < 0:
        raise ValueError("no such table")
    return out[:cnt].copy()


def op_apply(op: int, direction: int, kind: int, a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a)
    out = np.zeros_like(a)
    dt = F64 if a.dtype == np.float64 else F32
    ny, nx = a.shape
    rc = lib().orc_op_apply(op, direction, kind, dt, a.ctypes.data, out.ctypes.data, ny, nx)
    if rc:
        raise ValueError(f"orc_op_apply failed ({rc})")
    return out


def diffxi(op, a):
    return op_apply(op, XI, DIFF, a)


def diffeta(op, a):
    return op_apply(op, ETA, DIFF, a)


def dissxi(op, a):
    return op_apply(op, XI, DISS, a)


def disseta(op, a):
    return op_apply(op, ETA, DISS, a)


def metrics(op_xi: int, op_eta: int, x: np.ndarray, y: np.ndarray) -> np.ndarray:
    ny, nx = x.shape
    out = np.zeros((5, ny, nx))
    rc = lib().orc_metrics(op_xi, op_eta, _dp(np.ascontiguousarray(x)), _dp(np.ascontiguousarray(y)), ny, nx, _dp(out))
    if rc:
        raise ValueError(f"orc_metrics failed ({rc})")
    return out


def vortex_params(vortices, mach) -> VortexParams:
    vp = VortexParams()
    vp.nvortices = len(vortices)
    for i, v in enumerate(vortices):
        vp.x0[i], vp.y0[i], vp.rstar[i], vp.eps[i] = v["x0"], v["y0"], v["rstar"], v["eps"]
    vp.mach = mach
    return vp


def vortex(vortices, mach, gamma, t, x, y) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    q = np.zeros((4,) + x.shape)
    vp = vortex_params(vortices, mach)
    lib().orc_vortex(ctypes.byref(vp), gamma, t, _dp(x), _dp(y), x.size, _dp(q))
    return q


def rhs(op_xi, op_eta, gamma, q, met, zn, zs, ze, zw, force_trad=False) -> np.ndarray:
    _, ny, nx = q.shape
    k = np.zeros_like(q)
    rc = lib().orc_rhs(op_xi, op_eta, gamma, _dp(q), _dp(met), _dp(zn), _dp(zs), _dp(ze), _dp(zw),
                       ny, nx, int(force_trad), _dp(k))
    if rc:
        raise ValueError(f"orc_rhs failed ({rc})")
    return k


def h2_err(op_xi, op_eta, a, b) -> float:
    _, ny, nx = a.shape
    return lib().orc_h2_err(op_xi, op_eta, _dp(np.ascontiguousarray(a)), _dp(np.ascontiguousarray(b)), ny, nx)


def set_bc(desc, d, bc, keep):
    """bc: (kind, neighbour), (BC_INTERPOLATE, neighbour, operator) or
    (BC_MULTIGRID, [(grid, start, end), ...])."""
    kind = bc[0]
    desc.bc_kind[d] = kind
    desc.bc_neighbour[d] = 0
    if kind == BC_MULTIGRID:
        tri = np.ascontiguousarray(np.array(bc[1], dtype=np.int32).reshape(-1))
        keep.append(tri)
        desc.bc_mg_count[d] = tri.size // 3
        desc.bc_mg[d] = tri.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    else:
        desc.bc_neighbour[d] = bc[1]
        if kind == BC_INTERPOLATE:
            desc.bc_interp_op[d] = bc[2]


def interpolate(op: int, fine2coarse: bool, x, dtype=np.float64) -> np.ndarray:
    """InterpolationOperator::fine2coarse / coarse2fine of one line (f64, or the reference's f32
    build for dtype float32)."""
    x = np.ascontiguousarray(x, dtype=dtype)
    n = x.size
    odd = op != INTERP9H2
    if fine2coarse:
        m = (n + 1) // 2 if odd else n // 2 + 1
    else:
        m = 2 * n - 1 if odd else 2 * (n - 1)
    out = np.empty(m, dtype=dtype)
    L = lib(False)
    dt = F64 if x.dtype == np.float64 else F32
    if L.orc_interpolate(op, int(fine2coarse), dt, x.ctypes.data, n, out.ctypes.data, m) != 0:
        raise ValueError("orc_interpolate: bad operator or sizes")
    return out


class System:
    """Multi-block system with the reference's single-threaded multigrid semantics."""

    def __init__(self, blocks, gamma=1.4, fast=False):
        """blocks: list of dicts {x, y, op_xi, op_eta, bc: [(kind, neighbour)] * 4 (N, S, E, W)}."""
        self._L = lib(fast)
        self._keep = []
        arr = (BlockDesc * len(blocks))()
        for i, b in enumerate(blocks):
            x = np.ascontiguousarray(b["x"], dtype=np.float64)
            y = np.ascontiguousarray(b["y"], dtype=np.float64)
            self._keep += [x, y]
            arr[i].ny, arr[i].nx = x.shape
            arr[i].op_xi, arr[i].op_eta = b["op_xi"], b["op_eta"]
            arr[i].x, arr[i].y = _dp(x), _dp(y)
            for d in range(4):
                set_bc(arr[i], d, b["bc"][d], self._keep)
        self.shapes = [(int(arr[i].ny), int(arr[i].nx)) for i in range(len(blocks))]
        self.h = self._L.orc_system_create(arr, len(blocks), gamma)
        if not self.h:
            raise ValueError("orc_system_create failed (non-positive Jacobian?)")

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self._L.orc_system_destroy(h)
            self.h = None

    def set_vortex(self, vortices, mach):
        self._vp = vortex_params(vortices, mach)
        self._L.orc_system_set_vortex(self.h, ctypes.byref(self._vp))

    def init_vortex(self, t=0.0):
        self._L.orc_system_init_vortex(self.h, t)

    def set_state(self, b, q):
        q = np.ascontiguousarray(q, dtype=np.float64)
        assert q.shape == (4,) + self.shapes[b]
        self._L.orc_system_set_state(self.h, b, _dp(q))

    def state(self, b) -> np.ndarray:
        q = np.zeros((4,) + self.shapes[b])
        self._L.orc_system_get_state(self.h, b, _dp(q))
        return q

    def metrics(self, b) -> np.ndarray:
        m = np.zeros((5,) + self.shapes[b])
        self._L.orc_system_get_metrics(self.h, b, _dp(m))
        return m

    def advance(self, nsteps, dt, force_trad=False):
        rc = self._L.orc_system_advance(self.h, nsteps, dt, int(force_trad))
        if rc:
            raise RuntimeError(f"orc_system_advance failed ({rc})")

    @property
    def time(self) -> float:
        return self._L.orc_system_time(self.h)

    @time.setter
    def time(self, t):
        self._L.orc_system_set_time(self.h, t)

    def advance_tableau(self, tableau: int, nsteps: int, dt: float, force_trad: bool = False):
        """integrate::<tableau> steps: 0 Rk4, 1 Rk4_38, 2 EulerMethod, 3 MidpointMethod, 4 Rk6,
        5 Fehlberg, 6 BogackiShampine."""
        rc = self._L.orc_system_advance_tableau(self.h, tableau, nsteps, dt, int(force_trad))
        if rc:
            raise RuntimeError(f"orc_system_advance_tableau: {rc}")

    def advance_adaptive(self, dt: float, guess_dt: float, maxerr: float) -> float:
        g = ctypes.c_double(guess_dt)
        rc = self._L.orc_system_advance_adaptive(self.h, dt, ctypes.byref(g), maxerr)
        if rc:
            raise RuntimeError(f"orc_system_advance_adaptive: {rc}")
        return g.value

    def max_dt(self) -> float:
        return self._L.orc_system_max_dt(self.h)

    def error(self) -> float:
        return self._L.orc_system_error(self.h)


def advance_many(systems, nsteps, dts, nthreads) -> None:
    """Advance independent systems concurrently on nthreads host threads."""
    n = len(systems)
    hs = (ctypes.c_void_p * n)(*[s.h for s in systems])
    st = (ctypes.c_int64 * n)(*[int(x) for x in nsteps])
    dt = np.ascontiguousarray(dts, dtype=np.float64)
    rc = systems[0]._L.orc_systems_advance(hs, n, st, _dp(dt), nthreads)
    if rc:
        raise RuntimeError(f"orc_systems_advance failed ({rc})")
