"""multigrid::System on the GPU: blocks coupled through characteristic SATs.

Mirrors the reference's multigrid driver (multigrid/src/system.rs:368-636):
    sys = System(grids, vortex_params)      # grids: list of Grid
    dt = sys.max_dt(); sys.set_dt(dt)
    sys.advance(nsteps)
    err = sys.error()                       # sum over blocks of h2_err vs the vortex
Boundary characteristics per side are BoundaryCharacteristic values (euler/src/lib.rs:737-745,
804-930): THIS (own opposite edge), ("grid", g) (block g's opposite edge), VORTEX (exact vortex
data at stage time), ("interpolate", g, op) (block g's opposite edge through a 2:1
interpolation operator, op 0..3 = Interpolation4, 8, 9, 9h2) and ("multi", [(g, start, end),
...]) (segments of several blocks' opposite edges).  The library returns SBP_ERR_SHAPE for
interfaces whose lengths do not fit.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from ._capi import BC_EVAL, BC_GRID, BC_INTERPOLATE, BC_MULTIGRID, BC_THIS, BC_VORTEX
from .system import BlockSpec, BlockSystem, VortexParameters

THIS = "this"
VORTEX = "vortex"
EVAL = "eval"  # boundary data from the system's boundary expressions


def grid_bc(g: int):
    return ("grid", g)


def interpolate_bc(g: int, op: int):
    return ("interpolate", g, op)


def multi_bc(segments):
    return ("multi", [tuple(int(v) for v in sgm) for sgm in segments])


@dataclass
class Grid:
    x: np.ndarray
    y: np.ndarray
    op: object
    north: object = VORTEX
    south: object = VORTEX
    east: object = VORTEX
    west: object = VORTEX
    name: str = ""


def _bc(v):
    if v == THIS:
        return (BC_THIS, 0)
    if v == VORTEX:
        return (BC_VORTEX, 0)
    if v == EVAL:
        return (BC_EVAL, 0)
    if isinstance(v, tuple) and v[0] == "grid":
        return (BC_GRID, int(v[1]))
    if isinstance(v, tuple) and v[0] == "interpolate":
        return (BC_INTERPOLATE, int(v[1]), int(v[2]))
    if isinstance(v, tuple) and v[0] == "multi":
        return (BC_MULTIGRID, list(v[1]))
    raise ValueError(f"unsupported boundary characteristic {v!r}")


class System:
    def __init__(self, grids: list[Grid], vortex, gamma: float = 1.4, precision: str = "f64",
                 device: int = 0, time: float = 0.0, boundary_vortex: VortexParameters | None = None,
                 boundary_expressions=None):
        """vortex: the initial conditions (and the exact solution of error()), a
        VortexParameters or an expr.Expressions (evaluated on the host at `time`, system.rs:135-153);
        boundary_vortex: the vortex of VORTEX sides when it differs from the initial one;
        boundary_expressions: the expr.Expressions of EVAL sides (evaluated on the device at every
        stage time)."""
        from .expr import Expressions
        specs = [BlockSpec(g.x, g.y, g.op, [_bc(g.north), _bc(g.south), _bc(g.east), _bc(g.west)], 0) for g in grids]
        self.grids = grids
        self.expressions = vortex if isinstance(vortex, Expressions) else None
        self.vortex = None if self.expressions is not None else vortex
        self.boundary_vortex = boundary_vortex or self.vortex
        self._sys = BlockSystem(specs, 1, precision, gamma, device)
        if self.expressions is not None:
            for b, g in enumerate(grids):
                self._sys.set_state(b, self.expressions.evaluate(time, g.x, g.y))
            if self.boundary_vortex is not None:
                self._sys.set_vortex(self.boundary_vortex)
        else:
            self._sys.set_vortex(vortex)
            self._sys.init_vortex(time)
            if self.boundary_vortex is not vortex:
                self._sys.set_vortex(self.boundary_vortex)
        if boundary_expressions is not None:
            self._sys.set_eval(boundary_expressions)
        self._sys.set_time(time)

    def max_dt(self) -> float:
        return self._sys.max_dt(0)

    def set_dt(self, dt: float) -> None:
        self._sys.set_dt(dt)

    def advance(self, nsteps: int) -> None:
        self._sys.advance(nsteps)

    def error(self) -> float:
        """Sum over blocks of h2_err against the initial conditions (vortex or expressions)
        evaluated at the current time (multigrid/src/system.rs:618-635)."""
        if self.expressions is not None:
            t = self.time
            return float(sum(self._sys.h2_err(b, self.expressions.evaluate(t, g.x, g.y))
                             for b, g in enumerate(self.grids)))
        if self.boundary_vortex is not self.vortex:
            self._sys.set_vortex(self.vortex)
            e = float(self._sys.errors()[0])
            self._sys.set_vortex(self.boundary_vortex)
            return e
        return float(self._sys.errors()[0])

    @property
    def time(self) -> float:
        return self._sys.time(0)

    def field(self, block: int) -> np.ndarray:
        return self._sys.state(block)

    def set_field(self, block: int, q: np.ndarray) -> None:
        self._sys.set_state(block, q)

    @property
    def engine(self) -> BlockSystem:
        return self._sys
