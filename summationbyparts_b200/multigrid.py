"""multigrid::System on the GPU: blocks coupled through characteristic SATs.

Mirrors the reference's multigrid driver (multigrid/src/system.rs:368-636):
    sys = System(grids, vortex_params)      # grids: list of Grid
    dt = sys.max_dt(); sys.set_dt(dt)
    sys.advance(nsteps)
    err = sys.error()                       # sum over blocks of h2_err vs the vortex
Boundary characteristics per side are BoundaryCharacteristic values: THIS (own opposite
edge), ("grid", g) (block g's opposite edge) or VORTEX (exact vortex data at stage time),
euler/src/lib.rs:737-745, 869-930.  Grids with fine = 2*coarse-1 interpolation or
multi-neighbour edges are not supported (the single-threaded driver also rejects nothing
here: the library returns SBP_ERR_SHAPE for unequal interface lengths).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from ._capi import BC_GRID, BC_THIS, BC_VORTEX
from .system import BlockSpec, BlockSystem, VortexParameters

THIS = "this"
VORTEX = "vortex"


def grid_bc(g: int):
    return ("grid", g)


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
    if isinstance(v, tuple) and v[0] == "grid":
        return (BC_GRID, int(v[1]))
    raise ValueError(f"unsupported boundary characteristic {v!r}")


class System:
    def __init__(self, grids: list[Grid], vortex: VortexParameters, gamma: float = 1.4, precision: str = "f64",
                 device: int = 0, time: float = 0.0):
        specs = [BlockSpec(g.x, g.y, g.op, [_bc(g.north), _bc(g.south), _bc(g.east), _bc(g.west)], 0) for g in grids]
        self.grids = grids
        self._sys = BlockSystem(specs, 1, precision, gamma, device)
        self._sys.set_vortex(vortex)
        self._sys.init_vortex(time)
        self._sys.set_time(time)

    def max_dt(self) -> float:
        return self._sys.max_dt(0)

    def set_dt(self, dt: float) -> None:
        self._sys.set_dt(dt)

    def advance(self, nsteps: int) -> None:
        self._sys.advance(nsteps)

    def error(self) -> float:
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
