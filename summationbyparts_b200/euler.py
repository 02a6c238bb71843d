"""euler::System on the GPU: one curvilinear block, periodic on all sides.

Drop-in for the reference's euler::System<SBP> (euler/src/lib.rs:20-188):
    sys = System(x, y, Upwind4())
    sys.vortex(0.0, VortexParameters([Vortice(-1.0, 0.0, 0.5, 1.0)], mach=0.5))
    sys.advance_upwind(dt)        # RHS_upwind + RK4
    sys.advance(dt)               # RHS_trad + RK4
    q = sys.field()               # (4, ny, nx) numpy array
The boundary characteristic is `This` on every side (euler/src/lib.rs:51-56), so the block
is periodic, and the RHS ignores time as the reference's closure does.
"""
from __future__ import annotations

import numpy as np

from ._capi import BC_THIS
from .system import BlockSpec, BlockSystem, Vortice, VortexParameters  # noqa: F401

GAMMA = 1.4  # euler::GAMMA (euler/src/lib.rs:15); read when a System is created


class System:
    def __init__(self, x: np.ndarray, y: np.ndarray, op, precision: str = "f64", device: int = 0):
        self._x = np.ascontiguousarray(x, dtype=np.float64)
        self._y = np.ascontiguousarray(y, dtype=np.float64)
        self.op = op
        self._sys = BlockSystem([BlockSpec(self._x, self._y, op, [(BC_THIS, 0)] * 4, 0)], 1, precision, GAMMA,
                                device)
        self._dt = None

    def vortex(self, t: float, params: VortexParameters) -> None:
        """Field::vortex (euler/src/lib.rs:319-328): state := vortex at time t."""
        self._sys.set_vortex(params)
        self._sys.init_vortex(t)

    def init_with_vortex(self, x0: float, y0: float) -> None:
        """System::init_with_vortex (euler/src/lib.rs:83-103)."""
        self.vortex(0.0, VortexParameters([Vortice(x0, y0, 1.0, 3.0)], mach=0.5))

    def _step(self, dt: float, trad: bool) -> None:
        if self._dt != dt:
            self._sys.set_dt(dt)
            self._dt = dt
        self._sys.set_force_trad(trad)
        self._sys.set_time(0.0)  # the reference integrates with a local time of 0 every step
        self._sys.advance(1)

    def advance(self, dt: float) -> None:
        """System::advance: one RK4 step of RHS_trad (euler/src/lib.rs:50-81)."""
        self._step(dt, True)

    def advance_upwind(self, dt: float) -> None:
        """System::advance_upwind: one RK4 step of RHS_upwind (euler/src/lib.rs:124-147)."""
        self._step(dt, False)

    def advance_upwind_n(self, dt: float, nsteps: int) -> None:
        """nsteps of advance_upwind in one call (one graph replay per step, no host sync between)."""
        if self._dt != dt:
            self._sys.set_dt(dt)
            self._dt = dt
        self._sys.set_force_trad(False)
        self._sys.advance(nsteps)

    def advance_adaptive(self, dt: float, guess_dt: float, maxerr: float) -> float:
        """System::advance_adaptive (euler/src/lib.rs:149-186): embedded Bogacki-Shampine steps
        with RHS_upwind until the local time reaches dt; returns the updated guess_dt (the
        reference updates its `&mut guess_dt` argument)."""
        self._sys.set_force_trad(False)
        return self._sys.advance_adaptive(dt, guess_dt, maxerr)

    def field(self) -> np.ndarray:
        return self._sys.state(0)

    def set_field(self, q: np.ndarray) -> None:
        self._sys.set_state(0, q)

    def x(self) -> np.ndarray:
        return self._x

    def y(self) -> np.ndarray:
        return self._y

    def nx(self) -> int:
        return self._x.shape[1]

    def ny(self) -> int:
        return self._x.shape[0]

    def h2_err(self, other: np.ndarray) -> float:
        """Field::h2_err of the current state against `other` (euler/src/lib.rs:377-431)."""
        return self._sys.h2_err(0, other)
