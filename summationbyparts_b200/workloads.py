"""Deterministic synthetic workloads (the benchmark and parity configurations).

The reference publishes no dataset or benchmark inputs; every workload here is generated
from a documented seed:

* SplitMix64 (Steele, Lea & Flood, "Fast splittable pseudorandom number generators",
  OOPSLA 2014) with the output z mapped to a double u = (z >> 11) * 2^-53 in [0, 1).
* vortex: centre (-1, 0), eps 1, rstar 0.5, Mach 0.5, gamma 1.4 (euler/tests/convergence.rs:23-35).
* grids: ndarray-style linspace (start + step * i, step = (end - start) / (n - 1)), optionally
  warped by x = xi + 0.1 sin(pi xi / 5) sin(pi eta / 5), y = eta + 0.1 sin(pi xi / 5) sin(pi eta / 5).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from ._capi import BC_GRID, BC_VORTEX
from .operators import BY_ID, UPWIND4, UPWIND9, Upwind4, Upwind9
from .system import BlockSpec, Vortice, VortexParameters

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
M1 = np.uint64(0xBF58476D1CE4E5B9)
M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, n: int, start: int = 0) -> np.ndarray:
    """Outputs start..start+n-1 of the SplitMix64 stream seeded with `seed` (uint64)."""
    with np.errstate(over="ignore"):
        i = np.arange(start + 1, start + n + 1, dtype=np.uint64)
        z = np.uint64(seed) + i * GOLDEN
        z = (z ^ (z >> np.uint64(30))) * M1
        z = (z ^ (z >> np.uint64(27))) * M2
        return z ^ (z >> np.uint64(31))


def uniform01(seed: int, n: int, start: int = 0) -> np.ndarray:
    return (splitmix64(seed, n, start) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def uniform_pm1(seed: int, n: int) -> np.ndarray:
    """Doubles in [-1, 1): 2u - 1."""
    return 2.0 * uniform01(seed, n) - 1.0


def linspace(a: float, b: float, n: int) -> np.ndarray:
    step = (b - a) / (n - 1)
    return a + step * np.arange(n, dtype=np.float64)


def cartesian(xa, xb, nx, ya, yb, ny):
    xs, ys = linspace(xa, xb, nx), linspace(ya, yb, ny)
    return np.ascontiguousarray(np.broadcast_to(xs[None, :], (ny, nx))), \
        np.ascontiguousarray(np.broadcast_to(ys[:, None], (ny, nx)))


def warped(xa, xb, nx, ya, yb, ny, amp=0.1):
    xi, eta = cartesian(xa, xb, nx, ya, yb, ny)
    s = amp * np.sin(np.pi * xi / 5.0) * np.sin(np.pi * eta / 5.0)
    return xi + s, eta + s


STANDARD_VORTEX = VortexParameters([Vortice(-1.0, 0.0, 0.5, 1.0)], mach=0.5)


# ----- configuration 0: single Cartesian block, vortex SATs --------------------------------
@dataclass
class Config0:
    n: int = 64
    steps: int = 100

    def blocks(self):
        x, y = cartesian(-5.0, 5.0, self.n, -5.0, 5.0, self.n)
        return [BlockSpec(x, y, Upwind4(), [(BC_VORTEX, 0)] * 4, 0)]

    @property
    def dt(self):
        return 0.2 * min(1.0 / (self.n - 1), 1.0 / (self.n - 1))


# ----- configuration 1: operator microbench fields ------------------------------------------
def operator_fields(n: int = 4096, nfields: int = 4, seed: int = 0) -> np.ndarray:
    """(nfields, n, n) i.i.d. U[-1, 1) doubles from SplitMix64(seed); f32 inputs are these rounded."""
    return uniform_pm1(seed, nfields * n * n).reshape(nfields, n, n)


# ----- configuration 2: curvilinear multi-block ---------------------------------------------
# The six sizes listed for this case (101x51, 81x81, 65x129, 49x97, 121x41, 73x73) share no
# edge length, so no conforming tiling exists and the reference's Grid coupling needs equal
# interface lengths (euler/src/lib.rs:1163).  The layout used is 2 columns x 3 rows with
# nx in (101, 81) and ny in (51, 81, 73): uneven blocks, every interface conforming.
MB_NX = (101, 81)
MB_NY = (51, 81, 73)


def multiblock(op=None, nx=MB_NX, ny=MB_NY):
    op = op or Upwind9()
    wx = np.array(nx) - 1
    wy = np.array(ny) - 1
    xb = -5.0 + 10.0 * np.concatenate([[0], np.cumsum(wx)]) / wx.sum()
    yb = -5.0 + 10.0 * np.concatenate([[0], np.cumsum(wy)]) / wy.sum()
    xb[-1] = yb[-1] = 5.0
    blocks = []
    ncol, nrow = len(nx), len(ny)
    for r in range(nrow):
        for c in range(ncol):
            b = r * ncol + c
            x, y = warped(xb[c], xb[c + 1], nx[c], yb[r], yb[r + 1], ny[r])
            north = (BC_GRID, b + ncol) if r < nrow - 1 else (BC_VORTEX, 0)
            south = (BC_GRID, b - ncol) if r > 0 else (BC_VORTEX, 0)
            east = (BC_GRID, b + 1) if c < ncol - 1 else (BC_VORTEX, 0)
            west = (BC_GRID, b - 1) if c > 0 else (BC_VORTEX, 0)
            blocks.append(BlockSpec(x, y, op, [north, south, east, west], 0))
    return blocks


def multiblock_dt(blocks) -> float:
    return 0.2 * min(min(1.0 / (b.x.shape[1] - 1), 1.0 / (b.x.shape[0] - 1)) for b in blocks)


# ----- configuration 3: batched ensemble ----------------------------------------------------
# Vortex radius of the ensemble: the reference's own System::init_with_vortex radius
# (euler/src/lib.rs:83-103).  With rstar = 0.5 the strongest draws (eps ~ 1.4, Mach ~ 0.7) are
# under-resolved on the coarsest grids and lose positivity before t = 2 under the reference's
# scheme itself (5 of the 125 draws with side <= 100, Upwind4), where the reference would stop
# on assert!(p > 0.0) (euler/src/lib.rs:642).
ENSEMBLE_RSTAR = 1.0


@dataclass
class Instance:
    x0: float
    y0: float
    eps: float
    mach: float
    side: int
    op_id: int

    @property
    def dt(self) -> float:
        return 0.2 / (self.side - 1)

    @property
    def steps_to_t2(self) -> int:
        return 10 * (self.side - 1)

    @property
    def vortex(self) -> VortexParameters:
        return VortexParameters([Vortice(self.x0, self.y0, ENSEMBLE_RSTAR, self.eps)], mach=self.mach)


def ensemble_instances(n: int = 512, seed: int = 1, first: int = 0) -> list[Instance]:
    """Instances first..first+n-1: six draws each from SplitMix64(seed), in the order
    x0 ~ U[-2,2], y0 ~ U[-2,2], eps ~ U[0.5,1.5], Mach ~ U[0.3,0.7], side ~ U{48..257},
    operator Upwind4 if the last draw < 0.5 else Upwind9."""
    u = uniform01(seed, 6 * n, 6 * first).reshape(n, 6)
    out = []
    for r in u:
        side = 48 + min(int(r[4] * 210.0), 209)
        out.append(Instance(x0=-2.0 + 4.0 * r[0], y0=-2.0 + 4.0 * r[1], eps=0.5 + r[2], mach=0.3 + 0.4 * r[3],
                            side=side, op_id=UPWIND4 if r[5] < 0.5 else UPWIND9))
    return out


def ensemble_blocks(insts: list[Instance]):
    blocks = []
    for i, inst in enumerate(insts):
        x, y = warped(-5.0, 5.0, inst.side, -5.0, 5.0, inst.side)
        blocks.append(BlockSpec(x, y, BY_ID[inst.op_id](), [(BC_VORTEX, 0)] * 4, i))
    return blocks


def ensemble_points(insts) -> int:
    return int(sum(i.side * i.side for i in insts))
