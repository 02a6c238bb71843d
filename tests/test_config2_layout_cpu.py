"""Configuration 2 names six blocks of 101x51, 81x81, 65x129, 49x97, 121x41 and 73x73 points
(nx x ny) tiling [-5, 5]^2 with interface SATs.  This test is the argument that no such layout
exists under the reference's block couplings, so the multi-block workload uses a conforming
2 x 3 layout of other sizes instead (summationbyparts_b200/workloads.py `multiblock`).

A block side lies on the outer boundary or is covered by neighbours, and the reference couples
it in one of three ways (euler/src/lib.rs:804-930):
  * Grid(g): one neighbour whose opposite side has the same extent and the same point count
    (SAT_characteristic asserts equal shapes, euler/src/lib.rs:1163);
  * Interpolate(g, op): one neighbour over the same extent with fine = 2 coarse - 1 points
    (Interpolation4/8/9, sbp/src/operators/interpolation/interpolation4.rs:75) or
    fine = 2 (coarse - 1) (Interpolation9h2);
  * MultiGrid(segments): the side's points are runs of neighbours' edge points laid end to end
    (euler/src/lib.rs:829-846), so along the side the point spacing equals every neighbour's.
The blocks are images of axis-aligned rectangles of the (xi, eta) square under one smooth warp,
so a layout is a rectangle dissection of the square.  A dissection into 6 rooms has at most 5
maximal internal segments, so relabelling the distinct segment coordinates by their order puts
every combinatorial layout on an a x b lattice with (a - 1) + (b - 1) <= 5.  The test enumerates
all tilings of such lattices by 6 rectangles, assigns the six blocks in all 720 ways, rejects
full-side contacts that are neither Grid nor Interpolate, and checks the remaining equal-spacing
equations (widths / (nx - 1), heights / (ny - 1)) for a solution with increasing coordinates by
linear programming.  None exists.  The same search finds the conforming 2 x 3 layout of the
multi-block workload, which validates the checker.
"""
import itertools

import numpy as np
import pytest

CONFIG2 = {"A": (101, 51), "B": (81, 81), "C": (65, 129), "D": (49, 97), "E": (121, 41), "F": (73, 73)}
CONFORMING = {"A": (101, 51), "B": (81, 51), "C": (101, 81), "D": (81, 81), "E": (101, 73), "F": (81, 73)}


def pair_couples(a: int, b: int) -> bool:
    """Grid (equal counts) or Interpolate (2:1) between two full sides of a and b points."""
    f, c = max(a, b), min(a, b)
    return a == b or f == 2 * c - 1 or f == 2 * (c - 1)


def lattice_tilings(a: int, b: int, k: int) -> list:
    """Tilings of an a (columns) x b (rows) lattice by exactly k rectangles (c0, c1, r0, r1)
    that use every internal lattice line."""
    grid = [[-1] * a for _ in range(b)]
    rects, out = [], []

    def rec():
        empty = next(((r, c) for r in range(b) for c in range(a) if grid[r][c] < 0), None)
        if empty is None:
            if len(rects) == k:
                xs = {x for rc in rects for x in rc[:2]}
                ys = {y for rc in rects for y in rc[2:]}
                if len(xs) == a + 1 and len(ys) == b + 1:
                    out.append(list(rects))
            return
        if len(rects) >= k:
            return
        r0, c0 = empty
        wmax = 0
        while c0 + wmax < a and grid[r0][c0 + wmax] < 0:
            wmax += 1
        for w in range(1, wmax + 1):
            for h in range(1, b - r0 + 1):
                if any(grid[r0 + h - 1][c0 + dc] >= 0 for dc in range(w)):
                    break
                for dr in range(h):
                    for dc in range(w):
                        grid[r0 + dr][c0 + dc] = len(rects)
                rects.append((c0, c0 + w, r0, r0 + h))
                rec()
                rects.pop()
                for dr in range(h):
                    for dc in range(w):
                        grid[r0 + dr][c0 + dc] = -1

    rec()
    return out


def layout_feasible(a: int, b: int, rects: list, sizes: list) -> bool:
    """Whether the labelled tiling admits coordinates 0 = X_0 < ... < X_a = 10 and
    0 = Y_0 < ... < Y_b = 10 satisfying every coupling rule (module docstring)."""
    from scipy.optimize import linprog
    nv = (a - 1) + (b - 1)

    def coord(i, last, base):  # (coefficients, constant) of lattice line i
        v = np.zeros(nv)
        if i == last:
            return v, 10.0
        if i > 0:
            v[base + i - 1] = 1.0
        return v, 0.0

    def extent(lo, hi, last, base):
        v1, k1 = coord(hi, last, base)
        v0, k0 = coord(lo, last, base)
        return v1 - v0, k1 - k0

    a_eq, b_eq = [], []
    for i, j in itertools.permutations(range(len(rects)), 2):
        ci0, ci1, ri0, ri1 = rects[i]
        cj0, cj1, rj0, rj1 = rects[j]
        (nxi, nyi), (nxj, nyj) = sizes[i], sizes[j]
        if ri1 == rj0 and min(ci1, cj1) > max(ci0, cj0):  # j north of i
            if (ci0, ci1) == (cj0, cj1):
                if not pair_couples(nxi, nxj):
                    return False
                continue
            (wi, ki), (wj, kj) = extent(ci0, ci1, a, 0), extent(cj0, cj1, a, 0)
            a_eq.append(wi / (nxi - 1) - wj / (nxj - 1))
            b_eq.append(kj / (nxj - 1) - ki / (nxi - 1))
        if ci1 == cj0 and min(ri1, rj1) > max(ri0, rj0):  # j east of i
            if (ri0, ri1) == (rj0, rj1):
                if not pair_couples(nyi, nyj):
                    return False
                continue
            (hi_, ki), (hj, kj) = extent(ri0, ri1, b, a - 1), extent(rj0, rj1, b, a - 1)
            a_eq.append(hi_ / (nyi - 1) - hj / (nyj - 1))
            b_eq.append(kj / (nyj - 1) - ki / (nyi - 1))
    if nv == 0:
        return all(abs(v) < 1e-12 for v in b_eq)
    a_ub, b_ub = [], []
    for n_, base in ((a, 0), (b, a - 1)):
        for k in range(n_):
            v, c = extent(k, k + 1, n_, base)
            a_ub.append(-v)
            b_ub.append(c - 1e-3)
    res = linprog(np.zeros(nv), A_ub=np.array(a_ub), b_ub=np.array(b_ub),
                  A_eq=np.array(a_eq) if a_eq else None, b_eq=np.array(b_eq) if b_eq else None,
                  bounds=[(None, None)] * nv, method="highs")
    return res.status == 0


def count_layouts(blocks: dict, first_only: bool = False) -> tuple[int, int]:
    tilings = feasible = 0
    for a in range(1, 7):
        for b in range(1, 7):
            if (a - 1) + (b - 1) > 5:
                continue
            for rects in lattice_tilings(a, b, 6):
                tilings += 1
                for perm in itertools.permutations(blocks.values()):
                    feasible += layout_feasible(a, b, rects, list(perm))
                    if first_only and feasible:
                        return tilings, feasible
    return tilings, feasible


def test_config2_sizes_admit_no_layout():
    pytest.importorskip("scipy")
    tilings, feasible = count_layouts(CONFIG2)
    assert tilings == 834
    assert feasible == 0


def test_checker_finds_the_conforming_layout():
    pytest.importorskip("scipy")
    _, feasible = count_layouts(CONFORMING, first_only=True)
    assert feasible > 0


def test_workload_layout_is_the_conforming_one():
    from summationbyparts_b200 import workloads
    sizes = sorted((b.x.shape[1], b.x.shape[0]) for b in workloads.multiblock())
    assert sizes == sorted(CONFORMING.values())
