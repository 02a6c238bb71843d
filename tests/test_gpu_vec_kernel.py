"""The compensated-f32 stage kernels of 16-row tiles (one column per thread) and of 32-row tiles
(2 x 2 micro-tiles, paired f32 FMAs, transposed xi arrays, RK operands prefetched into
registers) take every stencil sum in the same order; they differ only where the compiler may
contract a product into the following add.  Their states after several RK4 steps agree to f32
rounding (the bar is 1e-6 relative L2, the f32 unit roundoff being 6e-8) on every operator
family, closure case, partial tile and boundary kind, and the micro-tile kernel meets the f32c
bar against the f64 oracle.
"""
import numpy as np
import pytest
from _helpers import oracle_system, rel_l2

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

BAR = 1e-6


def _run(blocks, ty, steps, ninst=1, per_instance=None, vortex=None, force_trad=False):
    from summationbyparts_b200 import workloads
    from summationbyparts_b200.system import BlockSystem
    g = BlockSystem(blocks, ninst, "f32c", 1.4)
    if per_instance:
        for k, (vx, dt) in enumerate(per_instance):
            g.set_vortex(vx, k)
            g.set_dt(dt, k)
    else:
        g.set_vortex(vortex or workloads.STANDARD_VORTEX)
        g.set_dt(0.002)
    if force_trad:
        g.set_force_trad(True)
    g.init_vortex(0.0)
    g.set_tiles(ty, 32)
    g.advance(steps)
    out = np.concatenate([g.state(b).ravel() for b in range(len(blocks))])
    g.close()
    return out


def _both(*args, **kw):
    a = _run(*args[:1], 16, *args[1:], **kw)
    b = _run(*args[:1], 32, *args[1:], **kw)
    assert np.all(np.isfinite(b))
    return a, b


def test_ensemble_upwind4_upwind9():
    """Ragged square blocks (sides not multiples of 4 or 32) of both operator groups."""
    from summationbyparts_b200 import workloads
    insts = [i for i in workloads.ensemble_instances(80, seed=1) if i.side <= 150][:8]
    assert {i.op_id for i in insts} == {workloads.UPWIND4, workloads.UPWIND9}
    assert any(i.side % 4 for i in insts)
    blocks = workloads.ensemble_blocks(insts)
    a, b = _both(blocks, 12, ninst=len(insts), per_instance=[(i.vortex, i.dt) for i in insts])
    assert rel_l2(b, a) <= BAR


def test_multiblock_grid_interfaces():
    from summationbyparts_b200 import workloads
    a, b = _both(workloads.multiblock(), 10)
    assert rel_l2(b, a) <= BAR


@pytest.mark.parametrize("name", ["upwind4h2", "upwind9h2", "sbp4", "sbp8", "pair"])
def test_operator_families(name):
    """Every operator the stage kernels are built for, on a warped block whose width leaves a
    partial column group (nx = 71) and a short last tile row (ny = 45)."""
    from summationbyparts_b200 import operators, workloads
    from summationbyparts_b200.system import BC_VORTEX, BlockSpec
    op = operators.Pair(operators.Upwind9h2(), operators.Upwind9()) if name == "pair" else operators.BY_NAME[name]()
    x, y = workloads.warped(-5.0, 5.0, 71, -5.0, 5.0, 45)
    a, b = _both([BlockSpec(x, y, op, [(BC_VORTEX, 0)] * 4, 0)], 8)
    assert rel_l2(b, a) <= BAR


def test_force_trad():
    from summationbyparts_b200 import operators, workloads
    from summationbyparts_b200.system import BC_VORTEX, BlockSpec
    x, y = workloads.warped(-5.0, 5.0, 66, -5.0, 5.0, 70)
    a, b = _both([BlockSpec(x, y, operators.Upwind9(), [(BC_VORTEX, 0)] * 4, 0)], 8, force_trad=True)
    assert rel_l2(b, a) <= BAR


def test_micro_tile_against_f64_oracle(orc):
    from summationbyparts_b200 import workloads
    from summationbyparts_b200.system import BlockSystem
    cfg = workloads.Config0()
    blocks = cfg.blocks()
    o = oracle_system(orc, blocks, workloads.STANDARD_VORTEX)
    o.init_vortex(0.0)
    g = BlockSystem(blocks, 1, "f32c", 1.4)
    g.set_vortex(workloads.STANDARD_VORTEX)
    g.set_tiles(32, 32)
    g.set_state(0, o.state(0))
    g.set_dt(cfg.dt)
    g.advance(cfg.steps)
    o.advance(cfg.steps, cfg.dt)
    assert rel_l2(g.state(0), o.state(0)) <= 1e-5
    g.close()


@pytest.mark.parametrize("op_name,sizes", [
    ("upwind9", [(16, 17), (20, 33), (39, 40), (41, 64), (65, 71)]),
    ("upwind4", [(8, 9), (12, 35), (36, 37), (64, 33)]),
])
def test_closure_tile_split(op_name, sizes):
    """Lines whose closure rows would straddle a tile boundary or share a tile with the other
    end's closure (lengths 2 M .. 2 tiles, multiples of 32 and 32 k + 1 .. 32 k + M - 1): the tile
    lists move the boundary so one tile holds each end, and both kernels still agree."""
    from summationbyparts_b200 import operators, workloads
    from summationbyparts_b200.system import BC_VORTEX, BlockSpec
    op = operators.BY_NAME[op_name]()
    blocks = []
    for k, (nx, ny) in enumerate(sizes):
        x, y = workloads.warped(-5.0, 5.0, nx, -5.0, 5.0, ny)
        blocks.append(BlockSpec(x, y, op, [(BC_VORTEX, 0)] * 4, k))
    vortex = workloads.STANDARD_VORTEX
    a, b = _both(blocks, 6, ninst=len(sizes), per_instance=[(vortex, 0.002)] * len(sizes))
    assert rel_l2(b, a) <= BAR
