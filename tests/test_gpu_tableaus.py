"""GPU parity of the general explicit Runge-Kutta path (sbp_system_advance_tableau: every
tableau of utils/integrate/src/lib.rs) and of euler::System::advance_adaptive against the
oracle.  Bar: 1e-12 relative L2 (f64), as the fused RK4 path."""
import numpy as np
import pytest
from _helpers import oracle_system, rel_l2

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

PARITY = 1e-12
NAMES = ["rk4", "rk4_38", "euler", "midpoint", "rk6", "fehlberg", "bogacki_shampine"]


def _two_blocks():
    """Two Upwind4 blocks side by side (Grid interface), vortex data on the outer edges."""
    from summationbyparts_b200 import workloads
    from summationbyparts_b200.operators import Upwind4
    from summationbyparts_b200.system import BC_GRID, BC_VORTEX, BlockSpec
    v = (BC_VORTEX, 0)
    xa, ya = workloads.warped(-5.0, 0.0, 33, -5.0, 5.0, 41)
    xb, yb = workloads.warped(0.0, 5.0, 33, -5.0, 5.0, 41)
    a = BlockSpec(xa, ya, Upwind4(), [v, v, (BC_GRID, 1), v], 0)
    b = BlockSpec(xb, yb, Upwind4(), [v, v, v, (BC_GRID, 0)], 0)
    return [a, b]


@pytest.mark.parametrize("tableau", range(7))
def test_tableau_matches_oracle(orc, tableau):
    from summationbyparts_b200 import workloads
    from summationbyparts_b200.system import BlockSystem
    blocks = _two_blocks()
    dt = 0.2 / 40
    o = oracle_system(orc, blocks, workloads.STANDARD_VORTEX)
    o.init_vortex(0.0)
    g = BlockSystem(blocks, 1, "f64", 1.4)
    g.set_vortex(workloads.STANDARD_VORTEX)
    for b in range(2):
        g.set_state(b, o.state(b))
    g.set_dt(dt)
    g.advance_tableau(NAMES[tableau], 6)
    o.advance_tableau(tableau, 6, dt)
    for b in range(2):
        assert rel_l2(g.state(b), o.state(b)) <= PARITY, (tableau, b)
    assert g.time(0) == o.time
    g.close()


def test_rk4_tableau_equals_fused_path():
    """The general path with the RK4 tableau and the fused RK4 kernel give the same states."""
    from summationbyparts_b200 import workloads
    from summationbyparts_b200.system import BlockSystem
    out = []
    for mode in ("fused", "tableau"):
        g = BlockSystem(_two_blocks(), 1, "f64", 1.4)
        g.set_vortex(workloads.STANDARD_VORTEX)
        g.init_vortex(0.0)
        g.set_dt(0.2 / 40)
        if mode == "fused":
            g.advance(5)
        else:
            g.advance_tableau("rk4", 5)
        out.append(np.concatenate([g.state(b).ravel() for b in range(2)]))
        g.close()
    assert rel_l2(out[1], out[0]) <= PARITY


def test_advance_adaptive_matches_oracle(orc):
    from summationbyparts_b200 import workloads
    from summationbyparts_b200.operators import Upwind4
    from summationbyparts_b200.system import BC_THIS, BlockSpec, BlockSystem
    x, y = workloads.cartesian(-5.0, 5.0, 40, -5.0, 5.0, 40)
    blk = [BlockSpec(x, y, Upwind4(), [(BC_THIS, 0)] * 4, 0)]
    o = oracle_system(orc, blk, workloads.STANDARD_VORTEX)
    o.init_vortex(0.0)
    g = BlockSystem(blk, 1, "f64", 1.4)
    g.set_vortex(workloads.STANDARD_VORTEX)
    g.set_state(0, o.state(0))
    guess_g = g.advance_adaptive(0.02, 0.004, 2e-3)
    guess_o = o.advance_adaptive(0.02, 0.004, 2e-3)
    assert guess_g == guess_o
    assert rel_l2(g.state(0), o.state(0)) <= PARITY
    g.close()


def test_general_tableaus_need_f64():
    from summationbyparts_b200 import _capi, workloads
    from summationbyparts_b200.system import BlockSystem
    g = BlockSystem(_two_blocks(), 1, "f32c", 1.4)
    g.set_vortex(workloads.STANDARD_VORTEX)
    g.init_vortex(0.0)
    with pytest.raises(_capi.SbpError) as e:
        g.advance_tableau("rk6", 1)
    assert e.value.status == 3
    g.close()
