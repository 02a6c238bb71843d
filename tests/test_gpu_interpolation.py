"""GPU parity of the 2:1 interface interpolation operators (sbp/src/operators/interpolation*.rs)
and of the Interpolate / MultiGrid block boundaries (euler/src/lib.rs:816-846) against the oracle.

Bars: sbp_interpolate bit-identical to the oracle in f64 and f32; systems with these
boundaries <= 1e-12 relative L2 (f64), as the other Euler parity tests."""
import ctypes

import numpy as np
import pytest
from _helpers import oracle_system, rel_l2

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

PARITY = 1e-12


def _lines(op, f2c, nc, nbatch, dtype, seed):
    odd = op != 3
    nf = 2 * nc - 1 if odd else 2 * (nc - 1)
    nin, nout = (nf, nc) if f2c else (nc, nf)
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1.0, 1.0, (nbatch, nin + 3)).astype(dtype)  # stride nin + 3
    return x, nin, nout


@pytest.mark.parametrize("op", [0, 1, 2, 3])
@pytest.mark.parametrize("f2c", [True, False])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_interpolate_bitwise(orc, op, f2c, dtype):
    from summationbyparts_b200 import _capi
    for nc in (16, 37, 101):
        x, nin, nout = _lines(op, f2c, nc, 3, dtype, nc + op)
        d_in = torch.from_numpy(x).cuda()
        d_out = torch.zeros((3, nout + 5), dtype=d_in.dtype, device="cuda")
        _capi.check(_capi.lib.sbp_interpolate(op, int(f2c), _capi.F64 if dtype == np.float64 else _capi.F32,
                                              ctypes.c_void_p(d_in.data_ptr()), ctypes.c_void_p(d_out.data_ptr()),
                                              nin, nout, 3, nin + 3, nout + 5, None))
        torch.cuda.synchronize()
        out = d_out.cpu().numpy()
        for b in range(3):
            ref = orc.interpolate(op, f2c, x[b, :nin], dtype)
            assert out[b, :nout].tobytes() == ref.tobytes(), (nc, b)
            assert np.all(out[b, nout:] == 0)


def _interpolation_example():
    """The reference's multigrid/examples/interpolation.json: grid0 50 x 25 on [-5,5] x [0,5]
    above grid1 99 x 50 on [-5,5] x [-5,0], Upwind9, 2:1 interface through Interpolation9,
    vortex data on the other edges."""
    from summationbyparts_b200 import workloads
    from summationbyparts_b200.operators import Upwind9
    from summationbyparts_b200.system import BC_INTERPOLATE, BC_VORTEX, BlockSpec
    x0, y0 = workloads.cartesian(-5.0, 5.0, 50, 0.0, 5.0, 25)
    x1, y1 = workloads.cartesian(-5.0, 5.0, 99, -5.0, 0.0, 50)
    v = (BC_VORTEX, 0)
    b0 = BlockSpec(x0, y0, Upwind9(), [v, (BC_INTERPOLATE, 1, 2), v, v], 0)
    b1 = BlockSpec(x1, y1, Upwind9(), [(BC_INTERPOLATE, 0, 2), v, v, v], 0)
    return [b0, b1]


def _run_pair(orc, blocks, steps, dt):
    from summationbyparts_b200 import workloads
    from summationbyparts_b200.system import BlockSystem
    o = oracle_system(orc, blocks, workloads.STANDARD_VORTEX)
    o.init_vortex(0.0)
    g = BlockSystem(blocks, 1, "f64", 1.4)
    g.set_vortex(workloads.STANDARD_VORTEX)
    for b in range(len(blocks)):
        g.set_state(b, o.state(b))
    g.set_dt(dt)
    g.advance(steps)
    o.advance(steps, dt)
    out = [rel_l2(g.state(b), o.state(b)) for b in range(len(blocks))]
    g.close()
    return out


def test_interpolation_interface_system(orc):
    blocks = _interpolation_example()
    errs = _run_pair(orc, blocks, 30, 0.2 / 98)
    assert max(errs) <= PARITY, errs


def test_multigrid_boundary_system(orc):
    """A T-junction: block A (41 x 21) below blocks B and C (21 x 21 each); A's north edge is the
    MultiGrid concatenation of B's and C's south edges, B's and C's south edges are MultiGrid
    slices of A's north edge."""
    from summationbyparts_b200 import workloads
    from summationbyparts_b200.operators import Upwind4
    from summationbyparts_b200.system import BC_MULTIGRID, BC_VORTEX, BlockSpec
    v = (BC_VORTEX, 0)
    xa, ya = workloads.cartesian(-5.0, 5.0, 41, -5.0, 0.0, 21)
    xb, yb = workloads.cartesian(-5.0, 0.0, 21, 0.0, 5.0, 21)
    xc, yc = workloads.cartesian(0.0, 5.0, 21, 0.0, 5.0, 21)
    a = BlockSpec(xa, ya, Upwind4(), [(BC_MULTIGRID, [(1, 0, 21), (2, 0, 21)]), v, v, v], 0)
    b = BlockSpec(xb, yb, Upwind4(), [v, (BC_MULTIGRID, [(0, 0, 21)]), v, v], 0)
    c = BlockSpec(xc, yc, Upwind4(), [v, (BC_MULTIGRID, [(0, 20, 41)]), v, v], 0)
    errs = _run_pair(orc, [a, b, c], 10, 0.2 / 40)
    assert max(errs) <= PARITY, errs
