"""Expression boundaries (SBP_BC_EVAL, the reference's BoundaryCharacteristic::Eval with the
multigrid driver's evalexpr evaluator): expressions that restate the vortex of
euler/src/vortex.rs give, side by side with the built-in vortex boundary (SBP_BC_VORTEX), the same
states after several RK4 steps -- the boundary data are evaluated on the device at every stage
time, only their constants are folded in another order (bar 1e-12 relative L2 in f64, f32
rounding in the compensated form).  Programs that break the interpreter's limits are refused, a
system with expression sides does not step before it has its programs, and the driver runs a
configuration whose unspecified sides take the expression boundaries."""
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

VORTEX_EXPR = {
    "globals": "x0 = -1.0; y0 = 0.2; rs = 0.5; eps = 1.0; m = 0.5; pinf = 1/(GAMMA*m*m)",
    "rho": "dx = (x - x0) - t; dy = y - y0; f = (1 - (dx*dx + dy*dy))/(rs*rs); "
           "math::pow(1 - eps*eps*(GAMMA - 1)*m*m/(8*PI*PI*pinf*rs*rs)*math::exp(f), 1/(GAMMA - 1))",
    "u": "dx = (x - x0) - t; dy = y - y0; f = (1 - (dx*dx + dy*dy))/(rs*rs); "
         "1 - eps*dy/(2*PI*math::sqrt(pinf)*rs*rs)*math::exp(f/2)",
    "v": "dx = (x - x0) - t; dy = y - y0; f = (1 - (dx*dx + dy*dy))/(rs*rs); "
         "eps*dx/(2*PI*math::sqrt(pinf)*rs*rs)*math::exp(f/2)",
    "p": "math::pow(rho, GAMMA)*pinf",
}


def _vortex():
    from summationbyparts_b200.system import Vortice, VortexParameters
    return VortexParameters([Vortice(-1.0, 0.2, 0.5, 1.0)], mach=0.5)


def _run(kind, precision, steps=12):
    from summationbyparts_b200 import expr, operators, workloads
    from summationbyparts_b200.system import BC_EVAL, BC_VORTEX, BlockSpec, BlockSystem
    x, y = workloads.warped(-5.0, 5.0, 57, -5.0, 5.0, 49)
    g = BlockSystem([BlockSpec(x, y, operators.Upwind9(), [(kind, 0)] * 4, 0)], 1, precision, 1.4)
    g.set_vortex(_vortex())
    g.init_vortex(0.0)
    if kind == BC_EVAL:
        g.set_eval(expr.Expressions.from_config(VORTEX_EXPR, 1.4))
    g.set_dt(0.02)
    g.advance(steps)
    q = g.state(0)
    g.close()
    return q


@pytest.mark.parametrize("precision,bar", [("f64", 1e-12), ("f32c", 1e-7)])
def test_expression_vortex_matches_builtin_vortex(precision, bar):
    from summationbyparts_b200.system import BC_EVAL, BC_VORTEX
    a = _run(BC_VORTEX, precision)
    b = _run(BC_EVAL, precision)
    assert np.all(np.isfinite(b))
    rel = np.linalg.norm(b - a) / np.linalg.norm(a)
    assert rel <= bar, rel


def test_programs_are_validated_and_required():
    from summationbyparts_b200 import _capi, operators, workloads
    from summationbyparts_b200._capi import SbpError
    from summationbyparts_b200.system import BC_EVAL, BlockSpec, BlockSystem
    x, y = workloads.warped(-5.0, 5.0, 41, -5.0, 5.0, 41)
    g = BlockSystem([BlockSpec(x, y, operators.Upwind4(), [(BC_EVAL, 0)] * 4, 0)], 1, "f64", 1.4)
    g.set_vortex(_vortex())
    g.init_vortex(0.0)
    g.set_dt(0.01)
    with pytest.raises(SbpError, match="sbp_system_set_eval"):
        g.advance(1)
    import ctypes
    bad = [[5], [1, 0], [1, 0], [1, 0]]  # program 0: an addition (opcode 5) on an empty stack
    arrs = [np.array(c, dtype=np.int32) for c in bad]
    ptrs = (ctypes.POINTER(ctypes.c_int32) * 4)(*[a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)) for a in arrs])
    lens = (ctypes.c_int32 * 4)(*[len(c) for c in bad])
    consts = np.array([1.0])
    st = _capi.lib.sbp_system_set_eval(g.h, 0, ptrs, lens, consts.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 1)
    assert st == 1 and b"underflow" in _capi.lib.sbp_last_error()
    # program 0 reads local slot 2 (EV_LOAD = 3) that nothing has written
    unread = [[3, 2], [1, 0], [1, 0], [1, 0]]
    arrs = [np.array(c, dtype=np.int32) for c in unread]
    ptrs = (ctypes.POINTER(ctypes.c_int32) * 4)(*[a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)) for a in arrs])
    lens = (ctypes.c_int32 * 4)(*[len(c) for c in unread])
    st = _capi.lib.sbp_system_set_eval(g.h, 0, ptrs, lens, consts.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 1)
    assert st == 1 and b"read before it is written" in _capi.lib.sbp_last_error()
    g.close()


EVAL_CONFIG = """{
    grids: {
        grid: {
            operators: { xi: "upwind9", eta: "upwind9" },
            x: { linspace: { start: -5, end: 5, steps: 51 } },
            y: { linspace: { start: -5, end: 5, steps: 45 } },
        },
    },
    integration_time: 0.1,
    initial_conditions: { expressions: %s },
    boundary_conditions: "initial_conditions",
}""" % json.dumps(VORTEX_EXPR)

VORTEX_CONFIG = """{
    grids: {
        grid: {
            operators: { xi: "upwind9", eta: "upwind9" },
            x: { linspace: { start: -5, end: 5, steps: 51 } },
            y: { linspace: { start: -5, end: 5, steps: 45 } },
        },
    },
    integration_time: 0.1,
    initial_conditions: { vortex: { vortices: [{ x0: -1.0, y0: 0.2, rstar: 0.5, eps: 1.0 }], mach: 0.5 } },
    boundary_conditions: "initial_conditions",
}"""


def test_driver_expression_boundaries(tmp_path, capsys):
    """The same vortex as expressions (initial and boundary conditions) and as the built-in vortex:
    same final state and the same --error through the command-line entry point."""
    from summationbyparts_b200 import hdf5, main
    res = []
    for name, cfg in (("expr", EVAL_CONFIG), ("vortex", VORTEX_CONFIG)):
        path = tmp_path / f"{name}.json5"
        path.write_text(cfg)
        out = tmp_path / f"{name}.hdf"
        assert main.main([str(path), "-o", str(out), "--error", "--output-json"]) == 0
        info = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
        snaps = hdf5.read_flat(str(tmp_path / f"{name}.hdf"))
        res.append((info["error"], snaps["grid/rho"][-1]))
    (e1, r1), (e2, r2) = res
    assert np.max(np.abs(r1 - r2)) <= 1e-12 * np.max(np.abs(r2))
    assert abs(e1 - e2) <= 1e-8 * e2
