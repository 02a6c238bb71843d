"""The multigrid driver (summationbyparts_b200/main.py) end to end on the GPU: a configuration
file in the reference's format (a 2:1 interpolation interface like the reference's
examples/interpolation.json, shortened in time) is run through the command-line entry point, and
its reported error is compared with the oracle running the same parsed configuration with the
same dt and step count."""
import json

import numpy as np
import pytest
from _helpers import oracle_system

pytestmark = pytest.mark.gpu

CONFIG = """{
    // two grids coupled through Interpolation9 (fine2coarse into grid0, coarse2fine into grid1)
    grids: {
        default: { operators: { xi: "upwind9", eta: "upwind9" } },
        grid0: {
            x: { linspace: { start: -5, end: 5, steps: 50 } },
            y: { linspace: { start: 0, end: 5, steps: 25 } },
            boundary_conditions: { south: { interpolate: { neighbour: "grid1", operator: "9" } } },
        },
        grid1: {
            x: { linspace: { start: -5, end: 5, steps: 99 } },
            y: { linspace: { start: -5, end: 0, steps: 50 } },
            boundary_conditions: { north: { interpolate: { neighbour: "grid0", operator: "9" } } },
        },
    },
    integration_time: 0.1,
    initial_conditions: { vortex: { vortices: [{ x0: -1.0, y0: 0.0, rstar: 0.5, eps: 1.0 }], mach: 0.5 } },
    boundary_conditions: "initial_conditions",
}"""


def test_driver_matches_oracle(orc, tmp_path, capsys):
    from summationbyparts_b200 import config, hdf5, main, multigrid
    from summationbyparts_b200.system import BlockSpec
    path = tmp_path / "interp.json5"
    path.write_text(CONFIG)
    out = tmp_path / "run.hdf"
    assert main.main([str(path), "-o", str(out), "--error", "--timings", "--output-json"]) == 0
    info = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert info["filename"] == str(out) and "secs" in info["time_elapsed"]
    snaps = hdf5.read_flat(str(out))
    assert snaps["grid1/rho"].shape == (2, 50, 99)

    rt = config.into_runtime(config.loads(CONFIG))
    specs = [BlockSpec(g.x, g.y, g.op, [multigrid._bc(s) for s in (g.north, g.south, g.east, g.west)], 0)
             for g in rt.grids]
    o = oracle_system(orc, specs, rt.initial_vortex)
    o.init_vortex(0.0)
    dt = o.max_dt()
    ntime = int(round(rt.integration_time / dt))
    np.testing.assert_array_equal(snaps["t"], [0, ntime])  # step numbers of the outputs
    np.testing.assert_array_equal(snaps["grid1/t"], snaps["t"])  # the soft link t -> /t
    o.advance(ntime, dt)
    assert abs(info["error"] - o.error()) <= 1e-10 * o.error()
    assert np.max(np.abs(snaps["grid0/rho"][1] - o.state(0)[0])) <= 1e-12 * np.max(np.abs(o.state(0)[0]))


EXPR_CONFIG = """{
    // one periodic grid, initial conditions given as expressions (pressure form)
    grids: {
        grid: {
            operators: { xi: "upwind9", eta: "upwind9" },
            x: { linspace: { start: 0, end: 2, steps: 41 } },
            y: { linspace: { start: 0, end: 2, steps: 37 } },
            boundary_conditions: { north: "this", south: "this", east: "this", west: "this" },
        },
    },
    integration_time: 0.2,
    initial_conditions: {
        expressions: {
            globals: "ua = 0.8; va = -0.3; pa = 1.5;",
            rho: "1 + 0.25*math::sin(PI*((x - t*ua) + (y - t*va)))",
            u: "ua",
            v: "va",
            p: "pa",
        },
    },
    gamma: 1.4,
}"""


def test_driver_expression_initial_conditions(orc, tmp_path, capsys):
    """Expression initial conditions through the command-line entry point: the state matches the
    oracle started from the same evaluated fields, and --error is the h2 error against the
    expressions at the final time (an advected density wave, exact on a periodic domain)."""
    from summationbyparts_b200 import config, hdf5, main, multigrid
    from summationbyparts_b200.system import BlockSpec
    path = tmp_path / "wave.json5"
    path.write_text(EXPR_CONFIG)
    out = tmp_path / "run.hdf"
    assert main.main([str(path), "-o", str(out), "--error", "--output-json"]) == 0
    info = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    snaps = hdf5.read_flat(str(out))

    rt = config.into_runtime(config.loads(EXPR_CONFIG))
    g = rt.grids[0]
    specs = [BlockSpec(g.x, g.y, g.op, [multigrid._bc(s) for s in (g.north, g.south, g.east, g.west)], 0)]
    from summationbyparts_b200.system import VortexParameters
    o = oracle_system(orc, specs, VortexParameters([], mach=0.5))  # no vortex sides
    q0 = rt.initial.evaluate(0.0, g.x, g.y)
    o.set_state(0, q0)
    np.testing.assert_array_equal(snaps["grid/rho"][0], q0[0])
    dt = o.max_dt()
    ntime = int(round(rt.integration_time / dt))
    o.advance(ntime, dt)
    qo = o.state(0)
    assert np.max(np.abs(snaps["grid/rho"][1] - qo[0])) <= 1e-12 * np.max(np.abs(qo[0]))
    t = ntime * dt
    err = orc.h2_err(g.op.ids[0], g.op.ids[1], qo, rt.initial.evaluate(t, g.x, g.y))
    assert abs(info["error"] - err) <= 1e-9 * err
