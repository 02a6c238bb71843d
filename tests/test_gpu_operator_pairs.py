"""GPU parity for operator pairs from two families.

The reference composes a block's operator from any two of its six operators, one per direction
(the `(eta_op, xi_op)` tuple, sbp/src/operators.rs:115-150; the multigrid input picks xi and eta
independently, multigrid/src/parsing.rs:153-164).  The tuple has an upwind form only when both
operators have one, so every pair with SBP4 or SBP8 on either side runs RHS_trad.

Bars: f64 <= 1e-12 relative L2 against the oracle (the reference's arithmetic); compensated f32
<= 1e-5 relative L2 against the f64 oracle, on both tile shapes (16-row stage kernel, 32-row
micro-tile kernel).
"""
import json

import numpy as np
import pytest
from _helpers import oracle_system, physical_state, rel_l2

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

NAMES = ["Upwind4", "Upwind4h2", "Upwind9", "Upwind9h2", "SBP4", "SBP8"]
FAMILY = {"Upwind4": 0, "Upwind4h2": 0, "Upwind9": 1, "Upwind9h2": 1, "SBP4": 2, "SBP8": 3}
CROSS = [(x, e) for x in NAMES for e in NAMES if FAMILY[x] != FAMILY[e]]


def pair(xi_name, eta_name):
    from summationbyparts_b200 import operators
    return operators.Pair(getattr(operators, eta_name)(), getattr(operators, xi_name)())


def test_every_pair_is_built():
    """All 36 (xi, eta) combinations create a system (no SBP_ERR_UNSUPPORTED)."""
    from summationbyparts_b200 import workloads
    from summationbyparts_b200.system import BlockSpec, BlockSystem
    x, y = workloads.warped(-5.0, 5.0, 40, -5.0, 5.0, 36)
    for prec in ("f64", "f32c"):
        for xi_name in NAMES:
            for eta_name in NAMES:
                s = BlockSystem([BlockSpec(x, y, pair(xi_name, eta_name), [(0, 0)] * 4, 0)], 1, prec, 1.4)
                s.close()


@pytest.mark.parametrize("xi_name,eta_name", CROSS)
def test_one_step_periodic_cross_pair(orc, xi_name, eta_name):
    """One RK4 step with periodic (`This`) sides from a perturbed vortex, f64."""
    from summationbyparts_b200 import workloads
    from summationbyparts_b200.system import BlockSpec, BlockSystem
    x, y = workloads.warped(-5.0, 5.0, 45, -5.0, 5.0, 38)
    blocks = [BlockSpec(x, y, pair(xi_name, eta_name), [(0, 0)] * 4, 0)]
    q0 = physical_state(x, y)
    g = BlockSystem(blocks, 1, "f64", 1.4)
    g.set_vortex(workloads.STANDARD_VORTEX)
    g.set_state(0, q0)
    g.set_dt(0.01)
    g.advance(1)
    o = oracle_system(orc, blocks, workloads.STANDARD_VORTEX)
    o.set_state(0, q0)
    o.advance(1, 0.01)
    a, b = g.state(0), o.state(0)
    g.close()
    assert rel_l2(a, b) <= 1e-12
    assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()


NAMED = [("Upwind9", "SBP8"), ("Upwind4", "Upwind9"), ("SBP4", "Upwind4h2"), ("SBP8", "SBP4"),
         ("Upwind9h2", "Upwind4")]


@pytest.mark.parametrize("xi_name,eta_name", NAMED)
@pytest.mark.parametrize("prec,ty", [("f64", 16), ("f64", 32), ("f32c", 16), ("f32c", 32)])
def test_vortex_block_cross_pair(orc, xi_name, eta_name, prec, ty):
    """A curvilinear block with vortex SATs on every side, 40 RK4 steps."""
    from summationbyparts_b200 import workloads
    from summationbyparts_b200.system import BlockSpec, BlockSystem
    x, y = workloads.warped(-5.0, 5.0, 61, -5.0, 5.0, 53)
    vort = [(workloads.BC_VORTEX, 0)] * 4
    blocks = [BlockSpec(x, y, pair(xi_name, eta_name), vort, 0)]
    o = oracle_system(orc, blocks, workloads.STANDARD_VORTEX)
    o.init_vortex(0.0)
    g = BlockSystem(blocks, 1, prec, 1.4)
    g.set_vortex(workloads.STANDARD_VORTEX)
    g.set_tiles(ty, 32)
    g.set_state(0, o.state(0))
    dt = 0.2 / 60.0
    g.set_dt(dt)
    g.advance(40)
    o.advance(40, dt)
    a, b = g.state(0), o.state(0)
    g.close()
    assert rel_l2(a, b) <= (1e-12 if prec == "f64" else 1e-5)


# The layout of the reference's multigrid/examples/mix_operators.json (four blocks, Upwind9 and
# Upwind9h2 operators, 9 and 9h2 interpolation interfaces), with two blocks given operators of
# other families: grid2 runs SBP8 along eta, grid3 Upwind4 along xi.  Shortened in time.
MIX_CONFIG = {
    "grids": {
        "default": {"operators": {"xi": "upwind9", "eta": "upwind9"}},
        "grid0": {
            "x": {"linspace": {"start": -5, "end": 0, "steps": 50, "h2": True}},
            "y": {"linspace": {"start": 0, "end": 5, "steps": 50, "h2": True}},
            "operators": {"xi": "upwind9h2", "eta": "upwind9h2"},
            "boundary_conditions": {"south": {"interpolate": {"neighbour": "grid1", "operator": "9h2"}},
                                    "east": {"neighbour": "grid3"}},
        },
        "grid1": {
            "x": {"linspace": {"start": -5, "end": 0, "steps": 98, "h2": True}},
            "y": {"linspace": {"start": -5, "end": 0, "steps": 100}},
            "operators": {"xi": "upwind9h2"},
            "boundary_conditions": {"north": {"interpolate": {"neighbour": "grid0", "operator": "9h2"}},
                                    "east": {"neighbour": "grid2"}},
        },
        "grid2": {
            "x": {"linspace": {"start": 0, "end": 5, "steps": 99}},
            "y": {"linspace": {"start": -5, "end": 0, "steps": 100}},
            "operators": {"eta": "sbp8"},
            "boundary_conditions": {"north": {"interpolate": {"neighbour": "grid3", "operator": "9"}},
                                    "west": {"neighbour": "grid1"}},
        },
        "grid3": {
            "x": {"linspace": {"start": 0, "end": 5, "steps": 50}},
            "y": {"linspace": {"start": 0, "end": 5, "steps": 50, "h2": True}},
            "operators": {"xi": "upwind4", "eta": "upwind9h2"},
            "boundary_conditions": {"south": {"interpolate": {"neighbour": "grid2", "operator": "9"}},
                                    "west": {"neighbour": "grid0"}},
        },
    },
    "integration_time": 0.1,
    "initial_conditions": {"vortex": {"vortices": [{"x0": -1.0, "y0": 0.0, "rstar": 0.5, "eps": 1.0}],
                                      "mach": 0.5}},
    "boundary_conditions": "initial_conditions",
}


def test_driver_mixed_operators(orc, tmp_path, capsys):
    """The multigrid driver on a four-block layout whose blocks use pairs of different families."""
    from summationbyparts_b200 import config, hdf5, main, multigrid
    from summationbyparts_b200.system import BlockSpec
    text = json.dumps(MIX_CONFIG)
    path = tmp_path / "mix.json"
    path.write_text(text)
    out = tmp_path / "run.hdf"
    assert main.main([str(path), "-o", str(out), "--error", "--output-json"]) == 0
    info = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    snaps = hdf5.read_flat(str(tmp_path / "run.hdf"))

    rt = config.into_runtime(config.loads(text))
    ids = [g.op.ids for g in rt.grids]
    assert ids[2] == (2, 5) and ids[3] == (0, 3)  # (xi, eta): (Upwind9, SBP8), (Upwind4, Upwind9h2)
    specs = [BlockSpec(g.x, g.y, g.op, [multigrid._bc(s) for s in (g.north, g.south, g.east, g.west)], 0)
             for g in rt.grids]
    o = oracle_system(orc, specs, rt.initial_vortex)
    o.init_vortex(0.0)
    dt = o.max_dt()
    ntime = int(round(rt.integration_time / dt))
    o.advance(ntime, dt)
    assert abs(info["error"] - o.error()) <= 1e-10 * o.error()
    for b, name in enumerate(["grid0", "grid1", "grid2", "grid3"]):
        ref = o.state(b)[0]
        assert np.max(np.abs(snaps[f"{name}/rho"][1] - ref)) <= 1e-12 * np.max(np.abs(ref)), name
