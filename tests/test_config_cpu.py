"""The multigrid driver's configuration reading (summationbyparts_b200/config.py), which
restates multigrid/src/input.rs and parsing.rs: json5 syntax, the "default" grid, grid
broadcasting, operators and every boundary form.  CPU only."""
import numpy as np
import pytest

from summationbyparts_b200 import config, multigrid as mg


def test_json5_syntax():
    v = config.loads("""
    // line comment
    { unquoted: 1, 'single': 'it\\'s', "double": "a\\nb", /* block */ hex: 0x1F, plus: +2.5,
      lead: .5, trail: 5., inf: -Infinity, list: [1, 2, 3,], nested: { t: true, f: false, n: null, }, }
    """)
    assert v["unquoted"] == 1 and v["single"] == "it's" and v["double"] == "a\nb"
    assert v["hex"] == 31 and v["plus"] == 2.5 and v["lead"] == 0.5 and v["trail"] == 5.0
    assert v["inf"] == -np.inf and v["list"] == [1, 2, 3]
    assert v["nested"] == {"t": True, "f": False, "n": None}
    with pytest.raises(config.ConfigError):
        config.loads("{a: 1,, }")
    with pytest.raises(config.ConfigError):
        config.loads("{a: 1} x")


BASE = """{
  grids: { %s },
  integration_time: 0.5,
  initial_conditions: { vortex: { vortices: [{ x0: -1, y0: 0, rstar: 0.5, eps: 1 }], mach: 0.5 } },
  boundary_conditions: %s,
}"""


def rt(grids, bc='"initial_conditions"'):
    return config.into_runtime(config.loads(BASE % (grids, bc)))


def test_defaults_and_broadcasting():
    r = rt("""default: { operators: { xi: "upwind4", eta: "sbp8" }, y: { linspace: { start: -1, end: 1, steps: 9, h2: true } } },
              a: { x: { linspace: { start: 0, end: 1, steps: 5 } } },
              b: { x: [0, 1, 2], y: [[0, 0, 0], [1, 1, 1]], operators: { eta: "upwind9h2" } }""")
    assert r.names == ["a", "b"]
    a, b = r.grids
    assert a.x.shape == (9, 5) and np.allclose(a.x[3], [0, 0.25, 0.5, 0.75, 1.0])
    assert np.allclose(a.y[:, 0], config.h2linspace(-1.0, 1.0, 9))
    assert a.op.xi_op.__class__.__name__ == "Upwind4" and a.op.eta_op.__class__.__name__ == "SBP8"
    assert b.x.shape == (2, 3) and np.array_equal(b.y[1], [1, 1, 1])
    assert b.op.eta_op.__class__.__name__ == "Upwind9h2" and b.op.xi_op.__class__.__name__ == "Upwind4"
    assert (a.north, a.south, a.east, a.west) == (mg.VORTEX,) * 4


def test_boundary_forms():
    g = """default: { operators: { xi: "upwind9", eta: "upwind9" }, x: { linspace: { start: 0, end: 1, steps: 25 } },
                      y: { linspace: { start: 0, end: 1, steps: 25 } } },
           p: { boundary_conditions: { north: "this", south: { neighbour: "q" }, east: { interpolate: { neighbour: "q", operator: "9h2" } },
                                       west: { multi: [{ neighbour: "p", start: 0, end: 13 }, { neighbor: "q", start: 12, end: 25 }] } } },
           q: { boundary_conditions: { north: "vortex" } }"""
    p, q = rt(g).grids
    assert p.north == mg.THIS and p.south == ("grid", 1) and p.east == ("interpolate", 1, 3)
    assert p.west == ("multi", [(0, 0, 13), (1, 12, 25)])
    assert q.north == mg.VORTEX and q.south == mg.VORTEX


def test_configuration_errors():
    ops = 'default: { operators: { xi: "upwind4", eta: "upwind4" }, x: [0, 1, 2, 3, 4, 5, 6, 7], y: [0, 1, 2, 3, 4, 5, 6, 7] }'
    with pytest.raises(config.ConfigError, match="eta operator"):
        rt('a: { operators: { xi: "upwind4" }, x: [0, 1], y: [0, 1] }')
    with pytest.raises(config.ConfigError, match="unknown neighbour"):
        rt(ops + ', a: { boundary_conditions: { north: { neighbour: "zz" } } }')
    with pytest.raises(config.ConfigError, match="not available"):
        rt(ops + ", a: {}", '"not_needed"')
    # expression initial conditions; sides without their own boundary take expression (Eval)
    # boundaries from "initial_conditions" or from boundary expressions
    expr_ic = '{expressions: {rho: "1", rhou: "1", rhov: "0", e: "2"}}'
    r = config.into_runtime(config.loads('{grids: {' + ops + ', a: { boundary_conditions: { north: "this", '
                                         'south: "this", east: "this", west: "this" } } }, integration_time: 1, '
                                         'initial_conditions: ' + expr_ic + '}'))
    assert r.initial_vortex is None and r.initial is r.initial_expressions and r.boundary_expressions is None
    r = config.into_runtime(config.loads('{grids: {' + ops + ', a: { boundary_conditions: { north: "this" } } }, '
                                         'integration_time: 1, initial_conditions: ' + expr_ic
                                         + ', boundary_conditions: "initial_conditions"}'))
    a = r.grids[0]
    assert a.north == mg.THIS and a.south == a.east == a.west == mg.EVAL
    assert r.boundary_expressions is r.initial_expressions
    with pytest.raises(config.ConfigError, match="boundary expressions"):
        config.into_runtime(config.loads('{grids: {' + ops + ', a: {} }, integration_time: 1, initial_conditions: '
                                         + expr_ic + ', boundary_conditions: {expressions: {rho: "1", rhou: '
                                         '"math::nosuch(x)", rhov: "0", e: "2"}}}'))
    with pytest.raises(config.ConfigError, match="initial_conditions"):
        config.into_runtime(config.loads('{grids: {' + ops + ', a: {} }, integration_time: 1, initial_conditions: '
                                         '{expressions: {rho: "1", u: "1"}}}'))


def test_boundary_vortex_separate_from_initial():
    r = rt('default: { operators: { xi: "upwind4", eta: "upwind4" }, x: [0, 1, 2, 3, 4, 5, 6, 7], y: [0, 1, 2, 3, 4, 5, 6, 7] }, a: {}',
           '{ vortex: { vortices: [{ x0: 1, y0: 1, rstar: 0.5, eps: 2 }], mach: 0.7 } }')
    assert r.initial_vortex.mach == 0.5 and r.boundary_vortex.mach == 0.7
