"""The evalexpr subset of the multigrid driver's expression initial conditions
(summationbyparts_b200.expr): operator precedence and integer / float semantics of the
language, the reference's own context test (multigrid/src/eval/evalexpr.rs:292-305), the
reference's `if` and `case` functions, and both evaluator forms against numpy restatements of
the same formulas on a grid."""
import math

import numpy as np
import pytest

from summationbyparts_b200 import expr


def ev(src, **fixed):
    return expr.evaluate(expr.parse(src), expr.Context(expr.shared_context(1.4, None), fixed))


@pytest.mark.parametrize("src,want", [
    ("1 + 2 * 3", 7), ("(1 + 2) * 3", 9), ("7 / 2", 3), ("-7 / 2", -3), ("7 % 3", 1), ("-7 % 3", -1),
    ("7.0 / 2", 3.5), ("2 ^ 3", 8.0), ("-2 ^ 2", -4.0), ("2 ^ -1", 0.5), ("10 - 4 - 3", 3), ("2 * 3 % 4", 2),
    ("a = 2; a + 1", 3), ("a = 2; b = a * 3; b", 6), ("1 < 2 && 3 > 4", False), ("!(1 == 1) || 2 >= 2", True),
    ("if(1 < 2, 5, 6)", 5), ("case(false, 1, true, 2, 3)", 2), ("case(false, 1, false, 2, 3)", 3),
    ("min(3, 1, 2)", 1), ("max(1, 2.5)", 2.5), ("round(2.5)", 3.0), ("round(-2.5)", -3.0), ("floor(-1.5)", -2.0),
    ("math::hypot(3, 4)", 5.0), ("math::pow(2, 10)", 1024.0), ("math::sqrt(16)", 4.0), ("math::ln(E)", 1.0),
    ("math::log(8, 2)", 3.0), ("math::atan2(1, 0)", math.pi / 2), ("GAMMA", 1.4), ("x = 1;", None),
])
def test_language(src, want):
    got = ev(src)
    if isinstance(want, float):
        assert isinstance(got, float) and got == pytest.approx(want, rel=1e-15), (src, got)
    elif want is None:
        assert got is None
    else:
        assert got == want and type(got) is type(want), (src, got)


def test_reference_context_test():
    """evalexpr.rs:292-305: a = 2 in the base context, x = 3 and t = 4 in the wrapper."""
    shared = {"a": 2}
    assert expr.evaluate(expr.parse("a + x + t"), expr.Context(shared, {"x": 3, "t": 4})) == 9


def test_fixed_names_win_over_assignments_and_globals():
    shared = expr.shared_context(1.4, "k = 10; x = 99")
    ctx = expr.Context(shared, {"x": 1.0})
    assert expr.evaluate(expr.parse("k + x"), ctx) == 11.0


def test_errors():
    for bad in ("1 +", "foo(1)", "(1, 2) + 1", "1 / 0", "unknown_name + 1", "3 = 4"):
        with pytest.raises(expr.ExprError):
            ev(bad)


def grid():
    x, y = np.meshgrid(np.linspace(-1.0, 2.0, 13), np.linspace(-0.5, 1.5, 11))
    return x, y


def test_pressure_form_matches_numpy():
    """A smooth density wave in the pressure form: e = p/(g-1) + rho (u^2 + v^2)/2, rhou = u rho."""
    g = 1.4
    e = expr.Expressions.from_config({"globals": "u0 = 0.75; v0 = -0.25; p0 = 2", "rho": "1 + 0.3*math::sin(PI*(x + y - t*(u0 + v0)))",
                                      "u": "u0", "v": "v0", "p": "p0"}, g)
    x, y = grid()
    t = 0.4
    q = e.evaluate(t, x, y)
    rho = 1 + 0.3 * np.sin(np.pi * (x + y - t * (0.75 - 0.25)))
    want = np.stack([rho, 0.75 * rho, -0.25 * rho, 2 / (g - 1) + rho * (0.75 ** 2 + 0.25 ** 2) / 2])
    np.testing.assert_allclose(q, want, rtol=1e-14, atol=1e-14)


def test_piecewise_pressure_form_with_local_assignments():
    """case() over a radius assigned inside the expression, an integer global divided as a float."""
    g = 5.0 / 3.0
    e = expr.Expressions.from_config({
        "globals": "M = 0.5; q0 = 1/(GAMMA * M^2);",
        "rho": "1",
        "u": "r = math::hypot(x, y); -math::sin(math::atan2(y, x)) * case(r < 0.5, 2*r, r < 1, 2 - 2*r, 0)",
        "v": "r = math::hypot(x, y); math::cos(math::atan2(y, x)) * case(r < 0.5, 2*r, r < 1, 2 - 2*r, 0)",
        "p": "r = math::hypot(x, y); case(r < 0.5, q0 + 2*r*r, q0 + 0.5 + math::ln(2*r))"}, g)
    x, y = grid()
    q = e.evaluate(0.0, x, y)
    r = np.hypot(x, y)
    th = np.arctan2(y, x)
    s = np.where(r < 0.5, 2 * r, np.where(r < 1, 2 - 2 * r, 0.0))
    u, v = -np.sin(th) * s, np.cos(th) * s
    q0 = 1 / (g * 0.25)
    with np.errstate(divide="ignore"):
        p = np.where(r < 0.5, q0 + 2 * r * r, q0 + 0.5 + np.log(2 * r))
    want = np.stack([np.ones_like(x), u, v, p / (g - 1) + (u * u + v * v) / 2])
    np.testing.assert_allclose(q, want, rtol=1e-14, atol=1e-14)


def test_conservation_form_uses_earlier_fields():
    e = expr.Expressions.from_config({"rho": "2 + x", "rhou": "rho * y", "rhov": "-rho", "e": "rhou + rhov + t"}, 1.4)
    x, y = grid()
    q = e.evaluate(1.5, x, y)
    rho = 2 + x
    np.testing.assert_array_equal(q, np.stack([rho, rho * y, -rho, rho * y + -rho + 1.5]))


def test_scalar_results_fill_the_grid():
    e = expr.Expressions.from_config({"rho": "1", "u": "0", "v": "0", "p": "1"}, 1.4)
    x, y = grid()
    q = e.evaluate(0.0, x, y)
    assert q.shape == (4,) + x.shape and np.all(q[0] == 1.0) and np.all(q[3] == 1.0 / (1.4 - 1.0))


PROGRAM_CASES = [
    ({"globals": "M = 0.4; p0 = 1/(GAMMA * M^2);", "rho": "1",
      "u": "r = math::hypot(x, y); -math::sin(math::atan2(y, x)) * case(r < 0.2, 5*r, r < 0.4, 2 - 5*r, 0)",
      "v": "r = math::hypot(x, y); math::cos(math::atan2(y, x)) * case(r < 0.2, 5*r, r < 0.4, 2 - 5*r, 0)",
      "p": "r = math::hypot(x, y); case(r < 0.2, p0 + 25.0/2.0*r*r, p0 - 2 + 4*math::ln(2) + r)"}, 5.0 / 3.0),
    ({"globals": "ua = 1; va = 1; b = 5; Tf = (GAMMA - 1)*b*b/(8*GAMMA*PI*PI)",
      "rho": "x0 = ua*t; y0 = va*t; math::pow(1 - Tf*math::exp(1 - ((x - x0)*(x - x0) + (y - y0)*(y - y0))), 1.0/(GAMMA - 1))",
      "u": "x0 = ua*t; y0 = va*t; ua + b/(2*PI) * math::exp((1 - ((x - x0)^2 + (y - y0)^2))/2)*(-(y - y0))",
      "v": "x0 = ua*t; y0 = va*t; va + b/(2*PI) * math::exp((1 - ((x - x0)^2 + (y - y0)^2))/2)*(x - x0)",
      "p": "math::pow(rho, GAMMA)"}, 1.4),
    ({"rho": "2 + 0.1*math::cos(x) + if(y > 0.5, 0.05, -0.05)", "rhou": "rho * max(x, 0.3, y)",
      "rhov": "-rho * min(1, y)", "e": "10 + rhou*rhou/rho + floor(3.7) - 7 / 2 + 7 % 3 + round(x)"}, 1.4),
]


@pytest.mark.parametrize("case", range(len(PROGRAM_CASES)))
def test_device_programs_match_the_tree_evaluator(case):
    """The compiled device programs, run by a numpy restatement of the device interpreter, give
    the tree evaluator's fields: constant parts (integer arithmetic included) are folded on the
    host, the rest is the same f64 arithmetic in the same order."""
    d, gamma = PROGRAM_CASES[case]
    e = expr.Expressions.from_config(d, gamma)
    form, codes, consts = expr.compile_program(e)
    x, y = grid()
    t = 0.35
    q = e.evaluate(t, x, y)
    full = lambda v: np.broadcast_to(np.asarray(v, dtype=np.float64), x.shape)
    rho = full(expr.run_program(codes[0], consts, dict(x=x, y=y, t=t)))
    if form == 0:
        rhou = full(expr.run_program(codes[1], consts, dict(x=x, y=y, t=t, rho=rho)))
        rhov = full(expr.run_program(codes[2], consts, dict(x=x, y=y, t=t, rho=rho)))
        en = full(expr.run_program(codes[3], consts, dict(x=x, y=y, t=t, rho=rho, rhou=rhou, rhov=rhov)))
        got = np.stack([rho, rhou, rhov, en])
    else:
        u = full(expr.run_program(codes[1], consts, dict(x=x, y=y, t=t, rho=rho)))
        v = full(expr.run_program(codes[2], consts, dict(x=x, y=y, t=t, rho=rho)))
        p = full(expr.run_program(codes[3], consts, dict(x=x, y=y, t=t, rho=rho, u=u, v=v)))
        got = np.stack([rho, u * rho, v * rho, p / (gamma - 1.0) + rho * (u * u + v * v) / 2.0])
    np.testing.assert_array_equal(got, q)
    assert all(len(c) <= expr.MAX_CODE for c in codes) and len(consts) <= expr.MAX_CONSTS


def test_integer_parts_fold_exactly():
    """7 / 2 is the integer 3 in the language: folded on the host, never divided in f64."""
    e = expr.Expressions.from_config({"rho": "x + 7 / 2", "rhou": "0", "rhov": "0", "e": "1"}, 1.4)
    _, codes, consts = expr.compile_program(e)
    assert 3.0 in consts and 3.5 not in consts


def test_programs_reject_what_the_device_cannot_run():
    with pytest.raises(expr.ExprError):
        expr.compile_program(expr.Expressions.from_config({"rho": "math::nosuch(x)", "u": "0", "v": "0", "p": "1"}, 1.4))
    many = "; ".join(f"a{k} = x + {k}" for k in range(20)) + "; a0"
    with pytest.raises(expr.ExprError, match="local"):
        expr.compile_program(expr.Expressions.from_config({"rho": many, "u": "0", "v": "0", "p": "1"}, 1.4))
