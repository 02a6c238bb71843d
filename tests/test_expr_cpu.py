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
