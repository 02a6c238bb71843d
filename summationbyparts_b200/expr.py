"""Expression initial conditions of the multigrid driver (multigrid/src/eval/evalexpr.rs).

The reference evaluates its `initial_conditions: {expressions: ...}` with the evalexpr crate
(version 7.2, a dependency of the reference that is not vendored with it).  This module restates
the part of evalexpr's published expression language those inputs use, evaluated on whole grids
at once with numpy (every operation is pointwise, so the result is the same as evaluating point
by point):

* values: 64-bit integers, floats and booleans; integer + - * / % stay integers (/ truncates
  toward zero, % takes the dividend's sign, as Rust's i64 operators), any float operand makes the
  result a float; ^ is always a float power;
* operators by precedence, loosest first: `;` (sequence; the value of the last non-empty
  part), `,` (tuple), `=` (assignment), `||`, `&&`, `== != < > <= >=`, `+ -`, `* / %`, unary
  `-` and `!`, `^`; function calls `name(arguments)`;
* functions: `math::` sin cos tan asin acos atan atan2 sinh cosh tanh asinh acosh atanh exp exp2
  ln log (x, base) log2 log10 sqrt cbrt abs pow hypot, and min max floor ceil round; the
  reference's own `if(c, a, b)` and `case(c1, v1, c2, v2, ..., default)`
  (eval/evalexpr.rs:300-360); constants PI, E and GAMMA.

Evaluators (eval/evalexpr.rs:10-80, euler/src/eval.rs:72-100):

* conservation form: rho(x, y, t), then rhou and rhov (which may use rho), then e (rho, rhou,
  rhov);
* pressure form: rho, u (rho), v (rho), p (rho, u, v); then e = p / (gamma - 1) +
  rho (u u + v v) / 2 and rhou = u rho, rhov = v rho.

`globals` is evaluated once into the shared context; each field's expression runs in a fresh
scope of its own on top of it, where assignments such as `r = math::hypot(x, y);` live.
The math functions are numpy's, which may differ from the host libm in the last place.
"""
from __future__ import annotations

import math
import re
from dataclasses import dataclass

import numpy as np


class ExprError(ValueError):
    pass


_TOKEN = re.compile(r"""
    (?P<ws>\s+)
  | (?P<num>(?:\d+\.\d*|\.\d+|\d+)(?:[eE][+-]?\d+)?)
  | (?P<id>[A-Za-z_][A-Za-z0-9_]*(?:::[A-Za-z_][A-Za-z0-9_]*)*)
  | (?P<op>&&|\|\||==|!=|<=|>=|[-+*/%^<>!=;,()])
""", re.X)

_BINARY = {";": 0, ",": 40, "=": 50, "||": 70, "&&": 75, "==": 80, "!=": 80, "<": 80, ">": 80, "<=": 80, ">=": 80,
           "+": 95, "-": 95, "*": 100, "/": 100, "%": 100, "^": 120}
_UNARY_PREC = 110


def _tokens(src: str):
    out, pos = [], 0
    while pos < len(src):
        m = _TOKEN.match(src, pos)
        if not m:
            raise ExprError(f"unexpected character {src[pos]!r} at {pos} in {src!r}")
        pos = m.end()
        if m.lastgroup == "ws":
            continue
        text = m.group()
        if m.lastgroup == "num":
            is_float = "." in text or "e" in text or "E" in text
            out.append(("num", float(text) if is_float else int(text)))
        elif m.lastgroup == "id":
            out.append(("id", text))
        else:
            out.append(("op", text))
    out.append(("end", None))
    return out


class _Parser:
    def __init__(self, src: str):
        self.t = _tokens(src)
        self.i = 0

    def peek(self):
        return self.t[self.i]

    def take(self):
        tok = self.t[self.i]
        self.i += 1
        return tok

    def expect(self, op):
        tok = self.take()
        if tok != ("op", op):
            raise ExprError(f"expected {op!r}, found {tok[1]!r}")

    def parse(self):
        node = self.expr(0)
        if self.peek()[0] != "end":
            raise ExprError(f"unexpected {self.peek()[1]!r}")
        return node

    def at_part_end(self):
        k, v = self.peek()
        return k == "end" or (k == "op" and v in (";", ")"))

    def expr(self, minp):
        # an empty part (`a = 1;;` or a trailing `;`) evaluates to nothing
        left = ("empty",) if self.at_part_end() else self.unary()
        while True:
            k, v = self.peek()
            if k != "op" or v not in _BINARY or _BINARY[v] < minp:
                return left
            p = _BINARY[v]
            self.take()
            right = self.expr(p if v == "=" else p + 1)  # assignment groups to the right
            if v == ";":
                left = ("seq", left, right)
            elif v == ",":
                left = ("tuple", (left[1] if left[0] == "tuple" else (left,)) + (right,))
            elif v == "=":
                if left[0] != "var":
                    raise ExprError("assignment to something that is not a name")
                left = ("assign", left[1], right)
            else:
                left = ("bin", v, left, right)

    def unary(self):
        k, v = self.peek()
        if k == "op" and v in ("-", "!"):
            self.take()
            return ("un", v, self.expr_from_unary())
        return self.primary()

    def expr_from_unary(self):
        # operand of a unary operator: everything binding tighter than it (only ^)
        left = self.unary()
        while True:
            k, v = self.peek()
            if k == "op" and v in _BINARY and _BINARY[v] > _UNARY_PREC:
                self.take()
                left = ("bin", v, left, self.expr(_BINARY[v] + 1))
            else:
                return left

    def primary(self):
        k, v = self.take()
        if k == "num":
            return ("num", v)
        if k == "id":
            if v in ("true", "false"):
                return ("num", v == "true")
            if self.peek() == ("op", "("):
                self.take()
                arg = ("empty",) if self.peek() == ("op", ")") else self.expr(0)
                self.expect(")")
                return ("call", v, arg)
            return ("var", v)
        if (k, v) == ("op", "("):
            inner = self.expr(0)
            self.expect(")")
            return inner
        raise ExprError(f"unexpected {v!r}")


def parse(src: str):
    return _Parser(src).parse()


def _is_int(v) -> bool:
    return isinstance(v, (int, np.integer)) and not isinstance(v, (bool, np.bool_))


def _f(v):
    if isinstance(v, tuple) or v is None:
        raise ExprError("a tuple or an empty expression where a number is needed")
    return np.asarray(v, dtype=np.float64) if isinstance(v, np.ndarray) else float(v)


def _idiv(a: int, b: int) -> int:
    if b == 0:
        raise ExprError("integer division by zero")
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b >= 0) else -q


def _irem(a: int, b: int) -> int:
    if b == 0:
        raise ExprError("integer remainder by zero")
    return a - b * _idiv(a, b)


def _py(v):
    """numpy scalars back to Python int / float / bool (arrays and tuples unchanged)."""
    return v.item() if isinstance(v, np.generic) else v


def _round(x):
    # Rust's f64::round: halves away from zero
    return np.sign(x) * np.floor(np.abs(x) + 0.5)


def _binary(op, a, b):
    if op in ("+", "-", "*", "/", "%") and _is_int(a) and _is_int(b):
        if op == "+":
            return a + b
        if op == "-":
            return a - b
        if op == "*":
            return a * b
        if op == "/":
            return _idiv(a, b)
        return _irem(a, b)
    if op == "+":
        return _f(a) + _f(b)
    if op == "-":
        return _f(a) - _f(b)
    if op == "*":
        return _f(a) * _f(b)
    if op == "/":
        return _f(a) / _f(b)
    if op == "%":
        return np.fmod(_f(a), _f(b))
    if op == "^":
        return np.power(_f(a), _f(b))
    if op in ("==", "!="):
        r = np.equal(a, b) if (isinstance(a, np.ndarray) or isinstance(b, np.ndarray)) else a == b
        return np.logical_not(r) if op == "!=" else r
    if op == "<":
        return np.less(_f(a), _f(b))
    if op == ">":
        return np.greater(_f(a), _f(b))
    if op == "<=":
        return np.less_equal(_f(a), _f(b))
    if op == ">=":
        return np.greater_equal(_f(a), _f(b))
    if op == "&&":
        return np.logical_and(a, b)
    if op == "||":
        return np.logical_or(a, b)
    raise ExprError(f"unknown operator {op}")


_UNARY_MATH = {"sin": np.sin, "cos": np.cos, "tan": np.tan, "asin": np.arcsin, "acos": np.arccos, "atan": np.arctan,
               "sinh": np.sinh, "cosh": np.cosh, "tanh": np.tanh, "asinh": np.arcsinh, "acosh": np.arccosh,
               "atanh": np.arctanh, "exp": np.exp, "exp2": np.exp2, "ln": np.log, "log2": np.log2, "log10": np.log10,
               "sqrt": np.sqrt, "cbrt": np.cbrt, "abs": np.abs}


def _args(v) -> tuple:
    return v if isinstance(v, tuple) else (v,)


def _call(name, arg):
    a = _args(arg)
    if name.startswith("math::"):
        f = name[6:]
        if f in _UNARY_MATH and len(a) == 1:
            return _UNARY_MATH[f](_f(a[0]))
        if f == "pow" and len(a) == 2:
            return np.power(_f(a[0]), _f(a[1]))
        if f == "hypot" and len(a) == 2:
            return np.hypot(_f(a[0]), _f(a[1]))
        if f == "atan2" and len(a) == 2:
            return np.arctan2(_f(a[0]), _f(a[1]))
        if f == "log" and len(a) == 2:
            return np.log(_f(a[0])) / np.log(_f(a[1]))
        raise ExprError(f"unknown function {name} with {len(a)} argument(s)")
    if name in ("min", "max") and a:
        if all(_is_int(v) for v in a):
            return min(a) if name == "min" else max(a)
        r = _f(a[0])
        for v in a[1:]:
            r = np.minimum(r, _f(v)) if name == "min" else np.maximum(r, _f(v))
        return r
    if name in ("floor", "ceil", "round") and len(a) == 1:
        if _is_int(a[0]):
            return a[0]
        return {"floor": np.floor, "ceil": np.ceil, "round": _round}[name](_f(a[0]))
    if name == "if":
        if len(a) != 3:
            raise ExprError("if takes 3 arguments")
        return np.where(a[0], _f(a[1]), _f(a[2])) if isinstance(a[0], np.ndarray) else (a[1] if a[0] else a[2])
    if name == "case":
        if len(a) % 2 == 0:
            raise ExprError("case takes an odd number of arguments")
        out = a[-1]
        for k in range(len(a) - 3, -1, -2):  # the first true condition wins: fold from the back
            c, v = a[k], a[k + 1]
            out = np.where(c, _f(v), _f(out)) if isinstance(c, np.ndarray) else (v if c else out)
        return out
    raise ExprError(f"unknown function {name}")


class Context:
    """Variables of one evaluation: fixed names (x, y, t, rho, ...), the scope of the
    expression's own assignments, then the shared context (globals and constants)."""

    def __init__(self, shared: dict, fixed: dict | None = None):
        self.shared = shared
        self.fixed = dict(fixed or {})
        self.scope: dict = {}

    def get(self, name):
        for d in (self.fixed, self.scope, self.shared):
            if name in d:
                return d[name]
        raise ExprError(f"unknown variable {name}")

    def set(self, name, value):
        self.scope[name] = value


def evaluate(node, ctx: Context):
    kind = node[0]
    if kind == "num":
        return node[1]
    if kind == "empty":
        return None
    if kind == "var":
        return ctx.get(node[1])
    if kind == "seq":
        a = evaluate(node[1], ctx)
        b = evaluate(node[2], ctx)
        return a if b is None else b
    if kind == "tuple":
        return tuple(evaluate(n, ctx) for n in node[1])
    if kind == "assign":
        ctx.set(node[1], evaluate(node[2], ctx))
        return None
    if kind == "un":
        v = evaluate(node[2], ctx)
        if node[1] == "-":
            return -v if _is_int(v) else _py(-_f(v))
        return _py(np.logical_not(v))
    if kind == "bin":
        return _py(_binary(node[1], evaluate(node[2], ctx), evaluate(node[3], ctx)))
    if kind == "call":
        return _py(_call(node[1], evaluate(node[2], ctx)))
    raise ExprError(f"bad node {kind}")


def shared_context(gamma: float, globals_src: str | None) -> dict:
    """default_context (eval/evalexpr.rs:300-330): PI, E, GAMMA, then the globals."""
    shared = {"PI": math.pi, "E": math.e, "GAMMA": float(gamma)}
    if globals_src:
        ctx = Context(shared)
        evaluate(parse(globals_src), ctx)
        shared.update(ctx.scope)  # assignments of the globals land in the shared context
    return shared


@dataclass
class Expressions:
    """initial_conditions: {expressions: ...} of the multigrid input (multigrid/src/input.rs:170-196)."""
    form: str            # "conservation" or "pressure"
    fields: dict         # field name -> source
    globals_src: str | None
    gamma: float

    def __post_init__(self):
        self._trees = {k: parse(v) for k, v in self.fields.items()}
        self._shared = shared_context(self.gamma, self.globals_src)

    @classmethod
    def from_config(cls, d: dict, gamma: float) -> "Expressions":
        if all(k in d for k in ("rho", "rhou", "rhov", "e")):
            form, names = "conservation", ("rho", "rhou", "rhov", "e")
        elif all(k in d for k in ("rho", "u", "v", "p")):
            form, names = "pressure", ("rho", "u", "v", "p")
        else:
            raise ExprError("expressions need rho, rhou, rhov, e or rho, u, v, p")
        return cls(form, {k: str(d[k]) for k in names}, d.get("globals"), gamma)

    def _field(self, name, x, y, t, **known):
        ctx = Context(self._shared, dict(x=x, y=y, t=float(t), **known))
        v = evaluate(self._trees[name], ctx)
        if v is None or isinstance(v, tuple):
            raise ExprError(f"expression for {name} has no numeric value")
        return np.broadcast_to(np.asarray(v, dtype=np.float64), x.shape).astype(np.float64)

    def evaluate(self, t: float, x: np.ndarray, y: np.ndarray) -> np.ndarray:
        """The (4, ny, nx) conserved state at time t on the grid (x, y)."""
        x = np.asarray(x, dtype=np.float64)
        y = np.asarray(y, dtype=np.float64)
        with np.errstate(all="ignore"):
            if self.form == "conservation":
                rho = self._field("rho", x, y, t)
                rhou = self._field("rhou", x, y, t, rho=rho)
                rhov = self._field("rhov", x, y, t, rho=rho)
                e = self._field("e", x, y, t, rho=rho, rhou=rhou, rhov=rhov)
            else:
                rho = self._field("rho", x, y, t)
                u = self._field("u", x, y, t, rho=rho)
                v = self._field("v", x, y, t, rho=rho)
                p = self._field("p", x, y, t, rho=rho, u=u, v=v)
                e = p / (self.gamma - 1.0) + rho * (u * u + v * v) / 2.0
                rhou = u * rho
                rhov = v * rho
        return np.stack([rho, rhou, rhov, e])
