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


# ----- programs for the device (SBP_BC_EVAL boundaries) --------------------------------------
# Opcodes, variables and function ids of csrc/eval_program.cuh.
(EV_CONST, EV_VAR, EV_LOAD, EV_STORE, EV_ADD, EV_SUB, EV_MUL, EV_DIV, EV_MOD, EV_POW, EV_NEG, EV_LT, EV_GT, EV_LE,
 EV_GE, EV_EQ, EV_NE, EV_AND, EV_OR, EV_NOT, EV_SELECT, EV_FN1, EV_FN2) = range(1, 24)
VARS = {"x": 0, "y": 1, "t": 2, "rho": 3, "rhou": 4, "rhov": 5, "u": 6, "v": 7}
FN1 = {n: i for i, n in enumerate(["sin", "cos", "tan", "asin", "acos", "atan", "sinh", "cosh", "tanh", "asinh",
                                   "acosh", "atanh", "exp", "exp2", "ln", "log2", "log10", "sqrt", "cbrt", "abs",
                                   "floor", "ceil", "round"])}
FN2 = {"pow": 0, "hypot": 1, "atan2": 2, "min": 3, "max": 4, "log": 5}
_BINOP = {"+": EV_ADD, "-": EV_SUB, "*": EV_MUL, "/": EV_DIV, "%": EV_MOD, "^": EV_POW, "<": EV_LT, ">": EV_GT,
          "<=": EV_LE, ">=": EV_GE, "==": EV_EQ, "!=": EV_NE, "&&": EV_AND, "||": EV_OR}
_WITH_ARG = (EV_CONST, EV_VAR, EV_LOAD, EV_STORE, EV_FN1, EV_FN2)
MAX_CODE, MAX_CONSTS, MAX_STACK, MAX_LOCALS = 512, 256, 32, 16
_SINK = MAX_LOCALS - 1  # slot that swallows the value of a discarded sequence part


class _Compiler:
    """One field's expression -> a stack program.  A subtree without runtime variables is
    evaluated here with the tree evaluator (exact integer semantics) and becomes a constant;
    the rest runs in f64 on the device."""

    def __init__(self, shared: dict, consts: list, runtime: tuple):
        self.shared, self.consts, self.runtime = shared, consts, runtime
        self.locals: dict = {}  # name -> ("const", value) or ("slot", index)
        self.nslots = 0

    def const_word(self, v) -> list:
        v = float(v)
        for k, c in enumerate(self.consts):
            if c == v and math.copysign(1.0, c) == math.copysign(1.0, v):
                return [EV_CONST, k]
        self.consts.append(v)
        return [EV_CONST, len(self.consts) - 1]

    def words(self, r) -> list:
        kind, v = r
        if kind in ("none", "store"):
            raise ExprError("an empty expression or an assignment where a number is needed")
        if kind == "tuple":
            raise ExprError("a tuple where a number is needed")
        return self.const_word(v) if kind == "const" else list(v)

    def comp(self, node):
        kind = node[0]
        if kind == "num":
            return ("const", node[1])
        if kind == "empty":
            return ("none", None)
        if kind == "var":
            name = node[1]
            if name in self.runtime:
                return ("code", [EV_VAR, VARS[name]])
            if name in self.locals:
                k, v = self.locals[name]
                return ("const", v) if k == "const" else ("code", [EV_LOAD, v])
            if name in self.shared:
                return ("const", self.shared[name])
            raise ExprError(f"unknown variable {name}")
        if kind == "assign":
            r = self.comp(node[2])
            if r[0] == "const":
                self.locals[node[1]] = r
                return ("none", None)
            prev = self.locals.get(node[1])
            if prev and prev[0] == "slot":
                slot = prev[1]
            else:
                if self.nslots >= _SINK:
                    raise ExprError("too many local variables")
                slot = self.nslots
                self.nslots += 1
            code = self.words(r) + [EV_STORE, slot]
            self.locals[node[1]] = ("slot", slot)
            return ("store", code)
        if kind == "seq":
            a = self.comp(node[1])
            b = self.comp(node[2])
            if b[0] == "none":
                return a
            pre = a[1] if a[0] == "store" else (a[1] + [EV_STORE, _SINK] if a[0] == "code" else [])
            if b[0] == "store":
                return ("store", pre + b[1])
            if not pre:
                return b
            return ("code", pre + self.words(b))
        if kind == "tuple":
            return ("tuple", [self.comp(n) for n in node[1]])
        if kind == "un":
            r = self.comp(node[2])
            if r[0] == "const":
                return ("const", evaluate(("un", node[1], ("num", r[1])), Context({})))
            return ("code", self.words(r) + [EV_NEG if node[1] == "-" else EV_NOT])
        if kind == "bin":
            a, b = self.comp(node[2]), self.comp(node[3])
            if a[0] == "const" and b[0] == "const":
                return ("const", _py(_binary(node[1], a[1], b[1])))
            return ("code", self.words(a) + self.words(b) + [_BINOP[node[1]]])
        if kind == "call":
            r = self.comp(node[2])
            args = r[1] if r[0] == "tuple" else ([] if r[0] == "none" else [r])
            if all(x[0] == "const" for x in args):
                vals = tuple(x[1] for x in args)
                return ("const", _py(_call(node[1], vals if len(vals) != 1 else vals[0])))
            return ("code", self.call(node[1], args))
        raise ExprError(f"bad node {kind}")

    def call(self, name, args) -> list:
        math_fn = name.startswith("math::")
        f = name[6:] if math_fn else name
        if math_fn and f in FN1 and f not in ("floor", "ceil", "round") and len(args) == 1:
            return self.words(args[0]) + [EV_FN1, FN1[f]]
        if not math_fn and f in ("floor", "ceil", "round") and len(args) == 1:
            return self.words(args[0]) + [EV_FN1, FN1[f]]
        if math_fn and f in ("pow", "hypot", "atan2", "log") and len(args) == 2:
            return self.words(args[0]) + self.words(args[1]) + [EV_FN2, FN2[f]]
        if not math_fn and f in ("min", "max") and args:
            code = self.words(args[0])
            for a in args[1:]:
                code += self.words(a) + [EV_FN2, FN2[f]]
            return code
        if name == "if" and len(args) == 3:
            return self.words(args[0]) + self.words(args[1]) + self.words(args[2]) + [EV_SELECT]
        if name == "case" and len(args) % 2 == 1:
            code = self.words(args[-1])
            for k in range(len(args) - 3, -1, -2):
                code = self.words(args[k]) + self.words(args[k + 1]) + code + [EV_SELECT]
            return code
        raise ExprError(f"function {name} with {len(args)} argument(s) cannot run on the device")


def _depth(code: list) -> int:
    sp = best = 0
    pc = 0
    while pc < len(code):
        op = code[pc]
        pc += 2 if op in _WITH_ARG else 1
        if op in (EV_CONST, EV_VAR, EV_LOAD):
            sp += 1
        elif op in (EV_STORE, EV_FN2) or op in _BINOP.values():
            sp -= 1
        elif op == EV_SELECT:
            sp -= 2
        best = max(best, sp)
    return best


def compile_program(e: "Expressions"):
    """The four device programs of an evaluator as sbp_system_set_eval takes them: (form: 0
    conservation / 1 pressure, [code of each field], constants)."""
    if e.form == "conservation":
        names = ("rho", "rhou", "rhov", "e")
        runtime = (("x", "y", "t"), ("x", "y", "t", "rho"), ("x", "y", "t", "rho"),
                   ("x", "y", "t", "rho", "rhou", "rhov"))
    else:
        names = ("rho", "u", "v", "p")
        runtime = (("x", "y", "t"), ("x", "y", "t", "rho"), ("x", "y", "t", "rho"), ("x", "y", "t", "rho", "u", "v"))
    consts: list = []
    codes = []
    for name, rt in zip(names, runtime):
        c = _Compiler(e._shared, consts, rt)
        r = c.comp(e._trees[name])
        if r[0] not in ("const", "code"):
            raise ExprError(f"expression for {name} has no numeric value")
        code = c.words(r)
        if len(code) > MAX_CODE or _depth(code) > MAX_STACK:
            raise ExprError(f"expression for {name} is too long for the device")
        codes.append(code)
    if len(consts) > MAX_CONSTS:
        raise ExprError("too many constants for the device")
    return (0 if e.form == "conservation" else 1), codes, consts


def run_program(code: list, consts: list, vars_: dict):
    """The device interpreter restated with numpy (test infrastructure for the compiler)."""
    st, loc = [], {}
    pc = 0
    v = [vars_.get(n, 0.0) for n in VARS]
    f1 = [np.sin, np.cos, np.tan, np.arcsin, np.arccos, np.arctan, np.sinh, np.cosh, np.tanh, np.arcsinh, np.arccosh,
          np.arctanh, np.exp, np.exp2, np.log, np.log2, np.log10, np.sqrt, np.cbrt, np.abs, np.floor, np.ceil, _round]
    f2 = [np.power, np.hypot, np.arctan2, np.fmin, np.fmax, lambda a, b: np.log(a) / np.log(b)]
    ops = {EV_ADD: np.add, EV_SUB: np.subtract, EV_MUL: np.multiply, EV_DIV: np.divide, EV_MOD: np.fmod,
           EV_POW: np.power}
    cmp = {EV_LT: np.less, EV_GT: np.greater, EV_LE: np.less_equal, EV_GE: np.greater_equal, EV_EQ: np.equal,
           EV_NE: np.not_equal}
    with np.errstate(all="ignore"):
        while pc < len(code):
            op = code[pc]
            arg = code[pc + 1] if op in _WITH_ARG else None
            pc += 2 if op in _WITH_ARG else 1
            if op == EV_CONST:
                st.append(np.float64(consts[arg]))
            elif op == EV_VAR:
                st.append(v[arg])
            elif op == EV_LOAD:
                st.append(loc[arg])
            elif op == EV_STORE:
                loc[arg] = st.pop()
            elif op == EV_NEG:
                st.append(-st.pop())
            elif op == EV_NOT:
                st.append(np.where(st.pop() != 0.0, 0.0, 1.0))
            elif op == EV_FN1:
                st.append(f1[arg](st.pop()))
            elif op == EV_FN2:
                b = st.pop()
                st.append(f2[arg](st.pop(), b))
            elif op == EV_SELECT:
                b, a, c = st.pop(), st.pop(), st.pop()
                st.append(np.where(c != 0.0, a, b))
            else:
                b, a = st.pop(), st.pop()
                if op in ops:
                    st.append(ops[op](a, b))
                elif op in cmp:
                    st.append(np.where(cmp[op](a, b), 1.0, 0.0))
                elif op == EV_AND:
                    st.append(np.where((a != 0.0) & (b != 0.0), 1.0, 0.0))
                else:
                    st.append(np.where((a != 0.0) | (b != 0.0), 1.0, 0.0))
    if len(st) != 1:
        raise ExprError("program did not leave exactly one value")
    return st[0]
