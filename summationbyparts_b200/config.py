"""The multigrid driver's configuration files: json5 reading and the reference's semantics.

A restatement, for the GPU driver, of multigrid/src/input.rs (the file format) and
multigrid/src/parsing.rs (into_runtime: the configuration turned into grids, operators and
boundary characteristics), so that the reference's example configurations run unchanged:

    {
      grids: {
        default: { operators: { xi: "upwind9", eta: "upwind9" } },       // fallback for every grid
        grid0: { x: { linspace: { start: -5, end: 5, steps: 50 } },
                 y: { linspace: { start: 0, end: 5, steps: 25 } },
                 boundary_conditions: { south: { interpolate: { neighbour: "grid1", operator: "9" } } } },
        grid1: { ... },
      },
      integration_time: 2.0,
      initial_conditions: { vortex: { vortices: [{ x0: -1, y0: 0, rstar: 0.5, eps: 1 }], mach: 0.5 } },
      boundary_conditions: "initial_conditions",
      gamma: 1.4,                                                         // default 1.4
    }

Grids: `x` / `y` are {linspace: {start, end, steps, h2}} or arrays (1-D, broadcast against the
other coordinate, or 2-D (ny, nx)); missing fields come from the "default" grid.  Operators:
upwind4, upwind9, upwind4h2, upwind9h2, sbp4, sbp8.  Boundaries per side (north, south, east,
west): "this", "vortex", {neighbour: name} (alias neighbor), {interpolate: {neighbour, operator:
"4" | "8" | "9" | "9h2"}}, {multi: [{neighbour, start, end}, ...]}; an unspecified side takes the
global boundary conditions ("initial_conditions", {vortex: ...} or "not_needed").  Initial
conditions are a vortex or evalexpr expressions (summationbyparts_b200.expr, evaluated on the
host); global boundary conditions given as expressions (or "initial_conditions" with expression
initial conditions) make the unspecified sides the reference's `Eval` boundaries, evaluated on
the device at every stage time.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import multigrid as mg
from .expr import Expressions, ExprError, compile_program
from .operators import SBP4, SBP8, Pair, Upwind4, Upwind4h2, Upwind9, Upwind9h2
from .system import Vortice, VortexParameters


class ConfigError(ValueError):
    """The configuration cannot be read or describes something this driver does not run."""


# ------------------------------------------------------------------------------------------
# json5 (https://spec.json5.org): JSON plus comments, trailing commas, unquoted keys,
# single-quoted strings, hexadecimal numbers, leading/trailing decimal points, Infinity / NaN.
class _Json5:
    def __init__(self, text: str):
        self.s = text
        self.i = 0

    def error(self, msg):
        line = self.s.count("\n", 0, self.i) + 1
        col = self.i - (self.s.rfind("\n", 0, self.i) + 1) + 1
        raise ConfigError(f"json5: {msg} at line {line}, column {col}")

    def skip(self):
        s = self.s
        while self.i < len(s):
            c = s[self.i]
            if c in " \t\r\n ﻿  ":
                self.i += 1
            elif s.startswith("//", self.i):
                j = s.find("\n", self.i)
                self.i = len(s) if j < 0 else j + 1
            elif s.startswith("/*", self.i):
                j = s.find("*/", self.i + 2)
                if j < 0:
                    self.error("unterminated comment")
                self.i = j + 2
            else:
                break

    def value(self):
        self.skip()
        if self.i >= len(self.s):
            self.error("unexpected end of input")
        c = self.s[self.i]
        if c == "{":
            return self.obj()
        if c == "[":
            return self.arr()
        if c in "\"'":
            return self.string()
        for word, val in (("true", True), ("false", False), ("null", None)):
            if self.s.startswith(word, self.i) and not self._ident_char(self.i + len(word)):
                self.i += len(word)
                return val
        return self.number()

    def _ident_char(self, j):
        return j < len(self.s) and (self.s[j].isalnum() or self.s[j] in "_$")

    def obj(self):
        self.i += 1
        out = {}
        while True:
            self.skip()
            if self.s[self.i] == "}":
                self.i += 1
                return out
            if self.s[self.i] in "\"'":
                key = self.string()
            else:
                j = self.i
                while self._ident_char(self.i):
                    self.i += 1
                if j == self.i:
                    self.error("expected a key")
                key = self.s[j:self.i]
            self.skip()
            if self.s[self.i] != ":":
                self.error("expected ':'")
            self.i += 1
            out[key] = self.value()
            self.skip()
            if self.s[self.i] == ",":
                self.i += 1
            elif self.s[self.i] != "}":
                self.error("expected ',' or '}'")

    def arr(self):
        self.i += 1
        out = []
        while True:
            self.skip()
            if self.s[self.i] == "]":
                self.i += 1
                return out
            out.append(self.value())
            self.skip()
            if self.s[self.i] == ",":
                self.i += 1
            elif self.s[self.i] != "]":
                self.error("expected ',' or ']'")

    def string(self):
        q = self.s[self.i]
        self.i += 1
        out = []
        esc = {"n": "\n", "t": "\t", "r": "\r", "b": "\b", "f": "\f", "v": "\v", "0": "\0"}
        while True:
            if self.i >= len(self.s):
                self.error("unterminated string")
            c = self.s[self.i]
            if c == q:
                self.i += 1
                return "".join(out)
            if c == "\\":
                n = self.s[self.i + 1]
                if n == "u":
                    out.append(chr(int(self.s[self.i + 2:self.i + 6], 16)))
                    self.i += 6
                    continue
                if n == "\n":
                    self.i += 2
                    continue
                out.append(esc.get(n, n))
                self.i += 2
                continue
            out.append(c)
            self.i += 1

    def number(self):
        j = self.i
        s = self.s
        sign = 1.0
        if s[self.i] in "+-":
            sign = -1.0 if s[self.i] == "-" else 1.0
            self.i += 1
        if s.startswith("Infinity", self.i):
            self.i += 8
            return sign * math.inf
        if s.startswith("NaN", self.i):
            self.i += 3
            return math.nan
        if s.startswith(("0x", "0X"), self.i):
            k = self.i + 2
            while k < len(s) and s[k] in "0123456789abcdefABCDEF":
                k += 1
            v = int(s[self.i + 2:k], 16)
            self.i = k
            return int(sign) * v
        k = self.i
        while k < len(s) and s[k] in "0123456789.eE+-":
            if s[k] in "+-" and s[k - 1] not in "eE":
                break
            k += 1
        text = s[self.i:k]
        if not text:
            self.error("unexpected character")
        self.i = k
        if any(ch in text for ch in ".eE"):
            return sign * float(text)
        return int(sign) * int(text)


def loads(text: str):
    p = _Json5(text)
    v = p.value()
    p.skip()
    if p.i != len(p.s):
        p.error("trailing characters")
    return v


# ------------------------------------------------------------------------------------------
OPERATORS = {"upwind4": Upwind4, "upwind9": Upwind9, "upwind4h2": Upwind4h2, "upwind9h2": Upwind9h2,
             "sbp4": SBP4, "sbp8": SBP8}
INTERPOLATION = {"4": 0, "8": 1, "9": 2, "9h2": 3}
SIDES = ("north", "south", "east", "west")


def h2linspace(start: float, end: float, n: int) -> np.ndarray:
    """sbp::utils::h2linspace (sbp/src/utils.rs:133-140)."""
    h = (end - start) / (n - 2)
    x = start + h * (np.arange(n, dtype=np.float64) - 0.5)
    x[0], x[-1] = start, end
    return x


def ndarray_linspace(start: float, end: float, n: int) -> np.ndarray:
    """ndarray::Array::linspace: start + step * i, step = (end - start) / (n - 1)."""
    if n == 1:
        return np.array([float(start)])
    step = (end - start) / (n - 1)
    return start + step * np.arange(n, dtype=np.float64)


def _array_form(g):
    """GridLike -> ("1d" | "2d", array) (input.rs:68-81)."""
    if isinstance(g, dict):
        if "linspace" in g:
            ls = g["linspace"]
            n = int(ls["steps"])
            f = h2linspace if ls.get("h2", False) else ndarray_linspace
            return "1d", f(float(ls["start"]), float(ls["end"]), n)
        if "array" in g:
            g = g["array"]
        else:
            raise ConfigError(f"unknown grid description {list(g)}")
    a = np.asarray(g, dtype=np.float64)
    if a.ndim == 1:
        return "1d", a
    if a.ndim == 2:
        return "2d", a
    raise ConfigError("grid arrays must be 1-D or 2-D")


def _grid_xy(gx, gy):
    """into_runtime's broadcasting of x and y (parsing.rs:70-110)."""
    (kx, x), (ky, y) = _array_form(gx), _array_form(gy)
    if kx == "1d" and ky == "1d":
        return np.broadcast_to(x[None, :], (y.size, x.size)).copy(), np.broadcast_to(y[:, None], (y.size, x.size)).copy()
    if kx == "1d" and ky == "2d":
        if x.size != y.shape[1]:
            raise ConfigError("x length differs from y's inner dimension")
        return np.broadcast_to(x[None, :], y.shape).copy(), y
    if kx == "2d" and ky == "1d":
        if x.shape[0] != y.size:
            raise ConfigError("y length differs from x's outer dimension")
        return x, np.broadcast_to(y[:, None], x.shape).copy()
    if x.shape != y.shape:
        raise ConfigError("x and y arrays differ in shape")
    return x, y


def _vortex(d) -> VortexParameters:
    """euler::VortexParameters as serialised (euler/src/vortex.rs:4-21)."""
    vs = [Vortice(float(v["x0"]), float(v["y0"]), float(v["rstar"]), float(v["eps"])) for v in d["vortices"]]
    return VortexParameters(vs, mach=float(d["mach"]))


@dataclass
class Runtime:
    """RuntimeConfiguration (parsing.rs:31-38) for the GPU driver."""
    names: list
    grids: list                      # multigrid.Grid with boundary characteristics resolved
    integration_time: float
    initial_vortex: VortexParameters | None   # vortex initial conditions, or
    boundary_vortex: VortexParameters | None
    gamma: float = 1.4
    raw: dict = field(default_factory=dict)
    initial_expressions: Expressions | None = None  # expression initial conditions
    boundary_expressions: Expressions | None = None  # data of EVAL sides

    @property
    def initial(self):
        """The initial conditions (and exact solution of --error): a vortex or expressions."""
        return self.initial_expressions if self.initial_expressions is not None else self.initial_vortex


def into_runtime(cfg: dict) -> Runtime:
    """Configuration::into_runtime (parsing.rs:40-232)."""
    grids = dict(cfg["grids"])
    default = grids.pop("default", {}) or {}
    names = list(grids)
    index = {n: i for i, n in enumerate(names)}
    gamma = float(cfg.get("gamma", 1.4))
    ic = cfg["initial_conditions"]
    initial, iexpr = None, None
    if isinstance(ic, dict) and "vortex" in ic:
        initial = _vortex(ic["vortex"])
    elif isinstance(ic, dict) and "expressions" in ic:
        try:
            iexpr = Expressions.from_config(ic["expressions"], gamma)
        except ExprError as e:
            raise ConfigError(f"initial_conditions: {e}") from None
    else:
        raise ConfigError("initial_conditions must be a vortex or expressions")
    # sides without their own boundary take the global boundary conditions: a vortex, or
    # expressions (BoundaryCharacteristic::Eval, parsing.rs:55-70, 179-186)
    gbc = cfg.get("boundary_conditions", "not_needed")
    bexpr = None
    if gbc == "initial_conditions":
        bvortex = initial
        bexpr = iexpr
    elif gbc == "not_needed":
        bvortex = None
    elif isinstance(gbc, dict) and "vortex" in gbc:
        bvortex = _vortex(gbc["vortex"])
    elif isinstance(gbc, dict) and "expressions" in gbc:
        bvortex = None
        try:
            bexpr = Expressions.from_config(gbc["expressions"], gamma)
        except ExprError as e:
            raise ConfigError(f"boundary_conditions: {e}") from None
    else:
        raise ConfigError(f"unknown boundary_conditions {gbc!r}")
    if bexpr is not None:
        try:
            compile_program(bexpr)  # every expression must run on the device
        except ExprError as e:
            raise ConfigError(f"boundary expressions: {e}") from None

    def neighbour(n):
        if n not in index:
            raise ConfigError(f"unknown neighbour grid {n!r}")
        return index[n]

    out = []
    for name in names:
        g = grids[name] or {}
        gx = g.get("x", default.get("x"))
        gy = g.get("y", default.get("y"))
        if gx is None or gy is None:
            raise ConfigError(f"grid {name!r} has no x or y")
        x, y = _grid_xy(gx, gy)
        ops = g.get("operators") or {}
        dops = default.get("operators") or {}
        xi = ops.get("xi", dops.get("xi"))
        eta = ops.get("eta", dops.get("eta"))
        if xi is None or eta is None:
            raise ConfigError(f"No {'xi' if xi is None else 'eta'} operator found for grid: {name}")
        if xi not in OPERATORS or eta not in OPERATORS:
            raise ConfigError(f"unknown operator in grid {name!r}")
        op = Pair(OPERATORS[eta](), OPERATORS[xi]())
        bcs = g.get("boundary_conditions") or {}
        dbcs = default.get("boundary_conditions") or {}
        sides = []
        for side in SIDES:
            bc = bcs.get(side, dbcs.get(side))
            if bc is None:
                if bexpr is not None:
                    sides.append(mg.EVAL)
                    continue
                if bvortex is None:
                    raise ConfigError(f"Boundary conditions are not available, but needed for grid {name}")
                sides.append(mg.VORTEX)
            elif bc == "this":
                sides.append(mg.THIS)
            elif bc == "vortex":
                if bvortex is None:
                    raise ConfigError(f"Wanted vortex boundary conditions not found, needed for grid {name}")
                sides.append(mg.VORTEX)
            elif isinstance(bc, dict) and ("neighbour" in bc or "neighbor" in bc):
                sides.append(mg.grid_bc(neighbour(bc.get("neighbour", bc.get("neighbor")))))
            elif isinstance(bc, dict) and "interpolate" in bc:
                ip = bc["interpolate"]
                nb = ip.get("neighbour", ip.get("neighbor"))
                if ip.get("operator") is None:
                    raise ConfigError(f"grid {name!r}: interpolation without an operator")
                sides.append(mg.interpolate_bc(neighbour(nb), INTERPOLATION[str(ip["operator"])]))
            elif isinstance(bc, dict) and "multi" in bc:
                segs = [(neighbour(m.get("neighbour", m.get("neighbor"))), int(m["start"]), int(m["end"]))
                        for m in bc["multi"]]
                sides.append(mg.multi_bc(segs))
            else:
                raise ConfigError(f"grid {name!r}: unknown boundary {bc!r}")
        out.append(mg.Grid(x, y, op, *sides, name=name))
    return Runtime(names, out, float(cfg["integration_time"]), initial, bvortex, gamma, cfg, iexpr, bexpr)


def load(path: str) -> Runtime:
    with open(path) as f:
        return into_runtime(loads(f.read()))
