"""Generate the interpolation-operator coefficient headers from the reference's operator files.

    python oracle/gen_interp_coefficients.py <reference root>

Reads sbp/src/operators/interpolation/interpolation{4,8,9,9h2}.rs under the given checkout of
the reference (a required argument), evaluates every table entry as Rust does in both builds (each literal parsed
to the nearest f64, or f32 for the reference's f32 feature, a quotient of two literals divided
once in that type), and writes the values, printed so that they parse back to the identical
numbers, to

    summationbyparts_b200/csrc/interp_coefficients.h   (library)
    oracle/oracle_interp_coefficients.h                  (oracle)

The two headers hold the same numbers under different names, so the oracle and the library
share no code; tests/test_oracle_kat.py checks that they agree bit for bit.  The jump pairs
and the fine/coarse size relations are the arguments each operator passes to `interpolate`
(interpolation.rs:15-50) and its size asserts.
"""
from __future__ import annotations

import os
import re
import sys
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

# name, file, (jump f2c), (jump c2f), fine = 2 * coarse - 1 (False: 2 * (coarse - 1))
OPS = [("4", "interpolation4.rs", (3, 2), (4, 1), True),
       ("8", "interpolation8.rs", (0, 2), (8, 1), True),
       ("9", "interpolation9.rs", (5, 2), (8, 1), True),
       ("9H2", "interpolation9h2.rs", (4, 2), (8, 1), False)]


def f32_literal(text: str) -> np.float32:
    """The f32 nearest to a decimal literal (what the f32 build of the reference parses)."""
    exact = Fraction(text)
    c = np.float32(float(exact))
    best = c
    for cand in (np.nextafter(c, np.float32(-np.inf)), np.nextafter(c, np.float32(np.inf))):
        if abs(Fraction(float(cand)) - exact) < abs(Fraction(float(best)) - exact):
            best = cand
    return best


def value(expr: str, f32: bool = False):
    expr = expr.strip()
    neg = expr.startswith("-")
    if neg:
        expr = expr[1:].strip()
    parts = [p.strip() for p in expr.split("/")]
    conv = f32_literal if f32 else float
    v = conv(parts[0])
    if len(parts) == 2:
        v = v / conv(parts[1])
    elif len(parts) != 1:
        raise ValueError(expr)
    return -v if neg else v


def table(src: str, name: str, f32: bool = False):
    m = re.search(r"const\s+" + name + r"\s*:\s*&'static\s*\[\[Float;\s*(\d+)\]\]\s*=\s*&\[(.*?)\];", src, re.S)
    if not m:
        raise ValueError(name)
    cols = int(m.group(1))
    body = re.sub(r"//[^\n]*", "", m.group(2))
    rows = []
    for r in re.findall(r"\[(.*?)\]", body, re.S):
        vals = [value(x, f32) for x in r.split(",") if x.strip()]
        if len(vals) != cols:
            raise ValueError(f"{name}: row of {len(vals)} values, expected {cols}")
        rows.append(vals)
    return rows


def lit(v: float) -> str:
    r = repr(v)
    if "e" not in r and "." not in r and "inf" not in r and "nan" not in r:
        r += ".0"
    return r


def emit(ops, prefix: str, guard: str, note: str) -> str:
    out = [f"// {note}", "// Generated by oracle/gen_interp_coefficients.py from the reference's",
           "// sbp/src/operators/interpolation/interpolation{4,8,9,9h2}.rs; do not edit by hand.",
           "#pragma once", ""]
    for name, t, jf, jc, odd in ops:
        for d, key, jump in (("F2C", "f2c", jf), ("C2F", "c2f", jc)):
            blk, dia = t[d + "_BLOCK"], t[d + "_DIAG"]
            p = f"{prefix}{name}_{d}"
            out.append(f"// Interpolation{name.lower()} {key}: block {len(blk)} x {len(blk[0])}, "
                       f"diagonal {len(dia)} x {len(dia[0])}, jump ({jump[0]}, {jump[1]})")
            out.append(f"#define {p}_BROWS {len(blk)}")
            out.append(f"#define {p}_BCOLS {len(blk[0])}")
            out.append(f"#define {p}_DROWS {len(dia)}")
            out.append(f"#define {p}_DCOLS {len(dia[0])}")
            out.append(f"#define {p}_JUMP0 {jump[0]}")
            out.append(f"#define {p}_JUMP1 {jump[1]}")
            out.append(f"#define {p}_BLOCK " + ", ".join(lit(v) for row in blk for v in row))
            out.append(f"#define {p}_DIAG " + ", ".join(lit(v) for row in dia for v in row))
            b32, d32 = t[d + "_BLOCK_F32"], t[d + "_DIAG_F32"]
            out.append(f"#define {p}_BLOCK_F32 " + ", ".join(lit(float(v)) + "f" for row in b32 for v in row))
            out.append(f"#define {p}_DIAG_F32 " + ", ".join(lit(float(v)) + "f" for row in d32 for v in row))
            out.append("")
        out.append(f"#define {prefix}{name}_FINE_ODD {1 if odd else 0}  // fine = 2 coarse - 1 (else 2 (coarse - 1))")
        out.append("")
    return "\n".join(out) + "\n"


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python oracle/gen_interp_coefficients.py <reference root>")
    ref = sys.argv[1]
    ops = []
    for name, fn, jf, jc, odd in OPS:
        src = open(os.path.join(ref, "sbp", "src", "operators", "interpolation", fn)).read()
        t = {k: table(src, k) for k in ("F2C_DIAG", "F2C_BLOCK", "C2F_DIAG", "C2F_BLOCK")}
        t.update({k + "_F32": table(src, k, True) for k in ("F2C_DIAG", "F2C_BLOCK", "C2F_DIAG", "C2F_BLOCK")})
        ops.append((name, t, jf, jc, odd))
    with open(os.path.join(ROOT, "summationbyparts_b200", "csrc", "interp_coefficients.h"), "w") as f:
        f.write(emit(ops, "SBPI_", "", "Interpolation operator tables of the 2:1 block interfaces."))
    with open(os.path.join(HERE, "oracle_interp_coefficients.h"), "w") as f:
        f.write(emit(ops, "ORCI_", "", "Interpolation operator tables (oracle copy; test infrastructure only)."))


if __name__ == "__main__":
    main()
