"""Writes tests/golden/sbp_golden.npz: seeded inputs and the oracle's outputs for them.

The reference (a Rust workspace) ships no golden vectors and cannot be built here; its tests pin
the operators and the solver by analytic properties, which tests/test_oracle_kat.py restates on
the oracle.  This file freezes the pinned oracle's answers on small seeded cases, so that
tests/test_golden_cpu.py catches any later drift of the oracle and tests/test_gpu_golden.py
compares the CUDA path with fixed numbers:

* op_in_<dtype>: a 19 x 26 field of SplitMix64 U[-1, 1) values (seed 500 f64, 501 f32);
  op_<id>_<fn>_<dtype>: SbpOperator2d::diffxi / diffeta and UpwindOperator2d::dissxi /
  disseta (sbp/src/operators.rs:55-106) of every operator id 0..5 on it, in that dtype;
* met_x, met_y: a warped 29 x 21 grid; met_<xi>_<eta>: Metrics::new (sbp/src/grid.rs:95-140)
  for the operator pairs (0, 0) and (2, 3), planes detJ, J xi_x, J xi_y, J eta_x, J eta_y;
* step_x, step_y, step_q0: a warped 45 x 38 grid and a smooth positive state on it;
  step_<op>: one RK4 step of dt 0.01 of euler::System with periodic (This) boundaries
  (euler/src/lib.rs:124-147, utils/integrate/src/lib.rs:176-222) for Upwind4 and Upwind9.

Run from the repository root: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

OUT = os.path.join(HERE, "sbp_golden.npz")
OP_SHAPE = (19, 26)
OP_FUNCS = ("diffxi", "diffeta", "dissxi", "disseta")
MET_PAIRS = ((0, 0), (2, 3))
STEP_OPS = ("Upwind4", "Upwind9")
STEP_DT = 0.01
DTYPES = (("f64", np.float64, 500), ("f32", np.float32, 501))


def oracle_op(orc, op, fn, a):
    d, k = {"diffxi": (orc.XI, orc.DIFF), "diffeta": (orc.ETA, orc.DIFF), "dissxi": (orc.XI, orc.DISS),
            "disseta": (orc.ETA, orc.DISS)}[fn]
    return orc.op_apply(op, d, k, a)


def funcs_of(orc, op):
    upw = orc.op_shape(op)[4]
    return OP_FUNCS if upw else OP_FUNCS[:2]


def step_blocks(op_name, x, y):
    from summationbyparts_b200 import operators
    from summationbyparts_b200.system import BlockSpec
    return [BlockSpec(x, y, getattr(operators, op_name)(), [(0, 0)] * 4, 0)]


def oracle_step(orc, op_name, x, y, q0):
    from _helpers import oracle_system
    from summationbyparts_b200 import workloads
    o = oracle_system(orc, step_blocks(op_name, x, y), workloads.STANDARD_VORTEX)
    o.set_state(0, q0)
    o.advance(1, STEP_DT)
    return o.state(0)


def compute(orc):
    """Every fixture array, from the seeded inputs and the oracle."""
    from _helpers import physical_state
    from summationbyparts_b200 import workloads
    d = {}
    n = OP_SHAPE[0] * OP_SHAPE[1]
    for name, dt, seed in DTYPES:
        a = workloads.uniform_pm1(seed, n).reshape(OP_SHAPE).astype(dt)
        d[f"op_in_{name}"] = a
        for op in range(6):
            for fn in funcs_of(orc, op):
                d[f"op_{op}_{fn}_{name}"] = oracle_op(orc, op, fn, a)
    x, y = workloads.warped(-5.0, 5.0, 29, -4.0, 5.0, 21)
    d["met_x"], d["met_y"] = x, y
    for opx, ope in MET_PAIRS:
        d[f"met_{opx}_{ope}"] = orc.metrics(opx, ope, x, y)
    x, y = workloads.warped(-5.0, 5.0, 45, -5.0, 5.0, 38)
    q0 = physical_state(x, y)
    d["step_x"], d["step_y"], d["step_q0"] = x, y, q0
    for op_name in STEP_OPS:
        d[f"step_{op_name}"] = oracle_step(orc, op_name, x, y, q0)
    return d


def main():
    from oracle import oracle as orc
    orc.lib()
    d = compute(orc)
    np.savez_compressed(OUT, **d)
    print(f"wrote {OUT}: {len(d)} arrays, {os.path.getsize(OUT)} bytes")


if __name__ == "__main__":
    main()
