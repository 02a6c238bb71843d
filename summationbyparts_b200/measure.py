"""Measurements of the parity configurations other than the bench's batched ensemble.

    python -m summationbyparts_b200.measure operators   # configuration 1: operator HBM GB/s
    python -m summationbyparts_b200.measure config0     # configuration 0: 64 x 64 Upwind4 vortex
    python -m summationbyparts_b200.measure config2     # configuration 2: 6-block Upwind9 vortex

Each prints one JSON line.  Times are CUDA events on the launching stream after warm-up;
operator launches alternate between two field sets larger than L2 (4 fields x 4096^2 f64 is
537 MB) so every launch reads its input from HBM.

* operators: diffxi, diffeta (and dissxi, disseta for the upwind operators) of Upwind4, Upwind9
  and SBP8 on 4 fields of 4096 x 4096 (SplitMix64 seed 0, U[-1, 1)), in f64 and f32; one launch
  covers the 4 fields.  Algorithmic bytes: one read and one write per point and field (16 B in
  f64, 8 B in f32); GB/s against the measured copy bandwidth in MEASURED_PEAKS.json.
* config0: 100 RK4 steps of the single 64 x 64 Cartesian block (vortex SATs), f64 and f32c;
  point-updates/s (latency-bound: 4,096 points).
* config2: 500 RK4 steps of the 6-block layout of workloads.multiblock (Grid interfaces,
  vortex outer edges, Upwind9), f64 and f32c; point-updates/s and the f32c error against f64.
"""
from __future__ import annotations

import argparse
import json
import os

import numpy as np

from . import workloads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def operators(reps: int = 10) -> dict:
    import torch

    from .operators import SBP8, Upwind4, Upwind9
    n = 4096
    base = torch.from_numpy(workloads.operator_fields(n, 4, 0)).cuda()
    peak, kind = _peak()
    out = {"config": "4 fields x 4096 x 4096, SplitMix64 seed 0, U[-1,1)", "peak_gbs": peak,
           "peak_source": kind, "results": []}
    for dtype, bpp in ((torch.float64, 16), (torch.float32, 8)):
        a = [base.to(dtype).contiguous(), (base.flip(1) * 0.5).to(dtype).contiguous()]
        f = [torch.empty_like(a[0]), torch.empty_like(a[0])]
        for op in (Upwind4(), Upwind9(), SBP8()):
            fns = [("diffxi", op.diffxi), ("diffeta", op.diffeta)]
            if hasattr(op, "dissxi"):
                fns += [("dissxi", op.dissxi), ("disseta", op.disseta)]
            for name, fn in fns:
                for i in range(3):
                    fn(a[i % 2], f[i % 2])
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                for i in range(reps):
                    fn(a[i % 2], f[i % 2])
                e1.record()
                e1.synchronize()
                ms = e0.elapsed_time(e1) / reps
                gbs = 4 * n * n * bpp / (ms / 1e3) / 1e9
                out["results"].append({"op": type(op).__name__, "fn": name, "dtype": str(dtype).split(".")[-1],
                                       "ms": ms, "gbs": gbs, "frac": gbs / peak})
    return out


def _system(blocks, precision, vortex=workloads.STANDARD_VORTEX):
    from .system import BlockSystem
    s = BlockSystem(blocks, 1, precision, 1.4)
    s.set_vortex(vortex)
    s.init_vortex(0.0)
    return s


def _timed(s, steps):
    import torch
    st = torch.cuda.Stream()
    s.set_stream(st.cuda_stream)
    s.advance(5)
    s.init_vortex(0.0)
    s.set_time(0.0)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    s.advance(steps)
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3


def config0() -> dict:
    c = workloads.Config0()
    res = {"config": "64x64 Cartesian, Upwind4, vortex SATs, 100 RK4 steps, dt = 0.2/63", "runs": {}}
    for prec in ("f64", "f32c"):
        s = _system(c.blocks(), prec)
        s.set_dt(c.dt)
        sec = _timed(s, c.steps)
        res["runs"][prec] = {"seconds": sec, "point_updates_per_s": 64 * 64 * c.steps / sec,
                             "us_per_step": sec / c.steps * 1e6, "error_vs_vortex": float(s.errors()[0])}
        s.close()
    return res


def config2() -> dict:
    blocks = workloads.multiblock()
    dt = workloads.multiblock_dt(blocks)
    pts = sum(b.x.size for b in blocks)
    res = {"config": f"6 warped Upwind9 blocks ({pts} points), Grid interfaces, vortex outer edges, "
                     f"500 RK4 steps, dt = {dt}", "runs": {}}
    states = {}
    for prec in ("f64", "f32c"):
        s = _system(blocks, prec)
        s.set_dt(dt)
        sec = _timed(s, 500)
        states[prec] = np.concatenate([s.state(b).ravel() for b in range(len(blocks))])
        res["runs"][prec] = {"seconds": sec, "point_updates_per_s": pts * 500 / sec, "us_per_step": sec / 500 * 1e6,
                             "error_vs_vortex": float(s.errors()[0]),
                             "launches_per_step": s.launches_per_step()}
        s.close()
    d = states["f32c"] - states["f64"]
    res["f32c_vs_f64_rel_l2"] = float(np.linalg.norm(d) / np.linalg.norm(states["f64"]))
    return res


def main():
    p = argparse.ArgumentParser()
    p.add_argument("what", choices=["operators", "config0", "config2"])
    a = p.parse_args()
    print(json.dumps({"operators": operators, "config0": config0, "config2": config2}[a.what]()))


if __name__ == "__main__":
    main()
