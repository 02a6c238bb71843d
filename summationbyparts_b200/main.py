"""The multigrid driver on the GPU: the reference's `multigrid` binary (multigrid/src/main.rs)
for configuration files of the same format (see config.py).

    python -m summationbyparts_b200.main CONFIG [-o OUTPUT] [-n N] [--timings] [--error]
                                         [--no-progressbar] [--output-json] [--distribute]
                                         [--precision f64|f32c] [--device D]

Steps as main.rs:52-163 does: dt = max_dt(), ntime = round(integration_time / dt) RK4 steps,
outputs at step 0 and at the end, then "Time elapsed: <s> seconds" (--timings, the compute
loop, device-synchronised) and "Total error: <e>" (--error, the sum over grids of h2_err
against the initial-condition vortex), or with --output-json the same as one json line
{"filename": ..., "time_elapsed": {"secs": s, "nanos": ns}, "error": e}.

The output file (-o, default output.hdf) is HDF5 as the reference writes it: root dataset `t`
(u64 step numbers of the outputs) and per grid a group with `x`, `y`, a soft link `t` -> `/t` and
`rho`, `rhou`, `rhov`, `e` of shape (outputs, ny, nx), written by this package's own HDF5 writer
(hdf5.py; contiguous, uncompressed datasets).  Differences: there is no progress bar;
--distribute is accepted and changes nothing (every block of every grid already runs in one
launch per stage); --precision f32c selects the compensated-f32 form.
"""
from __future__ import annotations

import argparse
import decimal
import json
import os
import sys
import time

import numpy as np

from . import config as cfgmod
from . import hdf5
from . import multigrid as mg


def rust_lower_exp(x: float) -> str:
    """Rust's `{:e}` of an f64: shortest round-trip digits, d.ddd, then e<exponent>."""
    if x == 0.0:
        return "0e0" if not np.signbit(x) else "-0e0"
    if not np.isfinite(x):
        return "NaN" if x != x else ("inf" if x > 0 else "-inf")
    d = decimal.Decimal(repr(abs(x)))
    _, digits, exp = d.as_tuple()
    digits = "".join(str(v) for v in digits).rstrip("0") or "0"
    e10 = exp + len("".join(str(v) for v in d.as_tuple()[1])) - 1
    mant = digits[0] + ("." + digits[1:] if len(digits) > 1 else "")
    return ("-" if x < 0 else "") + mant + "e" + str(e10)


def rust_display(x: float) -> str:
    """Rust's `{}` of an f64: shortest round-trip digits without an exponent."""
    r = repr(float(x))
    if "e" in r or "E" in r:
        r = format(decimal.Decimal(r), "f")
    return r


class Snapshots:
    """The output file of the run: the state of every grid at step 0, at every intermediate output
    and at the end (System::output, multigrid/src/system.rs:591-616), written as HDF5 by
    `hdf5.write_snapshots` when the run ends."""

    def __init__(self, path: str, names, grids):
        self.path = path
        self.names = names
        self.grids = grids
        self.times = []
        self.frames = []

    def output(self, sys_, step: int):
        self.times.append(step)
        self.frames.append([sys_.field(b) for b in range(len(self.names))])

    def write(self):
        hdf5.write_snapshots(self.path, self.names, self.grids, self.times, self.frames)


def main(argv=None) -> int:
    p = argparse.ArgumentParser(description="Options for configuring and running the solver")
    p.add_argument("json")
    p.add_argument("-o", "--output", default="output.hdf", help="name of output file")
    p.add_argument("-n", "--number-of-outputs", type=int, default=None, help="number of outputs to save")
    p.add_argument("--timings", action="store_true", help="print the time to complete, taken in the compute loop")
    p.add_argument("--error", action="store_true", help="print error at the end of the run")
    p.add_argument("--no-progressbar", action="store_true", help="disable the progressbar")
    p.add_argument("--output-json", action="store_true",
                   help="output information regarding time elapsed and error in json format")
    p.add_argument("--distribute", action="store_true", help="distribute the computation (no effect on the GPU)")
    p.add_argument("--precision", default="f64", choices=["f64", "f32c"])
    p.add_argument("--device", type=int, default=0)
    a = p.parse_args(argv)
    try:
        with open(a.json) as f:
            rt = cfgmod.into_runtime(cfgmod.loads(f.read()))
    except (cfgmod.ConfigError, KeyError, TypeError, ValueError) as e:
        print(f"Configuration could not be read: {e}", file=sys.stderr)
        return 0
    import torch

    s = mg.System(rt.grids, rt.initial, rt.gamma, a.precision, a.device, boundary_vortex=rt.boundary_vortex,
                  boundary_expressions=rt.boundary_expressions)
    dt = s.max_dt()
    s.set_dt(dt)
    ntime = int(round(rt.integration_time / dt))
    snaps = Snapshots(a.output, rt.names, rt.grids)
    snaps.output(s, 0)
    torch.cuda.synchronize(a.device)
    t0 = time.perf_counter()
    # main.rs:116-125: steps_between_outputs = max(n / ntime, 1) and the next output step is
    # max(itime + steps_between_outputs, ntime): one advance to ntime
    itime = 0
    while itime < ntime:
        nexttime = max(itime + (max((a.number_of_outputs or ntime) // ntime, 1)), ntime)
        s.advance(nexttime - itime)
        itime = nexttime
        if itime != ntime:
            snaps.output(s, itime)
    torch.cuda.synchronize(a.device)
    elapsed = time.perf_counter() - t0
    snaps.output(s, ntime)
    snaps.write()
    err = s.error() if a.error else None
    if a.output_json:
        info = {"filename": a.output}
        if a.timings:
            secs = int(elapsed)
            info["time_elapsed"] = {"secs": secs, "nanos": int(round((elapsed - secs) * 1e9))}
        if err is not None:
            info["error"] = err
        print(json.dumps(info, separators=(",", ":")))
    else:
        if a.timings:
            print(f"Time elapsed: {rust_display(elapsed)} seconds")
        if err is not None:
            print(f"Total error: {rust_lower_exp(err)}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
