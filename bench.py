#!/usr/bin/env python
"""Benchmark: Euler RK4 point-updates/s on one B200, batched FP32 (compensated) vs plain FP64.

Workload (one "step" = one RK4 step of every instance): the batched ensemble -- 512
independent isentropic-vortex solves drawn from SplitMix64 seed 1 (centre ~ U[-2,2]^2,
eps ~ U[0.5,1.5], Mach ~ U[0.3,0.7], side ~ U{48..257}, Upwind4/Upwind9 50/50) on single
warped curvilinear blocks with vortex SATs on every edge, each with its own dt = 0.2/(side-1).
Synthetic inputs: the reference has no dataset.  Under torchrun each rank runs its own 512
instances (the next 512 of the same stream): weak scaling, no data-path collective.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Euler RK4 point-updates/s, 1 B200: batched FP32 vs plain FP64 at same L2 error"
UNIT = "point-updates/s"
# Algorithmic HBM bytes per point-update of the fused stage design (sum over the 4 stage
# launches of the state, accumulator and metric planes each launch must read and write once).
BYTES_PER_POINT_UPDATE = {"f32c": 384, "f64": 672}
# The same per stage launch (stage 0..3).  f64: stage 0 reads the step-start state and the
# metrics and writes the accumulator and the next stage input; stages 1 and 2 also read the
# accumulator and the step-start state; stage 3 reads the accumulator and writes the new state.
# f32c (state as a (hi, lo) f32 pair, the step's increment accumulated in one f32 array):
# stage 0 reads the state's hi part and the metrics, writes the next stage input and the
# increment; stages 1 and 2 read the stage input, metrics, increment and hi part and write the
# next input and the increment; stage 3 reads the stage input, metrics, increment, hi and lo
# parts and writes the new hi and lo parts.
BYTES_PER_POINT_STAGE = {"f32c": (68, 100, 100, 116), "f64": (136, 200, 200, 136)}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=300)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--ninst", type=int, default=512)
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--no-fp64", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--chunks", type=int, default=0,
                   help="instance chunks of the end-to-end call (0: the library default)")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-accuracy", action="store_true")
    p.add_argument("--tiles", default="", help="TY,TX,THREADS: fixed tile schedule instead of the autotuner")
    p.add_argument("--kernel-reps", type=int, default=5, help="repetitions of the per-kernel timing")
    p.add_argument("--kernel-only", action="store_true",
                   help="only the per-kernel timing of the stage kernels (for profiling runs)")
    return p.parse_args()


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")), int(
        os.environ.get("WORLD_SIZE", "1"))


# ------------------------------------------------------------------------------------------
class Clocks:
    """Samples the SM clock and the clock-event (throttle) reasons of this rank's GPU while the
    timed region runs.  NVML is polled every 5 ms from a thread (the timed region can be well
    under a second, shorter than nvidia-smi's sampling loop); the GPU is found by its UUID, so
    CUDA_VISIBLE_DEVICES remapping cannot select another GPU.  Without NVML, nvidia-smi is
    sampled instead and started before the timed region, once its first sample has arrived."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.thread = None
        self.rows = []
        self.source = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        uuid = str(torch.cuda.get_device_properties(self.gpu).uuid)
        for cand in (uuid, "GPU-" + uuid):
            try:
                return pynvml, pynvml.nvmlDeviceGetHandleByUUID(cand)
            except pynvml.NVMLError:
                continue
        raise RuntimeError("no NVML device with this UUID")

    def start(self):
        import threading
        try:
            nv, h = self._nvml_handle()
            bits = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                    nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
            max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.stop_flag = threading.Event()

            def poll():
                while True:
                    try:
                        mhz = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                        r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.rows.append((mhz, max_mhz, ["Active" if r & b else "Not Active" for b in bits]))
                    except nv.NVMLError:
                        pass
                    if self.stop_flag.wait(0.005):
                        break

            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            self.source = "nvml, 5 ms"
            return
        except Exception:
            self.thread = None
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            t0 = time.time()
            while time.time() - t0 < 5.0 and os.path.getsize(self.path) == 0:
                time.sleep(0.02)
            self.source = "nvidia-smi, 50 ms"
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join(timeout=5)
            rows = self.rows
        elif self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            rows = []
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    rows.append((float(f[1]), float(f[2]), f[5:9]))
                except ValueError:
                    continue
            os.unlink(self.path)
        else:
            return None
        if not rows:
            return None
        reasons = sorted({self.NAMES[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows), "source": self.source}


OP_NAMES = {0: "Upwind4", 1: "Upwind4h2", 2: "Upwind9", 3: "Upwind9h2", 4: "SBP4", 5: "SBP8"}


def group_schedule(sysx) -> list:
    """The tile schedule of every operator group (the autotuner's choice, or the fixed one)."""
    out = []
    for g, (ox, oy, pts) in enumerate(sysx.groups()):
        ty, cps, grid = sysx.group_tiles(g)
        out.append({"op_xi": OP_NAMES.get(ox, ox), "op_eta": OP_NAMES.get(oy, oy), "points": pts, "tile_rows": ty,
                    "tile_cols": 32, "ctas_per_sm": "max" if cps < 0 else ("one per tile" if cps == 0 else cps),
                    "grid": grid})
    return out


def measured_hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def recorded_traffic(precision: str):
    """Per-launch DRAM bytes of the stage kernel from the committed ncu summary, scaled per point."""
    path = os.path.join(ROOT, "profiles", "stage_kernel_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return d.get(precision)
    except (OSError, ValueError):
        return None


# ------------------------------------------------------------------------------------------
def build_system(insts, precision, device):
    from summationbyparts_b200 import workloads
    from summationbyparts_b200.system import BlockSystem
    blocks = workloads.ensemble_blocks(insts)
    s = BlockSystem(blocks, len(insts), precision, 1.4, device)
    for k, inst in enumerate(insts):
        s.set_vortex(inst.vortex, k)
        s.set_dt(inst.dt, k)
    s.init_vortex(0.0)
    return s


def timed_advance(torch, s, stream, steps, barrier):
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s.advance(steps)
    e1.record(stream)
    e1.synchronize()
    barrier()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def kernel_timing(torch, s, stream, precision, reps):
    """Stage-kernel roofline: every group's stage kernel for each RK4 stage, launched one at a
    time and timed with CUDA events on the system's stream.  Returns algorithmic bytes / kernel
    time over all those launches and the per-launch detail.  Leaves the stage buffers as the
    launches leave them (the system must be re-initialised before its results mean anything)."""
    groups = s.groups()
    per_stage = BYTES_PER_POINT_STAGE[precision]
    for g in range(len(groups)):  # warm-up
        for st in range(4):
            s.launch_stage(g, st)
    torch.cuda.synchronize()
    ev = []
    for _ in range(reps):
        for g, (_, _, pts) in enumerate(groups):
            for st in range(4):
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                s.launch_stage(g, st)
                b.record(stream)
                ev.append((g, st, pts, a, b))
    torch.cuda.synchronize()
    total_bytes = total_ms = 0.0
    detail = {}
    for g, st, pts, a, b in ev:
        ms = a.elapsed_time(b)
        total_bytes += per_stage[st] * pts
        total_ms += ms
        key = f"group{g}_stage{st}"
        detail.setdefault(key, []).append(ms)
    launches = [{"group": g, "op_xi": groups[g][0], "op_eta": groups[g][1], "points": groups[g][2], "stage": st,
                 "algorithmic_bytes": per_stage[st] * groups[g][2],
                 "ms_median": statistics.median(detail[f"group{g}_stage{st}"])}
                for g in range(len(groups)) for st in range(4)]
    return total_bytes / (total_ms / 1e3) / 1e9, total_ms / len(ev), launches


_CPU_SYSTEMS = {}


def cpu_baseline(insts, seconds, nthreads, steps_per_sample=1):
    """The oracle (C++ port of the reference arithmetic) on the host cores: time RK4 steps of a
    bounded sample of instances (several steps of the whole workload when it fits the budget),
    all threads.  Returns (point-updates/s, description)."""
    from oracle import oracle as orc
    from summationbyparts_b200 import workloads
    # calibrate on one small instance
    small = min(insts, key=lambda i: i.side)
    blk = workloads.ensemble_blocks([small])[0]
    s = orc.System([dict(x=blk.x, y=blk.y, op_xi=small.op_id, op_eta=small.op_id, bc=list(blk.bc))], fast=True)
    s.set_vortex([dict(x0=small.x0, y0=small.y0, rstar=workloads.ENSEMBLE_RSTAR, eps=small.eps)], small.mach)
    s.init_vortex(0.0)
    t0 = time.perf_counter()
    s.advance(1, small.dt)
    per_point = (time.perf_counter() - t0) / (small.side ** 2)
    budget_points = seconds * nthreads / max(per_point, 1e-9) / steps_per_sample
    # round-robin sample so the operator and size mix follows the ensemble
    order = insts[::max(1, len(insts) // 64)] + insts
    sample, pts = [], 0
    for inst in order:
        if inst in sample:
            continue
        if pts + inst.side ** 2 > budget_points and sample:
            break
        sample.append(inst)
        pts += inst.side ** 2
    systems = []
    for inst in sample:
        so = _CPU_SYSTEMS.get(id(inst))  # built once per instance, then advanced further by each call
        if so is None:
            b = workloads.ensemble_blocks([inst])[0]
            so = orc.System([dict(x=b.x, y=b.y, op_xi=inst.op_id, op_eta=inst.op_id, bc=list(b.bc))], fast=True)
            so.set_vortex([dict(x0=inst.x0, y0=inst.y0, rstar=workloads.ENSEMBLE_RSTAR, eps=inst.eps)], inst.mach)
            so.init_vortex(0.0)
            _CPU_SYSTEMS[id(inst)] = so
        systems.append(so)
    if len(sample) == len(insts):
        # the whole workload fits the budget: one untimed step on all threads gives the time per
        # step, then as many steps as the budget holds are timed
        t0 = time.perf_counter()
        orc.advance_many(systems, [1] * len(systems), [i.dt for i in sample], nthreads)
        steps_per_sample = max(steps_per_sample, int(seconds / max(time.perf_counter() - t0, 1e-9)))
    t0 = time.perf_counter()
    orc.advance_many(systems, [steps_per_sample] * len(systems), [i.dt for i in sample], nthreads)
    dt = time.perf_counter() - t0
    return pts * steps_per_sample / dt, {"instances": len(sample), "points": pts, "steps": steps_per_sample,
                                         "seconds": dt}


# ------------------------------------------------------------------------------------------
def run_reference(args):
    rank, _, world = env_rank()
    if rank != 0:
        return
    from summationbyparts_b200 import workloads
    insts = workloads.ensemble_instances(args.ninst, seed=1)
    nthreads = os.cpu_count() or 1
    # about two minutes of CPU work in all (at least one RK4 step of the whole sample per step)
    per_step = min(4.0, 120.0 / max(1, args.steps + args.warmup))
    for _ in range(args.warmup):
        cpu_baseline(insts, per_step * 0.25, nthreads)
    vals, descs = [], []
    for _ in range(args.steps):
        v, d = cpu_baseline(insts, per_step, nthreads)
        vals.append(v)
        descs.append(d)
    value = statistics.mean(vals)
    ms = 1e3 * statistics.mean(d["seconds"] for d in descs)
    sample = (f"{descs[0]['instances']} of {len(insts)} instances ({descs[0]['points']} points), "
              f"{descs[0]['steps']} RK4 step(s) per timed step, {nthreads} threads")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "batched ensemble, 512 vortex solves (SplitMix64 seed 1), sides 48-257, "
                                   "Upwind4/Upwind9, vortex SATs", "instances": args.ninst},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    import torch.distributed as dist

    rank, local, world = env_rank()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

        def barrier():
            dist.barrier()
    else:
        def barrier():
            pass

    from summationbyparts_b200 import sharding, workloads
    first, count = sharding.weak_shard(args.ninst, rank)
    insts = workloads.ensemble_instances(count, seed=1, first=first)
    points = workloads.ensemble_points(insts)
    stream = torch.cuda.Stream()
    s32 = build_system(insts, "f32c", local)
    s32.set_stream(stream.cuda_stream)
    fixed = tuple(int(v) for v in args.tiles.split(",")) if args.tiles else None
    if fixed:
        s32.set_tiles(*fixed)
        tiles = fixed
    else:
        tiles = s32.autotune()
    if args.kernel_only:
        s32.advance(1)
        gbs, ms_launch, launches = kernel_timing(torch, s32, stream, "f32c", args.kernel_reps)
        if rank == 0:
            print(json.dumps({"kernel": "stage_kernel", "achieved_gbs": gbs, "ms_per_launch": ms_launch,
                              "launches": launches, "tiles": list(tiles), "points": points}), flush=True)
        s32.close()
        if world > 1:
            dist.destroy_process_group()
        return
    for _ in range(args.warmup):
        s32.advance(1)
    clocks = Clocks(local)
    clocks.start()
    ms = timed_advance(torch, s32, stream, args.steps, barrier)
    clk = clocks.stop()
    tiles32 = group_schedule(s32)  # the schedule that was timed (the accuracy run retires instances)
    ms = sharding.max_over_ranks(ms, dist if world > 1 else None)
    total_points = points * world
    value = total_points * args.steps / (ms / 1e3)
    ms_step = ms / args.steps
    launches = s32.launches_per_step() * args.steps

    # FP64 plain form on the same ensemble
    fp64 = None
    acc = None
    s64 = None
    if not args.no_fp64:
        s64 = build_system(insts, "f64", local)
        s64.set_stream(stream.cuda_stream)
        if fixed:
            s64.set_tiles(*fixed)
            t64 = fixed
        else:
            t64 = s64.autotune()
        for _ in range(args.warmup):
            s64.advance(1)
        ms64 = sharding.max_over_ranks(timed_advance(torch, s64, stream, args.steps, barrier), dist if world > 1 else None)
        v64 = total_points * args.steps / (ms64 / 1e3)
        fp64 = {"value": v64, "ms_per_step": ms64 / args.steps, "tiles": group_schedule(s64),
                "bytes_per_point_update": BYTES_PER_POINT_UPDATE["f64"],
                "achieved_gbs": BYTES_PER_POINT_UPDATE["f64"] * points / (ms64 / args.steps / 1e3) / 1e9,
                "speedup_f32_over_f64": value / v64}

    # end to end through the C ABI with host buffers: per step, upload the state from pinned host
    # memory, advance one RK4 step, read the new state back (euler::System::advance_upwind + field()),
    # as one sbp_system_advance_host call that pipelines the copies and the steps over chunks of
    # instances
    e2e = None
    if not args.no_e2e:
        n = s32.state_count(0)
        host = torch.empty(n, dtype=torch.float64, pin_memory=True)
        s32.get_state_all(host)
        ke = max(3, min(args.steps, 10))
        chunks = 0
        for _ in range(2):
            chunks = s32.advance_host(host, host, 1, nchunks=args.chunks)
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(ke):
            s32.advance_host(host, host, 1, nchunks=args.chunks)
        e1.record(stream)
        e1.synchronize()
        barrier()
        me = sharding.max_over_ranks(e0.elapsed_time(e1), dist if world > 1 else None)
        e2e = {"value": total_points * ke / (me / 1e3), "unit": UNIT, "h2d_bytes_per_step": n * 8,
               "d2h_bytes_per_step": n * 8, "steps": ke, "chunks": chunks,
               "path": "sbp_system_advance_host(q, q, 1): f64 host state in, one RK4 step, f64 host state out "
                       "(= set_state_all + advance(1) + get_state_all), copies and steps pipelined over chunks "
                       "of instances"}

    # per-kernel roofline of the stage kernels, with every instance active (the accuracy run
    # below re-initialises both systems)
    k64 = None
    if s64 is not None:
        k64, _, _ = kernel_timing(torch, s64, stream, "f64", args.kernel_reps)
        if fp64 is not None:
            fp64["stage_kernel_achieved_gbs"] = k64
    achieved, ms_launch, klaunch = kernel_timing(torch, s32, stream, "f32c", args.kernel_reps)

    # same-error check: every instance of both forms to t = 2 (ragged step counts)
    if s64 is not None and not args.no_accuracy:
        import numpy as np
        steps_t2 = [i.steps_to_t2 for i in insts]
        runs = {}
        for name, sysx in (("f32c", s32), ("f64", s64)):
            sysx.init_vortex(0.0)
            sysx.set_time(0.0)
            t0 = time.perf_counter()
            sysx.advance_instances(steps_t2)
            runs[name] = (sysx.errors(), time.perf_counter() - t0)
        e32, e64 = runs["f32c"][0], runs["f64"][0]
        n = s32.state_count(0)
        a = torch.empty(n, dtype=torch.float64, pin_memory=True)
        b = torch.empty(n, dtype=torch.float64, pin_memory=True)
        s32.get_state_all(a)
        s64.get_state_all(b)
        rel = np.abs(e32 - e64) / e64
        acc = {"t_end": 2.0, "instances": len(insts), "point_updates": int(sum(i.side ** 2 * i.steps_to_t2 for i in insts)),
               "seconds_to_t2_f32c": runs["f32c"][1], "seconds_to_t2_f64": runs["f64"][1],
               "l2_err_vs_exact_f64_median": float(np.median(e64)), "l2_err_vs_exact_f64_max": float(e64.max()),
               "l2_err_vs_exact_f32c_median": float(np.median(e32)), "l2_err_vs_exact_f32c_max": float(e32.max()),
               "err_rel_diff_f32c_vs_f64_max": float(rel.max()),
               "state_rel_l2_f32c_vs_f64": (a - b).norm().item() / b.norm().item()}
        # per instance (one block each, packed (4, side, side) in instance order)
        per, off = [], 0
        for inst in insts:
            m = 4 * inst.side * inst.side
            per.append((a[off:off + m] - b[off:off + m]).norm().item() / b[off:off + m].norm().item())
            off += m
        acc["state_rel_l2_f32c_vs_f64_per_instance_median"] = float(np.median(per))
        acc["state_rel_l2_f32c_vs_f64_per_instance_max"] = float(np.max(per))
    if s64 is not None:
        s64.close()

    peak, peak_kind = measured_hbm_peak()
    bpp = BYTES_PER_POINT_UPDATE["f32c"]
    launches_stage = (s32.launches_per_step() - 1) // 2  # a stage kernel and an edge kernel per group and stage
    bytes_per_launch = bpp * points / 4.0  # average over the 4 stage launches of a step
    traffic = recorded_traffic("f32c")
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": (traffic * points / 4.0) if traffic else None,
            "kernel": "stage_kernel (fused RK4 stage, compensated f32)",
            "achieved_from": "algorithmic bytes of every group's stage-kernel launch for stages 0-3, "
                             "divided by their CUDA-event durations on the launching stream, "
                             f"{args.kernel_reps} repetitions",
            "ms_per_launch": ms_launch, "launches": klaunch,
            "algorithmic_bytes_per_point_update": bpp, "bytes_per_launch": bytes_per_launch,
            "stage_launches_per_step": launches_stage,
            "whole_step_gbs": bpp * points / (ms_step / 1e3) / 1e9,
            "peak_source": f"{peak_kind} hbm_gbs (copy bandwidth, burst)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        nthreads = os.cpu_count() or 1
        v, d = cpu_baseline(insts, args.cpu_seconds, nthreads)
        cpu = {"value": v, "unit": UNIT, "cores": nthreads, "kind": "port",
               "sample": f"{d['instances']} of {len(insts)} instances ({d['points']} points), "
                         f"{d['steps']} RK4 step(s), {nthreads} threads, {d['seconds']:.1f} s"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "batched ensemble: 512 vortex solves per GPU (SplitMix64 seed 1), sides 48-257, "
                                       "Upwind4/Upwind9 50/50, warped single blocks, vortex SATs, FP32 compensated RK4",
                           "instances_per_gpu": len(insts), "points_per_gpu": points, "precision": "f32c",
                           "tiles": tiles32, "l2": f"inputs larger than L2 (state+metrics "
                                                       f"{points * 4 * (8 + 8 + 4 + 4 + 5) / 1e6:.0f} MB per GPU)",
                           "parallelism": f"ensemble sharded, {world} rank(s), no collective"},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk,
                "fp64_plain": fp64, "accuracy": acc}
        print(json.dumps(line), flush=True)
    s32.close()
    if world > 1:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
