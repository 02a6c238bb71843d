"""Learned correction of a coarse vortex solve (configuration 4).

A coarse 64 x 64 Upwind4 solve in compensated FP32 is corrected by a 5-layer 3x3
convolutional network (4 -> 32 -> 32 -> 32 -> 32 -> 4 channels, GELU; the library's BF16
tensor-core kernels with FP32 accumulation, ``sbp_cnn_*``) toward the restriction of a fine
256 x 256 Upwind9 FP64 solve.  The network is trained on coarse/fine pairs the solver itself
generates; vortex parameters are drawn like the batched ensemble's (centre ~ U[-2,2]^2,
eps ~ U[0.5,1.5], Mach ~ U[0.3,0.7], r* = the ensemble radius) from SplitMix64 seed 2, on the
warped single block of the ensemble, to t = 2 with dt = 0.2 / (n - 1).

Restriction (fine -> coarse): both grids are linspace grids of the same warped map, so the
fine solution is interpolated in the computational coordinates: tensor-product 6-point
Lagrange interpolation at the coarse nodes (``sbp_restrict_linspace``; exact for degree-5
polynomials in each direction).  64 and 256 points do not nest (255 / 63 is not an integer)
and the reference has no 4:1 operator, so this is stated here as the choice made.

Fallback: the indicator of a case is a residual of the corrected output, the relative L2 size
of the network's correction, |corrected - coarse| / |coarse|.  The network learned corrections
of the sizes the training cases needed; a case that it corrects by more than ``FALLBACK_FACTOR``
times the largest correction it applies to any training case is outside what it was trained on,
and is solved on the fine grid instead (the fine FP64 solve is both the error reference and the
fallback).
The indicator costs one norm per case, no second solve.

    python -m summationbyparts_b200.learned --pairs 4096 --heldout 512 --epochs 40 --json out.json
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import time

import numpy as np

from . import _capi, workloads
from ._capi import F64, check
from .operators import BY_ID, UPWIND4, UPWIND9
from .system import BC_VORTEX, BlockSpec, BlockSystem

COARSE, FINE = 64, 256
PAIR_SEED = 2
FALLBACK_FACTOR = 1.5
T_END = 2.0


def draws(n: int, first: int = 0) -> list[workloads.Instance]:
    """Vortex parameters of cases first .. first + n - 1 (SplitMix64 seed 2)."""
    return workloads.ensemble_instances(n, seed=PAIR_SEED, first=first)


def _torch():
    import torch
    return torch


def solve(cases, side: int, op_id: int, precision: str, device: int = 0):
    """Solve every case to t = 2 on a side x side warped block with operator op_id, all cases in
    one batched system.  Returns (state [n][4][side][side] f64 on the device, GPU seconds of the
    time stepping)."""
    torch = _torch()
    blocks = []
    for i, _ in enumerate(cases):
        x, y = workloads.warped(-5.0, 5.0, side, -5.0, 5.0, side)
        blocks.append(BlockSpec(x, y, BY_ID[op_id](), [(BC_VORTEX, 0)] * 4, i))
    s = BlockSystem(blocks, len(cases), precision, 1.4, device)
    try:
        dt = 0.2 / (side - 1)
        for k, c in enumerate(cases):
            s.set_vortex(c.vortex, k)
            s.set_dt(dt, k)
        s.init_vortex(0.0)
        stream = torch.cuda.Stream(device)
        s.set_stream(stream.cuda_stream)
        steps = int(round(T_END / dt))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(device)
        e0.record(stream)
        s.advance(steps)
        e1.record(stream)
        e1.synchronize()
        out = torch.empty((len(cases), 4, side, side), dtype=torch.float64, device=f"cuda:{device}")
        s.get_state_all_device(out.data_ptr(), F64)
        return out, e0.elapsed_time(e1) / 1e3
    finally:
        s.close()


def restrict(fine, nc: int = COARSE):
    """Tensor-product 6-point Lagrange restriction of [n][4][nf][nf] to [n][4][nc][nc] (f64)."""
    torch = _torch()
    n, _, nf, _ = fine.shape
    out = torch.empty((n, 4, nc, nc), dtype=torch.float64, device=fine.device)
    check(_capi.lib.sbp_restrict_linspace(n, nf, nc, ctypes.c_void_p(fine.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                          ctypes.c_void_p(torch.cuda.current_stream(fine.device).cuda_stream)))
    return out


def rel_l2(a, b) -> np.ndarray:
    """Per case |a - b| / |b| over the 4 component planes (device f64 tensors [n][4][m][m])."""
    torch = _torch()
    n = a.shape[0]
    pts = a.shape[2] * a.shape[3]
    out = torch.empty(n, dtype=torch.float64, device=a.device)
    st = torch.cuda.current_stream(a.device)
    check(_capi.lib.sbp_rel_l2_images(n, pts, ctypes.c_void_p(a.data_ptr()), F64, 4 * pts,
                                      ctypes.c_void_p(b.data_ptr()), F64, 4 * pts, ctypes.c_void_p(out.data_ptr()),
                                      ctypes.c_void_p(st.cuda_stream)))
    st.synchronize()
    return out.cpu().numpy()


class CorrectionNet:
    """The correction network (``sbp_cnn``): parameters, Adam state and activation buffers for
    batches of up to max_batch coarse states."""

    def __init__(self, max_batch: int = 64, seed: int = 0, device: int = 0):
        torch = _torch()
        self.max_batch = max_batch
        self.device = device
        h = ctypes.c_void_p()
        check(_capi.lib.sbp_cnn_create(device, max_batch, seed, ctypes.byref(h)))
        self.h = h
        self.nparams = _capi.lib.sbp_cnn_param_count(self.h)
        self.norm = None

    def close(self) -> None:
        if getattr(self, "h", None):
            _capi.lib.sbp_cnn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- parameters
    def params(self) -> np.ndarray:
        p = np.empty(self.nparams, dtype=np.float32)
        check(_capi.lib.sbp_cnn_get_params(self.h, p.ctypes.data_as(ctypes.c_void_p)))
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.nparams
        check(_capi.lib.sbp_cnn_set_params(self.h, p.ctypes.data_as(ctypes.c_void_p)))

    def set_normalisation(self, in_mean, in_scale, out_scale) -> None:
        arrs = [np.ascontiguousarray(v, dtype=np.float32) for v in (in_mean, in_scale, out_scale)]
        self.norm = [a.astype(np.float64) for a in arrs]
        check(_capi.lib.sbp_cnn_set_normalisation(self.h, *[a.ctypes.data_as(ctypes.c_void_p) for a in arrs]))

    def fit_normalisation(self, coarse, fine_r) -> None:
        """Per component: input mean and standard deviation of the coarse states, output scale the
        RMS of the correction (fine_r - coarse)."""
        torch = _torch()
        c = coarse.transpose(0, 1).reshape(4, -1)
        d = (fine_r - coarse).transpose(0, 1).reshape(4, -1)
        mean = c.mean(dim=1)
        std = c.std(dim=1).clamp_min(1e-6)
        rms = torch.sqrt((d * d).mean(dim=1)).clamp_min(1e-12)
        self.set_normalisation(mean.cpu().numpy(), std.cpu().numpy(), rms.cpu().numpy())

    # -- passes (coarse, fine_r: contiguous device f64 tensors [n][4][64][64])
    def _sync_inputs(self):
        """Launch on torch's current stream: the inputs were made there, and torch's caching
        allocator may hand their memory to the next tensor as soon as they are released, which
        is safe only for work ordered on that stream."""
        st = _torch().cuda.current_stream(self.device)
        check(_capi.lib.sbp_cnn_set_stream(self.h, ctypes.c_void_p(st.cuda_stream)))
        self.stream = st

    def gradients(self, coarse, fine_r):
        self._sync_inputs()
        n = coarse.shape[0]
        loss = ctypes.c_float()
        g = np.empty(self.nparams, dtype=np.float32)
        check(_capi.lib.sbp_cnn_gradients(self.h, n, ctypes.c_void_p(coarse.data_ptr()), F64, 4 * COARSE * COARSE,
                                          ctypes.c_void_p(fine_r.data_ptr()), ctypes.byref(loss),
                                          g.ctypes.data_as(ctypes.c_void_p)))
        return loss.value, g

    def output(self, coarse):
        """Network output y [n][64*64][8] (f32, channels 0..3 used) for a batch."""
        torch = _torch()
        self._sync_inputs()
        n = coarse.shape[0]
        y = torch.empty((n, COARSE * COARSE, 8), dtype=torch.float32, device=coarse.device)
        check(_capi.lib.sbp_cnn_forward(self.h, n, ctypes.c_void_p(coarse.data_ptr()), F64, 4 * COARSE * COARSE))
        check(_capi.lib.sbp_cnn_output(self.h, n, ctypes.c_void_p(y.data_ptr())))
        self.stream.synchronize()
        return y

    def train_step(self, coarse, fine_r, lr: float, want_loss: bool = False):
        self._sync_inputs()
        n = coarse.shape[0]
        loss = ctypes.c_float(float("nan"))
        check(_capi.lib.sbp_cnn_train_step(self.h, n, ctypes.c_void_p(coarse.data_ptr()), F64, 4 * COARSE * COARSE,
                                           ctypes.c_void_p(fine_r.data_ptr()), ctypes.c_float(lr),
                                           ctypes.byref(loss) if want_loss else None))
        return loss.value

    def apply(self, coarse):
        """Corrected states (f64 [n][4][64][64]) for any number of coarse states."""
        torch = _torch()
        self._sync_inputs()
        out = torch.empty_like(coarse, dtype=torch.float64)
        for a in range(0, coarse.shape[0], self.max_batch):
            b = min(a + self.max_batch, coarse.shape[0])
            check(_capi.lib.sbp_cnn_apply(self.h, b - a, ctypes.c_void_p(coarse[a].data_ptr()), F64,
                                          4 * COARSE * COARSE, ctypes.c_void_p(out[a].data_ptr())))
        self.stream.synchronize()
        return out

    def fit(self, coarse, fine_r, epochs: int, lr: float = 2e-3, seed: int = 0, batch: int | None = None):
        """Adam over shuffled mini-batches with a cosine learning-rate decay to lr / 20.
        Returns the mean loss of every epoch."""
        torch = _torch()
        batch = batch or self.max_batch
        n = coarse.shape[0]
        rng = np.random.default_rng(seed)
        steps_per_epoch = max(1, n // batch)
        total = epochs * steps_per_epoch
        hist = []
        k = 0
        for _ in range(epochs):
            perm = torch.from_numpy(rng.permutation(n)).to(coarse.device)
            losses = []
            for s in range(steps_per_epoch):
                idx = perm[s * batch:(s + 1) * batch]
                cb = coarse.index_select(0, idx).contiguous()
                fb = fine_r.index_select(0, idx).contiguous()
                rate = lr * (0.05 + 0.95 * 0.5 * (1.0 + math.cos(math.pi * k / max(1, total - 1))))
                losses.append(self.train_step(cb, fb, rate, want_loss=(s == steps_per_epoch - 1)))
                k += 1
            hist.append(float(np.nanmean(losses)))
        return hist


def make_pairs(count: int, first: int = 0, fine: int = FINE, chunk: int = 512, device: int = 0):
    """Coarse f32c Upwind4 states and restricted fine f64 Upwind9 states of cases first ..
    first + count - 1, with the GPU seconds of each kind of solve."""
    torch = _torch()
    coarse_l, fine_l = [], []
    tc = tf = 0.0
    for a in range(0, count, chunk):
        cases = draws(min(chunk, count - a), first + a)
        c, t = solve(cases, COARSE, UPWIND4, "f32c", device)
        tc += t
        f, t = solve(cases, fine, UPWIND9, "f64", device)
        tf += t
        coarse_l.append(c)
        fine_l.append(restrict(f))
        del f
    return torch.cat(coarse_l), torch.cat(fine_l), tc, tf


def indicator(corrected, coarse):
    """Fallback indicator per case: the relative L2 size of the network's correction."""
    return rel_l2(corrected, coarse)


def run(pairs: int, heldout: int, epochs: int, fine: int = FINE, lr: float = 2e-3, seed: int = 0,
        max_batch: int = 64, device: int = 0, fallback_factor: float = FALLBACK_FACTOR) -> dict:
    """Train on `pairs` cases, evaluate on the next `heldout` cases; returns the report."""
    torch = _torch()
    t0 = time.perf_counter()
    train_c, train_f, _, tf_train = make_pairs(pairs, 0, fine, device=device)
    t_data = time.perf_counter() - t0

    net = CorrectionNet(max_batch=max_batch, seed=seed, device=device)
    net.fit_normalisation(train_c, train_f)
    torch.cuda.synchronize(device)
    t1 = time.perf_counter()
    hist = net.fit(train_c, train_f, epochs, lr=lr, seed=seed)
    torch.cuda.synchronize(device)
    t_train = time.perf_counter() - t1
    threshold = fallback_factor * float(indicator(net.apply(train_c), train_c).max())

    # held-out cases: the fine solve is the error reference (and the fallback); the coarse path is timed
    cases = draws(heldout, pairs)
    coarse, t_coarse = solve(cases, COARSE, UPWIND4, "f32c", device)
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record()
    corrected = net.apply(coarse)
    e1.record()
    ind = indicator(corrected, coarse)
    e2.record()
    e2.synchronize()
    t_net = e0.elapsed_time(e1) / 1e3
    t_ind = e1.elapsed_time(e2) / 1e3
    fine_state, t_fine = solve(cases, fine, UPWIND9, "f64", device)
    fine_r = restrict(fine_state)
    del fine_state
    flagged = [k for k in range(heldout) if ind[k] > threshold]
    t_fallback = 0.0
    final = corrected.clone()
    if flagged:
        fb_state, t_fallback = solve([cases[k] for k in flagged], fine, UPWIND9, "f64", device)
        fb_r = restrict(fb_state)
        for j, k in enumerate(flagged):
            final[k] = fb_r[j]
    err_coarse = rel_l2(coarse, fine_r)
    err_corr = rel_l2(corrected, fine_r)
    err_final = rel_l2(final, fine_r)
    t_path = t_coarse + t_ind + t_net + t_fallback
    net.close()
    return {
        "config": {"coarse": f"{COARSE}x{COARSE} Upwind4 compensated f32", "fine": f"{fine}x{fine} Upwind9 f64",
                   "t_end": T_END, "pairs": pairs, "heldout": heldout, "epochs": epochs, "batch": max_batch,
                   "lr": lr, "seed": PAIR_SEED, "restriction": "tensor-product 6-point Lagrange in (xi, eta)",
                   "network": "5 x conv3x3 4-32-32-32-32-4, GELU, bf16 activations, f32 accumulation "
                              "on the tcgen05 tensor cores (convolutions and weight gradients)",
                   "fallback": f"relative size of the network's correction > {fallback_factor} x training maximum"},
        "train": {"loss_first_epoch": hist[0], "loss_last_epoch": hist[-1], "seconds": t_train,
                  "data_seconds": t_data, "fine_solve_gpu_seconds": tf_train},
        "heldout": {
            "rel_l2_coarse_vs_fine_median": float(np.median(err_coarse)),
            "rel_l2_coarse_vs_fine_max": float(err_coarse.max()),
            "rel_l2_corrected_vs_fine_median": float(np.median(err_corr)),
            "rel_l2_corrected_vs_fine_max": float(err_corr.max()),
            "rel_l2_final_vs_fine_median": float(np.median(err_final)),
            "rel_l2_final_vs_fine_max": float(err_final.max()),
            "error_reduction_median": float(np.median(err_coarse / np.maximum(err_corr, 1e-300))),
            "fallbacks": len(flagged), "threshold": threshold,
            "seconds_fine_path": t_fine,
            "seconds_learned_path": t_path,
            "seconds_learned_parts": {"coarse_u4": t_coarse, "network": t_net, "indicator": t_ind,
                                      "fallback": t_fallback},
            "speedup_time_to_solution": t_fine / t_path,
        },
    }


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--pairs", type=int, default=4096)
    p.add_argument("--heldout", type=int, default=512)
    p.add_argument("--epochs", type=int, default=40)
    p.add_argument("--fine", type=int, default=FINE)
    p.add_argument("--lr", type=float, default=2e-3)
    p.add_argument("--json", default="")
    a = p.parse_args()
    rep = run(a.pairs, a.heldout, a.epochs, a.fine, a.lr)
    s = json.dumps(rep, indent=1)
    print(s)
    if a.json:
        with open(a.json, "w") as f:
            f.write(s + "\n")


if __name__ == "__main__":
    main()
