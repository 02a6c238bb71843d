"""Shared test helpers: build the oracle counterpart of a GPU system description."""
import numpy as np


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def oracle_blocks(blocks):
    out = []
    for b in blocks:
        ox, oe = b.op.ids
        out.append(dict(x=b.x, y=b.y, op_xi=ox, op_eta=oe, bc=list(b.bc)))
    return out


def oracle_vortex(params):
    return [dict(x0=v.x0, y0=v.y0, rstar=v.rstar, eps=v.eps) for v in params.vortices], params.mach


def oracle_system(orc, blocks, vortex, gamma=1.4, fast=True):
    s = orc.System(oracle_blocks(blocks), gamma=gamma, fast=fast)
    vs, mach = oracle_vortex(vortex)
    s.set_vortex(vs, mach)
    return s


def physical_state(x, y, seed=3, amp=0.02):
    """A smooth, non-trivial, positive state on a grid: the standard vortex plus a smooth
    perturbation, so every term of the RHS is exercised."""
    from summationbyparts_b200 import workloads
    from oracle import oracle as orc
    q = orc.vortex([dict(x0=-0.7, y0=0.3, rstar=0.6, eps=1.2)], 0.55, 1.4, 0.0, x, y)
    u = workloads.uniform01(seed, 4)
    for c in range(4):
        q[c] = q[c] * (1.0 + amp * np.sin(1.3 * x + 2.0 * u[c]) * np.cos(0.7 * y - u[c]))
    return q
