"""GPU tests of the learned correction (configuration 4): the restriction operator, the
network's forward pass and gradients against the CPU oracle (oracle/cnn_oracle.py), the Adam
step, and a small end-to-end run showing what the trained network gains over the uncorrected
coarse solve."""
import numpy as np
import pytest

from oracle import cnn_oracle as co

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def test_restriction_exact_for_quintics():
    torch = _torch()
    from summationbyparts_b200 import learned
    rng = np.random.default_rng(1)
    nf, nc = 256, 64
    s = np.arange(nf) / (nf - 1)
    S = np.arange(nc) / (nc - 1)
    fine = np.empty((2, 4, nf, nf))
    ref = np.empty((2, 4, nc, nc))
    for i in range(2):
        for c in range(4):
            a = rng.standard_normal((6, 6))
            fine[i, c] = np.polynomial.polynomial.polygrid2d(s, s, a)
            ref[i, c] = np.polynomial.polynomial.polygrid2d(S, S, a)
    out = learned.restrict(torch.from_numpy(fine).cuda(), nc).cpu().numpy()
    assert np.max(np.abs(out - ref)) <= 1e-11 * np.max(np.abs(ref))


def _batch(n=2, seed=3):
    """Smooth vortex states on the 64 x 64 warped grid and a smooth 'fine' target near them."""
    from oracle import oracle as orc
    from summationbyparts_b200 import workloads
    x, y = workloads.warped(-5.0, 5.0, 64, -5.0, 5.0, 64)
    rng = np.random.default_rng(seed)
    coarse = np.empty((n, 4, 64, 64))
    for i in range(n):
        coarse[i] = orc.vortex([dict(x0=rng.uniform(-2, 2), y0=rng.uniform(-2, 2), rstar=1.0,
                                     eps=rng.uniform(0.5, 1.5))], rng.uniform(0.3, 0.7), 1.4, 0.0, x, y)
    pert = 1e-3 * np.sin(0.7 * x + 0.3)[None, None] * np.cos(0.5 * y)[None, None] * rng.standard_normal((n, 4, 1, 1))
    return coarse, coarse + pert


def _params(net, seed=7):
    rng = np.random.default_rng(seed)
    layers = co.unpack(np.zeros(net.nparams))
    out = []
    for l, (w, b) in enumerate(layers):
        cin_real = 4 if l == 0 else 32
        cout_real = 4 if l == 4 else w.shape[0]
        w = np.zeros_like(w)
        w[:cout_real, :, :cin_real] = rng.standard_normal((cout_real, 9, cin_real)) * np.sqrt(2.0 / (9 * cin_real))
        b = np.zeros_like(b)
        b[:cout_real] = 0.1 * rng.standard_normal(cout_real)
        out.append((w, b))
    return co.pack(out).astype(np.float32)


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a - b)) / np.linalg.norm(np.ravel(b)))


def test_forward_and_gradients_match_oracle():
    torch = _torch()
    from summationbyparts_b200.learned import CorrectionNet
    coarse, fine_r = _batch()
    net = CorrectionNet(max_batch=4, seed=11)
    p = _params(net)
    net.set_params(p)
    in_mean = np.array([1.0, 0.5, 0.0, 2.5])
    in_scale = np.array([0.05, 0.1, 0.1, 0.2])
    out_scale = np.array([1e-3, 1.2e-3, 0.8e-3, 2e-3])
    net.set_normalisation(in_mean, in_scale, out_scale)
    in_scale32 = net.norm[1]
    out_scale32 = net.norm[2]
    dc = torch.from_numpy(coarse).cuda().contiguous()
    df = torch.from_numpy(fine_r).cuda().contiguous()
    y = net.output(dc).cpu().numpy().reshape(2, 64, 64, 8)
    y_ref, _, _ = co.forward(p.astype(np.float64), coarse, net.norm[0], in_scale32)
    # bf16 activations: the GPU and the oracle round the same quantities; pre-activations are
    # f32 on the GPU and f64 here, so a few activations land on the other side of a rounding
    # boundary.  Bar: 1e-2 relative L2 for the output, 3e-2 for each layer's gradients.
    assert _rel(y[..., :4], y_ref[..., :4]) < 1e-2
    loss, g = net.gradients(dc, df)
    loss_ref, g_ref = co.loss_and_grads(p.astype(np.float64), coarse, fine_r, net.norm[0], in_scale32, out_scale32)
    assert abs(loss - loss_ref) <= 1e-2 * loss_ref
    gl, gl_ref = co.unpack(g), co.unpack(g_ref)
    for l in range(5):
        assert _rel(gl[l][0], gl_ref[l][0]) < 3e-2, l
        assert _rel(gl[l][1], gl_ref[l][1]) < 3e-2, l
    # padded parameters get no gradient
    assert np.all(gl[0][0][:, :, 4:] == 0.0)
    assert np.all(gl[4][0][4:] == 0.0) and np.all(gl[4][1][4:] == 0.0)
    net.close()


def test_adam_first_step():
    """Adam's first step moves every parameter with a non-negligible gradient by lr * sign(g)."""
    torch = _torch()
    from summationbyparts_b200.learned import CorrectionNet
    coarse, fine_r = _batch(seed=4)
    net = CorrectionNet(max_batch=2, seed=5)
    net.set_normalisation([1.0, 0.5, 0.0, 2.5], [0.05, 0.1, 0.1, 0.2], [1e-3, 1e-3, 1e-3, 2e-3])
    dc = torch.from_numpy(coarse).cuda().contiguous()
    df = torch.from_numpy(fine_r).cuda().contiguous()
    p0 = net.params()
    _, g = net.gradients(dc, df)
    lr = 1e-3
    net.train_step(dc, df, lr)
    p1 = net.params()
    big = np.abs(g) > 1e-5
    assert big.sum() > 1000
    np.testing.assert_allclose((p0 - p1)[big], lr * np.sign(g[big]), rtol=1e-3, atol=1e-7)
    assert np.all(p1[g == 0.0] == p0[g == 0.0])
    net.close()


def test_training_gains_over_coarse():
    """A short run at reduced size (48 training cases, 128 x 128 fine grid, 16 held-out cases):
    the trained network must cut the held-out coarse error against the restricted fine solve,
    and the coarse + network path must be faster than the fine solve."""
    from summationbyparts_b200 import learned
    rep = learned.run(pairs=48, heldout=16, epochs=80, fine=128, lr=3e-3, max_batch=16)
    h = rep["heldout"]
    assert rep["train"]["loss_last_epoch"] < 0.5 * rep["train"]["loss_first_epoch"]
    assert h["rel_l2_corrected_vs_fine_median"] < 0.7 * h["rel_l2_coarse_vs_fine_median"], h
    assert h["fallbacks"] < 8
    assert h["seconds_learned_path"] < h["seconds_fine_path"]


def test_fallback_replaces_flagged_cases_by_the_fine_solve():
    """The fallback path: with the threshold scaled far down every held-out case is flagged, so
    the answer of each is its restricted fine f64 solve (no error against the fine solve) and the
    fallback solves enter the time to solution."""
    from summationbyparts_b200 import learned
    rep = learned.run(pairs=16, heldout=8, epochs=5, fine=128, lr=3e-3, max_batch=16, fallback_factor=1e-9)
    h = rep["heldout"]
    assert h["fallbacks"] == 8
    assert h["rel_l2_final_vs_fine_max"] <= 1e-12
    assert h["seconds_learned_parts"]["fallback"] > 0.0
    assert h["rel_l2_corrected_vs_fine_max"] > 1e-8  # the network alone does not reach the fine solve
