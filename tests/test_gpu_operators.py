"""GPU parity of the standalone operators (diffxi/diffeta/dissxi/disseta) against the oracle.

Bar: bit-identical results in the same dtype (the oracle restates the reference's row path
without fma and its column path with the f64x8 / f32x16 fma split).  f32 results are also
reported against the f64 oracle with a tolerance of 2e-5 relative to the input scale.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

OPS = range(6)
SHAPES = [(16, 16), (37, 53), (64, 64), (20, 1031), (1030, 23), (129, 384), (97, 520)]


def gpu_apply(op_obj, which, a: np.ndarray) -> np.ndarray:
    t = torch.from_numpy(a).cuda()
    out = torch.empty_like(t)
    getattr(op_obj, which)(t, out)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def oracle_apply(orc, op, which, a):
    d, k = {"diffxi": (orc.XI, orc.DIFF), "diffeta": (orc.ETA, orc.DIFF), "dissxi": (orc.XI, orc.DISS),
            "disseta": (orc.ETA, orc.DISS)}[which]
    if a.ndim == 3:
        return np.stack([orc.op_apply(op, d, k, x) for x in a])
    return orc.op_apply(op, d, k, a)


def field(shape, seed, dtype):
    from summationbyparts_b200 import workloads
    n = int(np.prod(shape))
    return workloads.uniform_pm1(seed, n).reshape(shape).astype(dtype)


@pytest.mark.parametrize("op", OPS)
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_bitwise_against_oracle(orc, op, dtype):
    from summationbyparts_b200 import operators
    o = operators.BY_ID[op]()
    m, n_, d, h2, upw = orc.op_shape(op)
    which_all = ["diffxi", "diffeta"] + (["dissxi", "disseta"] if upw else [])
    for si, shape in enumerate(SHAPES):
        a = field(shape, 100 + si, dtype)
        for which in which_all:
            g = gpu_apply(o, which, a)
            r = oracle_apply(orc, op, which, a)
            assert g.dtype == dtype
            if g.tobytes() != r.tobytes():
                bad = np.argwhere(g != r)
                pytest.fail(f"{which} op={op} {shape} {dtype.__name__}: {len(bad)} mismatches, first {bad[:3]}, "
                            f"max abs diff {np.abs(g - r).max()}")


@pytest.mark.parametrize("op", [0, 2, 5])
def test_batched_planes(orc, op):
    from summationbyparts_b200 import operators
    o = operators.BY_ID[op]()
    a = field((3, 40, 72), 7, np.float64)
    for which in ["diffxi", "diffeta"]:
        assert gpu_apply(o, which, a).tobytes() == oracle_apply(orc, op, which, a).tobytes()


@pytest.mark.parametrize("op", [0, 2, 5])
def test_f32_error_against_f64_oracle(orc, op):
    from summationbyparts_b200 import operators
    o = operators.BY_ID[op]()
    a64 = field((256, 256), 11, np.float64)
    a32 = a64.astype(np.float32)
    for which in ["diffxi", "diffeta"]:
        g = gpu_apply(o, which, a32).astype(np.float64)
        r = oracle_apply(orc, op, which, a64)
        # values scale like idx * sum|c| ~ n; tolerance relative to that scale
        scale = np.abs(r).max()
        assert np.abs(g - r).max() <= 2e-5 * scale, (which, np.abs(g - r).max() / scale)


def test_full_size_operator_bitwise(orc):
    """One 4096 x 4096 field of the operator microbench, Upwind9 f64, both directions, every
    element against the oracle."""
    from summationbyparts_b200 import operators, workloads
    a = workloads.operator_fields(4096, 1, seed=0)[0]
    o = operators.Upwind9()
    for which in ["diffxi", "diffeta", "dissxi", "disseta"]:
        g = gpu_apply(o, which, a)
        r = oracle_apply(orc, 2, which, a)
        assert g.tobytes() == r.tobytes(), which


def test_linear_function_exact_full_size():
    """Size-independent property at the microbench size: D(a x + b) = a to rounding, for 4 fields."""
    from summationbyparts_b200 import operators
    n = 4096
    x = torch.linspace(0, 1, n, dtype=torch.float64, device="cuda")
    f = (3.0 * x[None, :] + 0.5 * x[:, None]).expand(n, n).contiguous()
    f = torch.stack([f, 2 * f, -f, f + 1.0])
    out = torch.empty_like(f)
    for op in [operators.Upwind4(), operators.Upwind9(), operators.SBP8()]:
        op.diffxi(f, out)
        for c, s in enumerate([1.0, 2.0, -1.0, 1.0]):
            assert torch.allclose(out[c], torch.full_like(out[c], 3.0 * s), atol=1e-9)
        op.diffeta(f, out)
        for c, s in enumerate([1.0, 2.0, -1.0, 1.0]):
            assert torch.allclose(out[c], torch.full_like(out[c], 0.5 * s), atol=1e-9)
    d = operators.Upwind9()
    d.dissxi(f, out)
    assert out.abs().max().item() < 1e-9  # dissipation annihilates linear functions


def test_shape_errors_raise():
    from summationbyparts_b200 import SbpError, operators
    a = torch.zeros((10, 10), dtype=torch.float64, device="cuda")
    b = torch.zeros_like(a)
    with pytest.raises(SbpError):
        operators.Upwind9().diffxi(a, b)
    with pytest.raises(SbpError):
        operators.SBP8().diffeta(a, b)
    with pytest.raises(ValueError):
        operators.Upwind4().diffxi(a, torch.zeros((10, 11), dtype=torch.float64, device="cuda"))
