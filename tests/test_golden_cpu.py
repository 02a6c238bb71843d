"""The oracle against the committed golden fixtures (tests/golden/sbp_golden.npz, written by
tests/golden/make_golden.py): fed the stored inputs, the oracle must reproduce every stored
output bit for bit, so a change to the oracle cannot silently move the numbers the GPU parity
tests are held to."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden as mg  # noqa: E402

GOLDEN = os.path.join(HERE, "golden", "sbp_golden.npz")


@pytest.fixture(scope="module")
def gold():
    with np.load(GOLDEN) as z:
        return {k: z[k] for k in z.files}


def test_fixture_inventory(gold, orc):
    expected = {"met_x", "met_y", "step_x", "step_y", "step_q0"}
    for name, _, _ in mg.DTYPES:
        expected.add(f"op_in_{name}")
        for op in range(6):
            expected |= {f"op_{op}_{fn}_{name}" for fn in mg.funcs_of(orc, op)}
    expected |= {f"met_{a}_{b}" for a, b in mg.MET_PAIRS}
    expected |= {f"step_{o}" for o in mg.STEP_OPS}
    assert set(gold) == expected


def test_seeded_inputs_regenerate(gold):
    from summationbyparts_b200 import workloads
    n = mg.OP_SHAPE[0] * mg.OP_SHAPE[1]
    for name, dt, seed in mg.DTYPES:
        a = workloads.uniform_pm1(seed, n).reshape(mg.OP_SHAPE).astype(dt)
        assert a.tobytes() == gold[f"op_in_{name}"].tobytes()
    x, y = workloads.warped(-5.0, 5.0, 29, -4.0, 5.0, 21)
    np.testing.assert_allclose(x, gold["met_x"], rtol=1e-15, atol=1e-15)
    np.testing.assert_allclose(y, gold["met_y"], rtol=1e-15, atol=1e-15)


@pytest.mark.parametrize("name", ["f64", "f32"])
def test_oracle_operators_reproduce_fixtures(gold, orc, name):
    a = gold[f"op_in_{name}"]
    for op in range(6):
        for fn in mg.funcs_of(orc, op):
            r = mg.oracle_op(orc, op, fn, a)
            assert r.dtype == a.dtype
            assert r.tobytes() == gold[f"op_{op}_{fn}_{name}"].tobytes(), (op, fn, name)


def test_oracle_metrics_reproduce_fixtures(gold, orc):
    for opx, ope in mg.MET_PAIRS:
        r = orc.metrics(opx, ope, gold["met_x"], gold["met_y"])
        assert r.tobytes() == gold[f"met_{opx}_{ope}"].tobytes(), (opx, ope)


@pytest.mark.parametrize("op_name", mg.STEP_OPS)
def test_oracle_step_reproduces_fixture(gold, orc, op_name):
    r = mg.oracle_step(orc, op_name, gold["step_x"], gold["step_y"], gold["step_q0"])
    assert r.tobytes() == gold[f"step_{op_name}"].tobytes()


def test_fixtures_are_not_trivial(gold):
    """The step changes the state, and every operator output is finite and nonzero."""
    for op_name in mg.STEP_OPS:
        d = gold[f"step_{op_name}"] - gold["step_q0"]
        assert np.isfinite(d).all() and np.abs(d).max() > 1e-6
    for k, v in gold.items():
        if k.startswith("op_") and not k.startswith("op_in"):
            assert np.isfinite(v).all() and np.abs(v).max() > 0, k
