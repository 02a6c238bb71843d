"""The CUDA path against the committed golden fixtures (tests/golden/sbp_golden.npz; inputs
and oracle outputs frozen by tests/golden/make_golden.py, the oracle held to them by
tests/test_golden_cpu.py).  No oracle call: the expected numbers are the stored ones.

Bars as in the live-oracle parity tests: operators and metrics bit for bit in their dtype; one
FP64 RK4 step within 1e-12 relative L2 (CUDA's hypot/exp/pow against the host libm are the
only difference)."""
import os
import sys

import numpy as np
import pytest
from _helpers import rel_l2

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden as mg  # noqa: E402

GOLDEN = os.path.join(HERE, "golden", "sbp_golden.npz")
PARITY = 1e-12


@pytest.fixture(scope="module")
def gold():
    with np.load(GOLDEN) as z:
        return {k: z[k] for k in z.files}


def gpu_apply(op_obj, which, a: np.ndarray) -> np.ndarray:
    t = torch.from_numpy(a).cuda()
    out = torch.empty_like(t)
    getattr(op_obj, which)(t, out)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("name", ["f64", "f32"])
def test_operators_match_golden(gold, name):
    from summationbyparts_b200 import operators
    a = gold[f"op_in_{name}"]
    checked = 0
    for op in range(6):
        o = operators.BY_ID[op]()
        for fn in mg.OP_FUNCS:
            key = f"op_{op}_{fn}_{name}"
            if key not in gold:  # dissipation of a non-upwind operator
                continue
            g = gpu_apply(o, fn, a)
            assert g.dtype == a.dtype
            assert g.tobytes() == gold[key].tobytes(), key
            checked += 1
    assert checked == 4 * 4 + 2 * 2


def test_metrics_match_golden(gold):
    from summationbyparts_b200 import _capi
    x, y = gold["met_x"], gold["met_y"]
    dx = torch.from_numpy(x).cuda()
    dy = torch.from_numpy(y).cuda()
    for opx, ope in mg.MET_PAIRS:
        out = torch.empty((5,) + x.shape, dtype=torch.float64, device="cuda")
        _capi.check(_capi.lib.sbp_metrics(opx, ope, dx.data_ptr(), dy.data_ptr(), x.shape[0], x.shape[1],
                                          out.data_ptr(), None))
        torch.cuda.synchronize()
        assert out.cpu().numpy().tobytes() == gold[f"met_{opx}_{ope}"].tobytes(), (opx, ope)


@pytest.mark.parametrize("op_name", mg.STEP_OPS)
def test_one_step_matches_golden(gold, op_name):
    from summationbyparts_b200 import workloads
    from summationbyparts_b200.system import BlockSystem
    blocks = mg.step_blocks(op_name, gold["step_x"], gold["step_y"])
    s = BlockSystem(blocks, 1, "f64", 1.4)
    s.set_vortex(workloads.STANDARD_VORTEX)
    s.set_state(0, gold["step_q0"])
    s.set_dt(mg.STEP_DT)
    s.advance(1)
    a, b = s.state(0), gold[f"step_{op_name}"]
    assert rel_l2(a, b) <= PARITY
    assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()
