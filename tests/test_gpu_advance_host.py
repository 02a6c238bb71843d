"""sbp_system_advance_host (host state in, RK4 steps, host state out, pipelined over chunks of
whole instances) gives the state of sbp_system_set_state_all + sbp_system_advance +
sbp_system_get_state_all bit for bit, and the same instance times: the chunks run the same
kernels on the same blocks, only their launches are grouped per chunk."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _ensemble(precision, n=12):
    from summationbyparts_b200 import workloads
    from summationbyparts_b200.system import BlockSystem
    insts = [i for i in workloads.ensemble_instances(60, seed=1) if i.side <= 130][:n]
    g = BlockSystem(workloads.ensemble_blocks(insts), len(insts), precision, 1.4)
    for k, i in enumerate(insts):
        g.set_vortex(i.vortex, k)
        g.set_dt(i.dt, k)
    g.init_vortex(0.0)
    return g, len(insts)


@pytest.mark.parametrize("precision", ["f64", "f32c"])
def test_matches_set_advance_get(precision):
    from summationbyparts_b200.system import F32, F64
    for dtype in (F64, F32):
        a, ninst = _ensemble(precision)
        b, _ = _ensemble(precision)
        n = a.state_count(dtype)
        q0 = torch.empty(n, dtype=torch.float64 if dtype == F64 else torch.float32, pin_memory=True)
        a.get_state_all(q0, dtype)
        ref = torch.empty_like(q0)
        a.set_state_all(q0, dtype)
        a.advance(5)
        a.get_state_all(ref, dtype)
        out = torch.empty_like(q0)
        chunks = b.advance_host(q0, out, 5, dtype, nchunks=4)
        assert chunks == 4
        assert out.numpy().tobytes() == ref.numpy().tobytes()
        assert [b.time(k) for k in range(ninst)] == [a.time(k) for k in range(ninst)]
        # in place, continuing from the new host state (for an f64 system an SBP_F32 host state is
        # a hi + lo pair, about 48 bits: the reference takes the same round trip)
        a.set_state_all(ref, dtype)
        a.advance(3)
        a.get_state_all(ref, dtype)
        b.advance_host(out, out, 3, dtype, nchunks=4)
        assert out.numpy().tobytes() == ref.numpy().tobytes()
        a.close()
        b.close()


def test_coupled_blocks_run_as_one_chunk():
    """The 6-block layout couples its blocks through Grid interfaces: one chunk, same result."""
    from summationbyparts_b200 import workloads
    from summationbyparts_b200.system import F64, BlockSystem
    out = []
    for mode in ("plain", "host"):
        g = BlockSystem(workloads.multiblock(), 1, "f64", 1.4)
        g.set_vortex(workloads.STANDARD_VORTEX)
        g.set_dt(0.002)
        g.init_vortex(0.0)
        q = np.empty(g.state_count(F64))
        g.get_state_all(q)
        r = np.empty_like(q)
        if mode == "plain":
            g.set_state_all(q)
            g.advance(4)
            g.get_state_all(r)
        else:
            assert g.advance_host(q, r, 4, nchunks=8) == 1
        out.append(r)
        g.close()
    assert out[0].tobytes() == out[1].tobytes()


def test_zero_steps_round_trips():
    from summationbyparts_b200.system import F64
    g, _ = _ensemble("f32c", 5)
    q = np.empty(g.state_count(F64))
    g.get_state_all(q)
    r = np.empty_like(q)
    g.advance_host(q, r, 0)
    back = np.empty_like(q)
    g.get_state_all(back)
    assert r.tobytes() == back.tobytes()
    g.close()
