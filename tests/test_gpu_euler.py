"""GPU parity of the fused Euler RK4 path against the oracle.

Bar (FP64 plain form): relative L2 difference to the oracle <= 1e-12 after the full run.
The arithmetic is the reference's operation by operation; the only sources of difference
are CUDA's hypot/exp/pow versus the host libm (SAT normalisation and vortex boundary data)
and the summation order of the norms.  Metrics and max_dt are compared bit for bit.
The compensated-f32 form is compared with the f64 oracle at 1e-5 relative L2.
"""
import numpy as np
import pytest
from _helpers import oracle_system, physical_state, rel_l2

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

PARITY = 1e-12


def gpu_system(blocks, vortex, precision="f64", ninst=1):
    from summationbyparts_b200.system import BlockSystem
    s = BlockSystem(blocks, ninst, precision, 1.4)
    s.set_vortex(vortex)
    return s


@pytest.mark.parametrize("opx,ope", [(0, 0), (2, 2), (5, 5), (2, 3), (1, 1), (4, 4)])
def test_metrics_bitwise(orc, opx, ope):
    from summationbyparts_b200 import workloads
    x, y = workloads.warped(-5.0, 5.0, 53, -4.0, 5.0, 41)
    dx = torch.from_numpy(x).cuda()
    dy = torch.from_numpy(y).cuda()
    out = torch.empty((5,) + x.shape, dtype=torch.float64, device="cuda")
    import ctypes
    from summationbyparts_b200 import _capi
    _capi.check(_capi.lib.sbp_metrics(opx, ope, dx.data_ptr(), dy.data_ptr(), x.shape[0], x.shape[1],
                                      out.data_ptr(), None))
    torch.cuda.synchronize()
    ref = orc.metrics(opx, ope, x, y)
    assert out.cpu().numpy().tobytes() == ref.tobytes()


def test_metrics_reject_folded_grid():
    import ctypes
    from summationbyparts_b200 import SbpError, _capi, workloads
    x, y = workloads.cartesian(-5.0, 5.0, 20, -5.0, 5.0, 20)
    x = x[:, ::-1].copy()  # mirrored -> detJ < 0
    dx = torch.from_numpy(x).cuda()
    dy = torch.from_numpy(y).cuda()
    out = torch.empty((5, 20, 20), dtype=torch.float64, device="cuda")
    with pytest.raises(SbpError) as e:
        _capi.check(_capi.lib.sbp_metrics(0, 0, dx.data_ptr(), dy.data_ptr(), 20, 20, out.data_ptr(), None))
    assert e.value.status == 5


@pytest.mark.parametrize("op_name", ["Upwind4", "Upwind9", "SBP4", "SBP8", "Upwind4h2", "Upwind9h2"])
def test_one_step_periodic_each_operator(orc, op_name):
    """One RK4 step of euler::System (periodic `This` boundaries) from a perturbed state."""
    from summationbyparts_b200 import operators, workloads
    from summationbyparts_b200.system import BlockSpec
    op = getattr(operators, op_name)()
    x, y = workloads.warped(-5.0, 5.0, 45, -5.0, 5.0, 38)
    blocks = [BlockSpec(x, y, op, [(0, 0)] * 4, 0)]
    q0 = physical_state(x, y)
    g = gpu_system(blocks, workloads.STANDARD_VORTEX)
    g.set_state(0, q0)
    g.set_dt(0.01)
    g.advance(1)
    o = oracle_system(orc, blocks, workloads.STANDARD_VORTEX)
    o.set_state(0, q0)
    o.advance(1, 0.01)
    a, b = g.state(0), o.state(0)
    assert rel_l2(a, b) <= PARITY
    assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()


def test_config0_vortex_100_steps(orc):
    """Configuration 0: 64x64 Upwind4, vortex SATs on every side, dt = 0.2/63, 100 steps."""
    from summationbyparts_b200 import workloads
    cfg = workloads.Config0()
    blocks = cfg.blocks()
    g = gpu_system(blocks, workloads.STANDARD_VORTEX)
    g.init_vortex(0.0)
    g.set_dt(cfg.dt)
    g.advance(cfg.steps)
    o = oracle_system(orc, blocks, workloads.STANDARD_VORTEX)
    o.init_vortex(0.0)
    # start both from identical bits: the GPU vortex uses CUDA exp/pow
    g.set_state(0, o.state(0))
    g.set_time(0.0)
    g.advance(cfg.steps)
    o.advance(cfg.steps, cfg.dt)
    assert rel_l2(g.state(0), o.state(0)) <= PARITY
    assert abs(g.time(0) - o.time) == 0.0
    eg, eo = g.errors()[0], o.error()
    assert abs(eg - eo) <= 1e-10 * eo
    assert 1e-4 < eo < 1e-1  # a discretisation error, not a blow-up


def test_multiblock_interfaces(orc):
    """Configuration 2 layout (6 curvilinear Upwind9 blocks, Grid interfaces, vortex outer edges),
    the configured 500 RK4 steps: f64 within 1e-12 of the oracle, the compensated form within
    1e-6 of it (the six listed block sizes admit no layout under the reference's couplings,
    tests/test_config2_layout_cpu.py; this is the conforming 2 x 3 layout)."""
    from summationbyparts_b200 import workloads
    blocks = workloads.multiblock()
    dt = workloads.multiblock_dt(blocks)
    o = oracle_system(orc, blocks, workloads.STANDARD_VORTEX)
    o.init_vortex(0.0)
    q0 = [o.state(b) for b in range(len(blocks))]
    o.advance(500, dt)
    for prec, bar in (("f64", PARITY), ("f32c", 1e-6)):
        g = gpu_system(blocks, workloads.STANDARD_VORTEX, prec)
        for b in range(len(blocks)):
            g.set_state(b, q0[b])
        g.set_dt(dt)
        g.advance(500)
        for b in range(len(blocks)):
            assert rel_l2(g.state(b), o.state(b)) <= bar, (prec, b)
        assert abs(g.errors()[0] - o.error()) <= (1e-10 if prec == "f64" else 1e-3) * o.error()
        g.close()


def test_max_dt_bitwise(orc):
    from summationbyparts_b200 import workloads
    blocks = workloads.multiblock()
    o = oracle_system(orc, blocks, workloads.STANDARD_VORTEX)
    o.init_vortex(0.0)
    g = gpu_system(blocks, workloads.STANDARD_VORTEX)
    for b in range(len(blocks)):
        g.set_state(b, o.state(b))
    assert g.max_dt(0) == o.max_dt()


def test_force_trad_matches_rhs_trad(orc):
    """euler::System::advance uses RHS_trad even for upwind operators."""
    from summationbyparts_b200 import euler, operators, workloads
    x, y = workloads.cartesian(-5.0, 5.0, 40, -5.0, 5.0, 40)
    s = euler.System(x, y, operators.Upwind4())
    q0 = physical_state(x, y)
    s.set_field(q0)
    s.advance(0.005)
    from summationbyparts_b200.system import BlockSpec
    o = oracle_system(orc, [BlockSpec(x, y, operators.Upwind4(), [(0, 0)] * 4)], workloads.STANDARD_VORTEX)
    o.set_state(0, q0)
    o.advance(1, 0.005, force_trad=True)
    assert rel_l2(s.field(), o.state(0)) <= PARITY


def test_schedule_independence():
    """Different tile shapes give bit-identical results."""
    from summationbyparts_b200 import workloads
    blocks = workloads.multiblock()
    res = []
    for ty, tx in [(32, 32), (16, 32)]:
        g = gpu_system(blocks, workloads.STANDARD_VORTEX)
        g.init_vortex(0.0)
        g.set_dt(0.002)
        g.set_tiles(ty, tx)
        g.advance(3)
        res.append(np.concatenate([g.state(b).ravel() for b in range(len(blocks))]))
    assert res[0].tobytes() == res[1].tobytes()


def test_ensemble_ragged(orc):
    """A small ensemble (seed 1) with ragged step counts against per-instance oracle runs."""
    from summationbyparts_b200 import workloads
    from summationbyparts_b200.system import BlockSystem
    insts = [i for i in workloads.ensemble_instances(40, seed=1) if i.side <= 110][:4]
    assert len(insts) >= 3
    blocks = workloads.ensemble_blocks(insts)
    g = BlockSystem(blocks, len(insts), "f64", 1.4)
    steps = [5 + 3 * k for k in range(len(insts))]
    for k, inst in enumerate(insts):
        g.set_vortex(inst.vortex, k)
        g.set_dt(inst.dt, k)
    g.init_vortex(0.0)
    refs = []
    for k, inst in enumerate(insts):
        blocks[k].instance = 0
        o = oracle_system(orc, [blocks[k]], inst.vortex)
        o.init_vortex(0.0)
        g.set_state(k, o.state(0))
        o.advance(steps[k], inst.dt)
        refs.append(o)
    g.advance_instances(steps)
    for k, o in enumerate(refs):
        assert rel_l2(g.state(k), o.state(0)) <= PARITY, k
        assert g.time(k) == o.time
    errs = g.errors()
    for k, o in enumerate(refs):
        assert abs(errs[k] - o.error()) <= 1e-10 * o.error()


def test_compensated_f32_against_f64_oracle(orc):
    from summationbyparts_b200 import workloads
    cfg = workloads.Config0()
    blocks = cfg.blocks()
    o = oracle_system(orc, blocks, workloads.STANDARD_VORTEX)
    o.init_vortex(0.0)
    g = gpu_system(blocks, workloads.STANDARD_VORTEX, precision="f32c")
    g.set_state(0, o.state(0))
    g.set_dt(cfg.dt)
    g.advance(cfg.steps)
    o.advance(cfg.steps, cfg.dt)
    d = rel_l2(g.state(0), o.state(0))
    assert d <= 1e-5, d
    eg, eo = g.errors()[0], o.error()
    assert abs(eg - eo) <= 1e-3 * eo, (eg, eo)


def test_compensated_state_roundtrip():
    """set_state/get_state of the compensated form keep ~48 bits (hi + lo)."""
    from summationbyparts_b200 import workloads
    blocks = workloads.Config0(n=24).blocks()
    g = gpu_system(blocks, workloads.STANDARD_VORTEX, precision="f32c")
    q = physical_state(blocks[0].x, blocks[0].y)
    g.set_state(0, q)
    back = g.state(0)
    assert np.abs(back - q).max() <= 1e-13 * np.abs(q).max()


def test_nonphysical_state_is_reported():
    from summationbyparts_b200 import SbpError, workloads
    blocks = workloads.Config0(n=24).blocks()
    g = gpu_system(blocks, workloads.STANDARD_VORTEX)
    q = physical_state(blocks[0].x, blocks[0].y)
    q[0, 5, 7] = -1.0  # negative density
    g.set_state(0, q)
    g.set_dt(0.001)
    with pytest.raises(SbpError) as e:
        g.advance(1)
    assert e.value.status == 5


def test_interface_length_mismatch_rejected():
    from summationbyparts_b200 import SbpError, operators, workloads
    from summationbyparts_b200.system import BlockSpec, BlockSystem
    x1, y1 = workloads.cartesian(-5, 0, 30, -5, 5, 30)
    x2, y2 = workloads.cartesian(0, 5, 30, -5, 5, 31)
    b = [BlockSpec(x1, y1, operators.Upwind4(), [(2, 0), (2, 0), (1, 1), (2, 0)]),
         BlockSpec(x2, y2, operators.Upwind4(), [(2, 0), (2, 0), (2, 0), (1, 0)])]
    with pytest.raises(SbpError) as e:
        BlockSystem(b, 1)
    assert e.value.status == 2


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32c"])
def test_stage_launches_match_advance(precision):
    """Launching every group's stage and edge kernels stage by stage (sbp_system_launch_stage)
    gives the same state, bit for bit, as one graph-captured sbp_system_advance step; the groups
    partition the blocks by operator pair."""
    from summationbyparts_b200 import workloads
    from summationbyparts_b200.system import BlockSystem
    insts = [i for i in workloads.ensemble_instances(40, seed=1) if i.side <= 120][:4]
    assert {i.op_id for i in insts} == {workloads.UPWIND4, workloads.UPWIND9}
    out = []
    for mode in ("advance", "launch"):
        g = BlockSystem(workloads.ensemble_blocks(insts), len(insts), precision, 1.4)
        for k, inst in enumerate(insts):
            g.set_vortex(inst.vortex, k)
            g.set_dt(inst.dt, k)
        g.init_vortex(0.0)
        groups = g.groups()
        assert sorted((ox, oy) for ox, oy, _ in groups) == [(workloads.UPWIND4,) * 2, (workloads.UPWIND9,) * 2]
        assert sum(p for _, _, p in groups) == sum(i.side ** 2 for i in insts)
        if mode == "advance":
            g.advance(1)
        else:
            for st in range(4):
                for gi in range(len(groups)):
                    g.launch_stage(gi, st, with_edges=True)
        out.append(np.concatenate([g.state(b).ravel() for b in range(len(insts))]))
        g.close()
    assert out[0].tobytes() == out[1].tobytes()


def test_ragged_steps_on_a_caller_stream():
    """Ragged step counts on a caller's stream (sbp_system_set_stream): every instance ends at
    time steps * dt, summed step by step as the device does, and the states equal those of the
    same run on the system's own stream.  (The schedule changes between the ragged segments;
    steps still in flight must not see the next segment's instance mask.)"""
    from summationbyparts_b200 import workloads
    from summationbyparts_b200.system import BlockSystem
    insts = [i for i in workloads.ensemble_instances(40, seed=1) if i.side <= 90][:6]
    steps = [3, 40, 7, 25, 1, 60]
    out = []
    for use_stream in (False, True):
        g = BlockSystem(workloads.ensemble_blocks(insts), len(insts), "f32c", 1.4)
        st = torch.cuda.Stream()
        if use_stream:
            g.set_stream(st.cuda_stream)
        for k, inst in enumerate(insts):
            g.set_vortex(inst.vortex, k)
            g.set_dt(inst.dt, k)
        g.init_vortex(0.0)
        g.advance_instances(steps)
        for k, inst in enumerate(insts):
            t = 0.0
            for _ in range(steps[k]):
                t += inst.dt
            assert g.time(k) == t, (k, g.time(k), t)
        out.append(np.concatenate([g.state(b).ravel() for b in range(len(insts))]))
        g.close()
    assert out[0].tobytes() == out[1].tobytes()
