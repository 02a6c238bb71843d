"""CPU-only checks of the C-ABI library and the host logic (no GPU needed).

* the library loads and exports every function include/sbp_b200.h declares;
* the coefficient tables built into the kernels equal the oracle's (bit for bit);
* argument validation answers with the documented status codes;
* the workload generators are deterministic and have the documented shapes.
"""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def capi():
    from summationbyparts_b200 import _capi
    return _capi


def declared_functions():
    names = []
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            src = open(os.path.join(ROOT, "include", f)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"\b(sbp_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(capi):
    names = declared_functions()
    assert len(names) >= 30
    for n in names:
        assert hasattr(capi.lib, n), n
        assert n in capi.SIGNATURES, f"{n} has no ctypes signature"


def test_version(capi):
    assert "sm_100a" in capi.version()


@pytest.mark.parametrize("op", range(6))
def test_tables_match_oracle(capi, orc, op):
    from summationbyparts_b200 import operators
    m, n, d, h2, upw = orc.op_shape(op)
    assert capi.lib.sbp_operator_is_h2(op) == int(h2)
    assert capi.lib.sbp_operator_is_upwind(op) == int(upw)
    h = (ctypes.c_double * 8)()
    assert capi.lib.sbp_operator_h(op, h, 8) == m
    np.testing.assert_array_equal(np.array(h[:m]), orc.op_table(op, orc.DIFF, 3))
    for kind in ([0, 1] if upw else [0]):
        for part in range(3):
            a = operators.table(op, kind, part)
            b = orc.op_table(op, kind, part)
            assert a.tobytes() == b.tobytes(), (op, kind, part)
    if not upw:
        with pytest.raises(ValueError):
            operators.table(op, 1, 0)


def test_bad_operator_and_unsupported_dissipation(capi):
    assert capi.lib.sbp_operator_is_h2(17) == -1
    buf = (ctypes.c_double * 8)()
    assert capi.lib.sbp_operator_h(-1, buf, 8) == -1
    # dissipation of a non-upwind operator: refused before touching the device
    st = capi.lib.sbp_dissxi(4, 0, ctypes.c_void_p(16), ctypes.c_void_p(32), 16, 16, 1, 256, None)
    assert st == 3  # SBP_ERR_UNSUPPORTED
    assert "dissipation" in capi.lib.sbp_last_error().decode()


def test_shape_validation_without_device(capi):
    # Upwind9 needs n >= max(2M, N) = 16 along the operator direction
    st = capi.lib.sbp_diffxi(2, 0, ctypes.c_void_p(16), ctypes.c_void_p(32), 20, 15, 1, 300, None)
    assert st == 2  # SBP_ERR_SHAPE
    st = capi.lib.sbp_diffeta(2, 0, ctypes.c_void_p(16), ctypes.c_void_p(32), 15, 20, 1, 300, None)
    assert st == 2
    st = capi.lib.sbp_diffxi(0, 7, ctypes.c_void_p(16), ctypes.c_void_p(32), 20, 20, 1, 400, None)
    assert st == 1  # bad dtype
    st = capi.lib.sbp_diffxi(0, 0, None, ctypes.c_void_p(32), 20, 20, 1, 400, None)
    assert st == 1  # null pointer
    st = capi.lib.sbp_diffxi(0, 0, ctypes.c_void_p(32), ctypes.c_void_p(32), 20, 20, 1, 400, None)
    assert st == 1  # aliasing


def test_system_create_validation(capi):
    from summationbyparts_b200 import workloads
    blocks = workloads.Config0(n=16).blocks()
    arr = (capi.BlockDesc * 1)()
    x, y = blocks[0].x, blocks[0].y
    arr[0].ny, arr[0].nx = x.shape
    arr[0].op_xi = arr[0].op_eta = 0
    arr[0].x = x.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    arr[0].y = y.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    h = ctypes.c_void_p()
    assert capi.lib.sbp_system_create(0, arr, 0, 1, 0, 1.4, ctypes.byref(h)) == 1
    assert capi.lib.sbp_system_create(0, arr, 1, 1, 9, 1.4, ctypes.byref(h)) == 1
    st = capi.lib.sbp_system_create(0, arr, 1, 1, 0, 1.4, ctypes.byref(h))
    import torch
    if not torch.cuda.is_available():
        assert st == 6  # SBP_ERR_NO_DEVICE
    elif st == 0:
        capi.lib.sbp_system_destroy(h)


def test_splitmix64_known_answers():
    from summationbyparts_b200 import workloads
    z = workloads.splitmix64(0, 3)
    assert [int(v) for v in z] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]
    u = workloads.uniform_pm1(0, 1000)
    assert u.min() >= -1.0 and u.max() < 1.0
    np.testing.assert_array_equal(workloads.splitmix64(5, 10)[4:], workloads.splitmix64(5, 6, start=4))


def test_ensemble_definition():
    from summationbyparts_b200 import workloads
    insts = workloads.ensemble_instances(512, seed=1)
    assert len(insts) == 512
    sides = np.array([i.side for i in insts])
    assert sides.min() >= 48 and sides.max() <= 257
    assert all(-2 <= i.x0 <= 2 and -2 <= i.y0 <= 2 and 0.5 <= i.eps <= 1.5 and 0.3 <= i.mach <= 0.7 for i in insts)
    ops = {i.op_id for i in insts}
    assert ops == {0, 2}
    pts = workloads.ensemble_points(insts)
    assert 12.0e6 < pts < 15.5e6
    again = workloads.ensemble_instances(512, seed=1)
    assert again == insts
    tail = workloads.ensemble_instances(12, seed=1, first=500)
    assert tail == insts[500:]


def test_multiblock_layout_is_conforming():
    from summationbyparts_b200 import workloads
    blocks = workloads.multiblock()
    assert len(blocks) == 6
    for b, spec in enumerate(blocks):
        for d, (kind, g) in enumerate(spec.bc):
            if kind != 1:
                continue
            other = blocks[g]
            if d in (0, 1):  # north/south share nx
                assert spec.x.shape[1] == other.x.shape[1]
                mine = spec.x[-1 if d == 0 else 0]
                theirs = other.x[0 if d == 0 else -1]
            else:
                assert spec.x.shape[0] == other.x.shape[0]
                mine = spec.x[:, -1 if d == 2 else 0]
                theirs = other.x[:, 0 if d == 2 else -1]
            np.testing.assert_allclose(mine, theirs, atol=1e-12)
            # and the neighbour points back
            back = {0: 1, 1: 0, 2: 3, 3: 2}[d]
            assert other.bc[back] == (1, b)
    pts = sum(s.x.size for s in blocks)
    assert 30000 < pts < 40000


def test_interpolate_rejects_bad_sizes():
    """sbp_interpolate checks the operator's size relation and its read range before any device
    work (so this runs without a GPU)."""
    import ctypes
    from summationbyparts_b200 import _capi
    p = ctypes.c_void_p(16)
    # fine must be 2 coarse - 1 (Interpolation9)
    assert _capi.lib.sbp_interpolate(2, 1, _capi.F64, p, p, 40, 21, 1, 40, 21, None) == 2
    # too short for the operator's boundary block (22 fine columns)
    assert _capi.lib.sbp_interpolate(2, 1, _capi.F64, p, p, 21, 11, 1, 21, 11, None) == 2
    # unknown operator
    assert _capi.lib.sbp_interpolate(7, 1, _capi.F64, p, p, 41, 21, 1, 41, 21, None) == 1


def test_advance_host_rejects_null_system():
    from summationbyparts_b200 import _capi
    p = ctypes.c_void_p(64)
    assert _capi.lib.sbp_system_advance_host(None, _capi.F64, p, p, 1, 4) == 1
    assert _capi.lib.sbp_system_advance_host_chunks(None) == -1
