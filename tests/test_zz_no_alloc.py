"""sbp_metrics_noalloc: grid metrics with no device allocation.

Callers that cannot allocate device memory where they need metrics (all device memory owned
by another runtime's pool or arena, or a time-critical loop that forbids allocator calls) use
this entry point; its working memory is a fixed array inside the library.  The test calls it
through the C ABI twice in a row on different grids and operators -- the second call reuses
the array the first one left behind -- and checks each result bit for bit against the
allocating entry point sbp_metrics (the metric tests' bar), then checks that a grid beyond
the array's 512 x 512 limit is refused with a clear error.  The file is named to run last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _metrics(fn, opx, ope, x, y):
    from summationbyparts_b200 import _capi
    dx = torch.from_numpy(x).cuda()
    dy = torch.from_numpy(y).cuda()
    out = torch.full((5,) + x.shape, float("nan"), dtype=torch.float64, device="cuda")
    _capi.check(fn(opx, ope, dx.data_ptr(), dy.data_ptr(), x.shape[0], x.shape[1], out.data_ptr(), None))
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_metrics_match_allocating_entry_point_twice():
    from summationbyparts_b200 import _capi, workloads
    cases = [(2, 2, workloads.warped(-5.0, 5.0, 211, -4.0, 5.0, 173)),   # Upwind9, 36503 points
             (0, 1, workloads.warped(-2.0, 3.0, 64, -5.0, 5.0, 300))]    # Upwind4 / Upwind4h2
    for opx, ope, (x, y) in cases:
        ref = _metrics(_capi.lib.sbp_metrics, opx, ope, x, y)
        got = _metrics(_capi.lib.sbp_metrics_noalloc, opx, ope, x, y)
        assert np.isfinite(got).all()
        assert got.tobytes() == ref.tobytes()


def test_noalloc_refuses_grids_beyond_its_scratch():
    from summationbyparts_b200 import _capi
    p = ctypes.c_void_p(256)  # never dereferenced: the size check comes first
    st = _capi.lib.sbp_metrics_noalloc(0, 0, p, p, 513, 513, p, None)
    assert st == 2  # SBP_ERR_SHAPE
    assert "262144" in _capi.lib.sbp_last_error().decode()
    # sides whose product would overflow 64 bits are refused too, not wrapped to a small size
    for ny, nx in ((1 << 33, 1 << 31), (1 << 31, 1 << 33), (2, 1 << 62)):
        assert _capi.lib.sbp_metrics_noalloc(0, 0, p, p, ny, nx, p, None) == 2, (ny, nx)
