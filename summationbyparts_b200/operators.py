"""SBP operators on the GPU: the sbp::operators traits of the reference.

Mirrors sbp/src/operators.rs:
  * SbpOperator2d   -- diffxi, diffeta, hxi/heta, is_h2xi/is_h2eta, op_xi/op_eta, upwind()
  * UpwindOperator2d -- dissxi, disseta
  * Upwind4, Upwind4h2, Upwind9, Upwind9h2, SBP4, SBP8 (sbp/src/operators.rs:152-165)
  * Pair(eta, xi)   -- the (eta_op, xi_op) tuple composition (sbp/src/operators.rs:115-150)

`prev` and `fut` are CUDA tensors (torch) of shape (ny, nx) or (batch, ny, nx), float64 or
float32, C-contiguous, on the device the library runs on.  Every call launches a kernel of
libsbp_b200 on the current torch stream; results are bit-identical to the reference's CPU
path in the same dtype.  Shapes are checked like the reference's assert_eq! and reported
as SbpError.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi

UPWIND4, UPWIND4H2, UPWIND9, UPWIND9H2, SBP4_ID, SBP8_ID = range(6)


def _dtype_code(t) -> int:
    import torch

    if t.dtype == torch.float64:
        return _capi.F64
    if t.dtype == torch.float32:
        return _capi.F32
    raise TypeError(f"unsupported dtype {t.dtype}")


def _launch(fn, op_id: int, prev, fut) -> None:
    import torch

    if prev.shape != fut.shape:
        raise ValueError(f"prev {tuple(prev.shape)} and fut {tuple(fut.shape)} must have the same shape")
    if prev.dtype != fut.dtype:
        raise ValueError("prev and fut must have the same dtype")
    if not (prev.is_cuda and fut.is_cuda):
        raise ValueError("prev and fut must be CUDA tensors")
    if not (prev.is_contiguous() and fut.is_contiguous()):
        raise ValueError("prev and fut must be contiguous")
    if prev.dim() == 2:
        nb, (ny, nx) = 1, prev.shape
    elif prev.dim() == 3:
        nb, ny, nx = prev.shape
    else:
        raise ValueError("expected (ny, nx) or (batch, ny, nx)")
    stream = torch.cuda.current_stream(prev.device).cuda_stream
    _capi.check(fn(op_id, _dtype_code(prev), prev.data_ptr(), fut.data_ptr(), ny, nx, nb, ny * nx,
                   ctypes.c_void_p(stream)))


class SbpOperator1dInfo:
    """The 1-D facts the 2-D traits expose (SbpOperator1d::h / is_h2, sbp/src/operators.rs:11-32)."""

    def __init__(self, op_id: int):
        self.op_id = op_id

    def h(self) -> np.ndarray:
        buf = (ctypes.c_double * 8)()
        m = _capi.lib.sbp_operator_h(self.op_id, buf, 8)
        return np.array(buf[:m])

    def is_h2(self) -> bool:
        return _capi.lib.sbp_operator_is_h2(self.op_id) == 1


class SbpOperator2d:
    """Differentiation along xi (axis 1, contiguous) and eta (axis 0)."""

    op_id: int = -1

    def op_xi(self) -> SbpOperator1dInfo:
        return SbpOperator1dInfo(self.op_id)

    def op_eta(self) -> SbpOperator1dInfo:
        return self.op_xi()

    def diffxi(self, prev, fut) -> None:
        _launch(_capi.lib.sbp_diffxi, self.op_xi().op_id, prev, fut)

    def diffeta(self, prev, fut) -> None:
        _launch(_capi.lib.sbp_diffeta, self.op_eta().op_id, prev, fut)

    def hxi(self) -> np.ndarray:
        return self.op_xi().h()

    def heta(self) -> np.ndarray:
        return self.op_eta().h()

    def is_h2xi(self) -> bool:
        return self.op_xi().is_h2()

    def is_h2eta(self) -> bool:
        return self.op_eta().is_h2()

    def upwind(self):
        return None

    # ids of the (xi, eta) operators, as the system descriptors want them
    @property
    def ids(self) -> tuple[int, int]:
        return self.op_xi().op_id, self.op_eta().op_id


class UpwindOperator2d:
    """Upwind dissipation along xi and eta (sbp/src/operators.rs:90-106)."""

    def dissxi(self, prev, fut) -> None:
        _launch(_capi.lib.sbp_dissxi, self.op_xi().op_id, prev, fut)

    def disseta(self, prev, fut) -> None:
        _launch(_capi.lib.sbp_disseta, self.op_eta().op_id, prev, fut)


class _Single(SbpOperator2d):
    def __repr__(self):
        return type(self).__name__

    def __eq__(self, other):
        return type(self) is type(other)

    def __hash__(self):
        return hash(type(self))


class _SingleUpwind(_Single, UpwindOperator2d):
    def upwind(self):
        return self


class Upwind4(_SingleUpwind):
    op_id = UPWIND4


class Upwind4h2(_SingleUpwind):
    op_id = UPWIND4H2


class Upwind9(_SingleUpwind):
    op_id = UPWIND9


class Upwind9h2(_SingleUpwind):
    op_id = UPWIND9H2


class SBP4(_Single):
    op_id = SBP4_ID


class SBP8(_Single):
    op_id = SBP8_ID


class Pair(SbpOperator2d):
    """(eta_op, xi_op): diffxi uses xi_op, diffeta uses eta_op (sbp/src/operators.rs:115-135)."""

    def __init__(self, eta_op: SbpOperator2d, xi_op: SbpOperator2d):
        self.eta_op = eta_op
        self.xi_op = xi_op

    def op_xi(self) -> SbpOperator1dInfo:
        return self.xi_op.op_xi()

    def op_eta(self) -> SbpOperator1dInfo:
        return self.eta_op.op_eta()

    def upwind(self):
        if self.eta_op.upwind() is not None and self.xi_op.upwind() is not None:
            return _PairUpwind(self)
        return None

    def __repr__(self):
        return f"Pair(eta={self.eta_op!r}, xi={self.xi_op!r})"


class _PairUpwind(UpwindOperator2d):
    def __init__(self, pair: Pair):
        self.pair = pair

    def op_xi(self):
        return self.pair.op_xi()

    def op_eta(self):
        return self.pair.op_eta()


BY_NAME = {"upwind4": Upwind4, "upwind4h2": Upwind4h2, "upwind9": Upwind9, "upwind9h2": Upwind9h2,
           "sbp4": SBP4, "sbp8": SBP8}
BY_ID = {UPWIND4: Upwind4, UPWIND4H2: Upwind4h2, UPWIND9: Upwind9, UPWIND9H2: Upwind9h2, SBP4_ID: SBP4,
         SBP8_ID: SBP8}


def table(op_id: int, kind: int, part: int) -> np.ndarray:
    """The coefficients built into the kernels (kind 0 diff / 1 diss; part 0 start, 1 diag, 2 end)."""
    buf = (ctypes.c_double * (8 * 13))()
    n = _capi.lib.sbp_operator_table(op_id, kind, part, buf, 8 * 13)
    if n < 0:
        raise ValueError("no such table")
    return np.array(buf[:n])
