"""Pin the oracle against the reference's own known-answer tests.

The reference ships no golden vectors; its tests pin the operators and the
solver by analytic properties.  Each test here restates one of them, with the
reference's sizes and tolerances, and runs it on the oracle:

* polynomial exactness: sbp/src/operators/upwind4.rs:299-453 (upwind4_test,
  upwind4_test2), upwind9.rs:122-184, traditional4.rs:437-468,
  traditional8.rs:250-312, helper operators.rs:174-212;
* h2 operators: upwind4h2.rs:105-128, upwind9h2.rs:243-266;
* h2linspace: sbp/src/utils.rs:142-155;
* H-norm of ones: euler/src/lib.rs:434-448 (h2_diff);
* convergence of the vortex: euler/tests/convergence.rs:9-90.
"""
import math

import numpy as np
import pytest


def grid_eval(n, f):
    """operators.rs:174-187: f on the unit grid, x along axis 1."""
    ny, nx = n
    dx = 1.0 / (nx - 1)
    dy = 1.0 / (ny - 1)
    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    return f(dx * i, dy * j)


def check_operator_on(orc, op, n, f, dfdx, dfdy, eps):
    """operators.rs:189-212"""
    x = grid_eval(n, f).astype(np.float64)
    np.testing.assert_allclose(orc.diffxi(op, x), grid_eval(n, dfdx) + 0 * x, rtol=0, atol=eps)
    np.testing.assert_allclose(orc.diffeta(op, x), grid_eval(n, dfdy) + 0 * x, rtol=0, atol=eps)


P3 = (lambda x, y: x**3 + 2.0 * x**2 * y + 3.0 * x * y**2 + 4.0 * y**3,
      lambda x, y: 3.0 * x**2 + 4.0 * x * y + 3.0 * y**2,
      lambda x, y: 2.0 * x**2 + 6.0 * x * y + 12.0 * y**2)
P4 = (lambda x, y: x**4 + x**3 * y + x**2 * y**2 + x * y**3 + y**4,
      lambda x, y: 4.0 * x**3 + 3.0 * x**2 * y + 2.0 * x * y**2 + y**3,
      lambda x, y: x**3 + 2.0 * x**2 * y + 3.0 * x * y**2 + 4.0 * y**3)


def test_upwind4_1d(orc):
    """upwind4.rs:299-385 (diff on 1-D rows and on (nx, 8) columns)."""
    nx = 20
    dx = 1.0 / (nx - 1)
    xs = np.arange(nx) * dx
    for src, tgt, eps1d in ((xs, np.ones(nx), 1e-4), (xs * xs, 2.0 * xs, 1e-4), (xs**3, 3.0 * xs * xs, 1e-2)):
        res = orc.diffxi(orc.UPWIND4, src[None, :].copy())[0]
        np.testing.assert_allclose(res, tgt, atol=eps1d, rtol=0)
        col = np.repeat(src[:, None], 8, axis=1)
        res = orc.diffeta(orc.UPWIND4, col)
        np.testing.assert_allclose(res, np.repeat(tgt[:, None], 8, axis=1), atol=1e-2, rtol=0)


def test_upwind4_2d(orc):
    """upwind4.rs:414-453"""
    n = (16, 32)
    check_operator_on(orc, orc.UPWIND4, n, lambda x, y: x + 2.0 * y, lambda x, y: 1.0, lambda x, y: 2.0, 1e-4)
    check_operator_on(orc, orc.UPWIND4, n, lambda x, y: x * x + 2.0 * x * y + 3.0 * y * y,
                      lambda x, y: 2.0 * x + 2.0 * y, lambda x, y: 2.0 * x + 6.0 * y, 1e-3)
    check_operator_on(orc, orc.UPWIND4, n, *P3, 1e-1)
    check_operator_on(orc, orc.UPWIND4, (32, 32), *P3, 1e-1)


@pytest.mark.parametrize("op_name", ["UPWIND9", "SBP8"])
def test_order8_2d(orc, op_name):
    """upwind9.rs:122-184, traditional8.rs:250-312"""
    op = getattr(orc, op_name)
    n = (16, 32)
    check_operator_on(orc, op, n, lambda x, y: x + 2.0 * y, lambda x, y: 1.0, lambda x, y: 2.0, 1e-4)
    check_operator_on(orc, op, n, lambda x, y: x * x + 0.5 * y * y, lambda x, y: 2.0 * x, lambda x, y: y, 1e-4)
    check_operator_on(orc, op, n, lambda x, y: x * y, lambda x, y: y, lambda x, y: x, 1e-4)
    check_operator_on(orc, op, n, lambda x, y: x**3 + y**3 / 6.0, lambda x, y: 3.0 * x * x,
                      lambda x, y: y * y / 2.0, 1e-4)
    check_operator_on(orc, op, n, lambda x, y: x * x * y + x * y * y / 2.0, lambda x, y: 2.0 * x * y + y * y / 2.0,
                      lambda x, y: x * x + x * y, 1e-4)
    check_operator_on(orc, op, n, *P3, 1e-4)
    check_operator_on(orc, op, n, *P4, 1e-4)


def test_sbp4_2d(orc):
    """traditional4.rs:437-468"""
    n = (13, 20)
    check_operator_on(orc, orc.SBP4, n, lambda x, y: x + 2.0 * y, lambda x, y: 1.0, lambda x, y: 2.0, 1e-4)
    check_operator_on(orc, orc.SBP4, n, lambda x, y: x * x + 2.0 * x * y + 3.0 * y * y,
                      lambda x, y: 2.0 * x + 2.0 * y, lambda x, y: 2.0 * x + 6.0 * y, 1e-3)
    check_operator_on(orc, orc.SBP4, n, *P3, 1e-1)


def h2linspace(start, end, n):
    """sbp/src/utils.rs:130-140"""
    h = (end - start) / (n - 2)
    x = np.array([start + h * (i - 0.5) for i in range(n)])
    x[0], x[-1] = start, end
    return x


def test_h2linspace():
    """sbp/src/utils.rs:142-155"""
    x = h2linspace(-1.0, 1.0, 50)
    assert abs(x[0] + 1.0) < 1e-6 and abs(x[49] - 1.0) < 1e-6
    hend = x[1] - x[0]
    h = x[2] - x[1]
    assert abs((x[49] - x[48]) - hend) < 1e-6
    assert abs(2.0 * hend - h) < 1e-6
    for i in range(1, 48):
        assert abs((x[i + 1] - x[i]) - h) < 1e-6


@pytest.mark.parametrize("op_name,nx", [("UPWIND4H2", 20), ("UPWIND9H2", 30)])
def test_h2_operators(orc, op_name, nx):
    """upwind4h2.rs:105-128, upwind9h2.rs:243-266"""
    op = getattr(orc, op_name)
    x = h2linspace(0.0, 1.0, nx)
    for src, tgt, eps in ((x, np.ones(nx), 1e-4), (x * x / 2.0, x, 1e-4), (x**3 / 3.0, x * x, 1e-2)):
        res = orc.diffxi(op, src[None, :].copy())[0]
        np.testing.assert_allclose(res, tgt, atol=eps, rtol=0)


@pytest.mark.parametrize("op_name", ["UPWIND4", "UPWIND9", "SBP4", "SBP8"])
def test_h_norm_of_ones(orc, op_name):
    """euler/src/lib.rs:434-448: |1|_H^2 over the 4 fields of a (20, 21) grid is 4."""
    op = getattr(orc, op_name)
    a = np.ones((4, 20, 21))
    b = np.zeros((4, 20, 21))
    assert abs(orc.h2_err(op, op, a, b) ** 2 - 4.0) < 1e-3


@pytest.mark.parametrize("op_name", ["UPWIND4", "UPWIND4H2", "UPWIND9", "UPWIND9H2", "SBP4", "SBP8"])
def test_diss_annihilates_constants_and_is_negative_semidefinite(orc, op_name):
    """Structural check of the dissipation tables: H*DISS is symmetric negative semi-definite and
    kills constants (the property the upwind splitting D = Dc + H^-1 DISS relies on)."""
    op = getattr(orc, op_name)
    m, n_, d, h2, upw = orc.op_shape(op)
    if not upw:
        with pytest.raises(ValueError):
            orc.op_table(op, orc.DISS, 0)
        return
    n = 40
    I = np.eye(n)
    Dmat = orc.dissxi(op, I)  # row r of output = diss applied to e_r -> columns of the operator
    Dm = Dmat.T  # Dm[i, j]: output i from input j
    np.testing.assert_allclose(Dm @ np.ones(n), 0.0, atol=1e-12 * (n - 1))
    h = np.ones(n)
    hw = orc.op_table(op, orc.DIFF, 3)
    h[:m] = hw
    h[n - m:] = hw[::-1]
    HD = np.diag(h) @ Dm
    np.testing.assert_allclose(HD, HD.T, atol=1e-10 * (n - 1))
    assert np.linalg.eigvalsh(0.5 * (HD + HD.T)).max() < 1e-9 * (n - 1)


def linspace(a, b, n):
    """ndarray::Array1::linspace: a + step * i with step = (b - a) / (n - 1)."""
    step = (b - a) / (n - 1)
    return np.array([a + step * i for i in range(n)])


def run_with_size(orc, size, op):
    """euler/tests/convergence.rs:9-52 on the oracle (periodic euler::System, advance_upwind)."""
    nx = ny = size
    xs = linspace(-5.0, 5.0, nx)
    ys = linspace(-5.0, 5.0, ny)
    x = np.broadcast_to(xs[None, :], (ny, nx)).copy()
    y = np.broadcast_to(ys[:, None], (ny, nx)).copy()
    vort = [dict(x0=-1.0, y0=0.0, rstar=0.5, eps=1.0)]
    sysm = orc.System([dict(x=x, y=y, op_xi=op, op_eta=op, bc=[(orc.BC_THIS, 0)] * 4)], gamma=1.4, fast=True)
    sysm.set_vortex(vort, 0.5)
    sysm.init_vortex(0.0)
    time = 0.2
    dt = 0.2 * min(1.0 / (nx - 1), 1.0 / (ny - 1))
    nsteps = int(time / dt)
    sysm.advance(nsteps, dt)
    veri = orc.vortex(vort, 0.5, 1.4, nsteps * dt, x, y)
    return orc.h2_err(op, op, veri, sysm.state(0))


@pytest.mark.slow
@pytest.mark.parametrize("op_name,expected_q", [("UPWIND4", -4.0), ("UPWIND9", -8.5)])
def test_convergence(orc, op_name, expected_q):
    """euler/tests/convergence.rs:54-90"""
    op = getattr(orc, op_name)
    sizes = [25, 35, 50, 71, 100, 150, 200]
    prev = None
    q_last = None
    for size in sizes:
        e = run_with_size(orc, size, op)
        if prev is not None:
            size1, e1 = prev
            q = math.log10(e / e1) / math.log10((size * size / (size1 * size1)) ** 0.5)
            q_last = q
        prev = (size, e)
    assert q_last < expected_q, q_last


# ---- interpolation operators (sbp/src/operators/interpolation*.rs) -------------------------
def _ndarray_linspace(a, b, n):
    step = (b - a) / (n - 1)
    return a + step * np.arange(n)


@pytest.mark.parametrize("op,h2", [(0, False), (1, False), (2, False), (3, True)])
@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-11), (np.float32, 1e-4)])
def test_interpolation_exact_on_linear(orc, op, h2, dtype, tol):
    """test_interpolation_operator (interpolation.rs:52-74): coarse2fine and fine2coarse of a
    linear function (the grid itself) are exact to 1e-11 (f64; the f32 build to its precision:
    the values are about 50, so 1e-4 relative covers a few f32 ulps)."""
    nc = 101
    if h2:
        xc, xf = h2linspace(20.0, 50.0, nc), h2linspace(20.0, 50.0, 2 * (nc - 1))
    else:
        xc, xf = _ndarray_linspace(20.0, 50.0, 101), _ndarray_linspace(20.0, 50.0, 2 * nc - 1)
    xc, xf = xc.astype(dtype), xf.astype(dtype)
    f = orc.interpolate(op, False, xc, dtype)
    c = orc.interpolate(op, True, xf, dtype)
    scale = 1.0 if dtype == np.float64 else 50.0
    assert np.max(np.abs(f - xf)) <= tol * scale
    assert np.max(np.abs(c - xc)) <= tol * scale


def test_interpolation_tables_identical():
    """The library's and the oracle's interpolation tables (two headers written by
    oracle/gen_interp_coefficients.py) hold the same numbers."""
    import os
    import re
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    a = open(os.path.join(root, "summationbyparts_b200", "csrc", "interp_coefficients.h")).read()
    b = open(os.path.join(root, "oracle", "oracle_interp_coefficients.h")).read()
    da = dict(re.findall(r"#define SBPI_(\w+) ([^\n]*)", a))
    db = dict(re.findall(r"#define ORCI_(\w+) ([^\n]*)", b))
    assert da.keys() == db.keys() and len(da) == 4 * (2 * 10 + 1)
    for k in da:
        va = [float(v.strip().rstrip("f")) for v in da[k].split("//")[0].split(",")]
        vb = [float(v.strip().rstrip("f")) for v in db[k].split("//")[0].split(",")]
        assert va == vb, k
