"""Extra residual rows in the device LM (the reference's LmOptions::jacobian.extra): paraxial
constraints -- focal length, working distance, Petzval curvature -- evaluated on the host by the
reference's own paraxial_residuals, their Jacobian by central differences with the FD
Jacobian's pattern, appended after the trace rows of the normal equations, and sum r_e^2 added
to every merit. With the exact normal equations the LM trajectories equal the reference's
optimize_lm_cpu with the same constraints bit for bit."""

import math

import numpy as np
import pytest

from conftest import has_reference_build
from mikroptim_b200 import engine, workloads
from mikroptim_b200.batch import ResidualLayout
import oracle.pyoracle as po

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_reference_build(), reason="reference build missing")]

CONSTRAINTS = [(0, 0, 4.0, 48.0), (2, 1, 1.0, 47.5), (4, 2, 1e4, 0.001)]


def problem(n=4):
    b, st, vs, x0 = workloads.singlet(n)
    lay = ResidualLayout(b.topology, st)
    R = po.reference()
    extra = engine.ExtraResiduals(
        len(CONSTRAINTS), lambda one, v, out: out.__setitem__(
            slice(None), R.paraxial_residuals(one, lay, v, CONSTRAINTS)))
    return b, lay, vs, x0, extra


@pytest.mark.parametrize("method", ["adjoint", "fd"])
def test_lm_with_constraints_bitwise_equal_reference(method):
    b, lay, vs, x0, extra = problem(4)
    opt = engine.LmOptions(max_iterations=8,
                           jacobian=engine.JACOBIAN_ADJOINT if method == "adjoint"
                           else engine.JACOBIAN_FD, gram_exact=True, fail_weight_factor=1.0,
                           extra=extra)
    g = engine.optimize_lm_gpu(b, lay, vs, x0, opt)
    r = po.reference().optimize_lm(b, lay, vs, x0, max_iterations=8, method=method,
                                   penalty_rounds=1, threads=4, constraints=CONSTRAINTS)
    for k in ("status", "iterations", "accepted", "x", "merit"):
        assert np.array_equal(g[k], r[k]), k
    assert np.array_equal(g["history"], r["history"], equal_nan=True)


def test_constraints_move_the_optimum_and_fused_path_agrees():
    """The constraints change the result, the merit (trace rows plus constraint rows) falls
    from the start, and the fused tensor-core normal equations reach the exact path's merit
    within 1e-6 relative."""
    b, lay, vs, x0, extra = problem(4)
    base = engine.LmOptions(max_iterations=30, gram_exact=True, fail_weight_factor=1.0)
    plain = engine.optimize_lm_gpu(b, lay, vs, x0, base)
    exact = engine.optimize_lm_gpu(b, lay, vs, x0, engine.LmOptions(
        max_iterations=30, gram_exact=True, fail_weight_factor=1.0, extra=extra))
    fused = engine.optimize_lm_gpu(b, lay, vs, x0, engine.LmOptions(
        max_iterations=30, gram_exact=False, fail_weight_factor=1.0, extra=extra))
    assert not np.allclose(plain["x"], exact["x"])
    assert np.all(exact["merit"] < exact["history"][:, 0])
    assert np.all(np.abs(fused["merit"] - exact["merit"]) <= 1e-6 * np.abs(exact["merit"]))


TRACE = [(1, 0, 100.0, 4.8), (2, 0, 50.0, 4.7), (2, 1, 1e3, 0.9995)]


def trace_rows(one, v, ext, out):
    """The same rows as the reference driver's: semi-diameter and incidence-angle limits."""
    for i, (s, kind, w, lim) in enumerate(TRACE):
        q = ext[s][0] - lim if kind == 0 else lim - ext[s][1]
        out[i] = math.sqrt(w) * max(0.0, q)


@pytest.mark.parametrize("method", ["adjoint", "fd"])
def test_lm_with_trace_dependent_rows_bitwise_equal_reference(method):
    """Rows from the per-surface extrema (the reference's trace_extra: each FD point and each
    trial point traced with its own extrema), together with paraxial rows."""
    b, lay, vs, x0, extra = problem(4)
    opt = engine.LmOptions(max_iterations=8,
                           jacobian=engine.JACOBIAN_ADJOINT if method == "adjoint"
                           else engine.JACOBIAN_FD, gram_exact=True, fail_weight_factor=1.0,
                           extra=extra,
                           trace_extra=engine.TraceExtraResiduals(len(TRACE), trace_rows))
    g = engine.optimize_lm_gpu(b, lay, vs, x0, opt)
    r = po.reference().optimize_lm(b, lay, vs, x0, max_iterations=8, method=method,
                                   penalty_rounds=1, threads=4, constraints=CONSTRAINTS,
                                   trace_constraints=TRACE)
    for k in ("status", "iterations", "accepted", "x", "merit"):
        assert np.array_equal(g[k], r[k]), k
    assert np.array_equal(g["history"], r["history"], equal_nan=True)
