"""GPU parity with ghost plates (thin virtual plates with a Legendre thickness profile in an
air gap, trace/ghost_plate.hpp), their profile coefficients among the variables.

Precision FP64 reproduces the CPU oracle -- pinned bit for bit to the reference on these
batches, Jacobian columns of the coefficients included (tests/test_oracle.py) -- exactly:
RESIDUALS, MERIT, the FD and adjoint Jacobians and the LM trajectories of the reference's
optimize_lm_cpu. The fused adjoint normal equations are checked within the tolerances of the
coaxial tests, and a decentered batch with ghost plates exercises both features at once.
"""

import numpy as np
import pytest
import torch

from conftest import has_reference_build
from mikroptim_b200 import engine, workloads
from mikroptim_b200.batch import (PRECISION_FP64, PRECISION_FP64_FMA, PRECISION_MIXED,
                                  ResidualLayout, make_non_coaxial)
import oracle.pyoracle as po

pytestmark = pytest.mark.gpu


def batch(n=8, precision=PRECISION_FP64, **kw):
    b, st, vs, x0 = workloads.ghost(n, **kw)
    st.precision = precision
    return b, st, vs, x0, ResidualLayout(b.topology, st)


def to_np(*ts):
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in ts]


def gram_error(a, b):
    d = np.abs(np.diagonal(b, axis1=-2, axis2=-1))
    d = np.maximum(d, 1e-20 * d.max(axis=-1, keepdims=True) + 1e-300)
    return np.abs(a - b) / np.sqrt(d[..., :, None] * d[..., None, :])


def test_residuals_and_merit_bitwise():
    b, st, vs, x0, lay = batch(64)
    eng = engine.TraceEngine(0)
    r = eng.run(b, engine.TraceMode.RESIDUALS,
                engine.TraceSettings(lay.settings, opd=True)).residuals
    m = eng.run(b, engine.TraceMode.MERIT, lay.settings).merit
    ro, oo, so = po.port().residuals(b, lay, threads=8)
    mo, fo, ho = po.port().merit(b, lay, threads=8)
    assert np.array_equal(r.residuals, ro) and np.array_equal(r.opd, oo)
    assert np.array_equal(r.status, so)
    assert np.array_equal(m.merit, mo) and np.array_equal(m.failed, fo)


def test_fd_and_adjoint_jacobian_bitwise():
    b, st, vs, x0, lay = batch(6)
    db = engine.DeviceSystemBatch(b)
    Jf, rf, ch = to_np(*engine.fd_jacobian_device(db, lay, b, vs, x0))
    Jfo, rfo, cho = po.port().fd_jacobian(b, lay, vs, x0, threads=8)
    assert np.array_equal(Jf, Jfo) and np.array_equal(rf, rfo) and np.array_equal(ch, cho)
    Ja, ra, sa = to_np(*engine.adjoint_jacobian_device(db, lay, b, vs, x0))
    Jao, rao, sao = po.port().adjoint_jacobian(b, lay, vs, x0, threads=8)
    assert np.array_equal(Ja, Jao) and np.array_equal(ra, rao)


@pytest.mark.parametrize("precision,tol", [(PRECISION_FP64, 1e-10),
                                           (PRECISION_FP64_FMA, 1e-9)])
def test_fused_normal_equations_match_exact(precision, tol):
    b, st, vs, x0, lay = batch(16)
    db = engine.DeviceSystemBatch(b)
    J, r0, _ = engine.adjoint_jacobian_device(db, lay, b, vs, x0)
    ref = engine.normal_equations_device(J, r0, True)
    b2, st2, vs2, x02, lay2 = batch(16, precision=precision)
    fused = engine.adjoint_normal_equations_device(engine.DeviceSystemBatch(b2), lay2, b2, vs2,
                                                   x02)
    ref, fused = to_np(ref, fused)
    assert gram_error(fused, ref).max() <= tol


def test_mixed_normal_equations_within_the_mixed_bar():
    """MIXED (FP32 reverse sweep): the bar of the coaxial MIXED tests, median relative entry
    error <= 1e-6 and every entry <= 1e-3 of sqrt(A_ii A_jj)."""
    b, st, vs, x0, lay = batch(16)
    db = engine.DeviceSystemBatch(b)
    J, r0, _ = engine.adjoint_jacobian_device(db, lay, b, vs, x0)
    ref = engine.normal_equations_device(J, r0, True)
    b2, st2, vs2, x02, lay2 = batch(16, precision=PRECISION_MIXED)
    fused = engine.adjoint_normal_equations_device(engine.DeviceSystemBatch(b2), lay2, b2, vs2,
                                                   x02)
    ref, fused = to_np(ref, fused)
    err = gram_error(fused, ref)
    assert np.median(err) <= 1e-6 and err.max() <= 1e-3, (np.median(err), err.max())


def test_decentered_batch_with_ghost_plates_bitwise():
    b, st, vs, x0 = workloads.ghost(6, rings=4, spokes=8)
    nc = make_non_coaxial(b)
    rng = np.random.default_rng(7)
    nc.decenter_tilt[:, 1:, :2] = 0.01 * rng.standard_normal((6, b.surfaces - 1, 2))
    nc.decenter_tilt[:, 1:, 2:] = 3e-4 * rng.standard_normal((6, b.surfaces - 1, 2))
    lay = ResidualLayout(nc.topology, st)
    db = engine.DeviceSystemBatch(nc)
    r = engine.TraceEngine(0).run(nc, engine.TraceMode.RESIDUALS, lay.settings).residuals
    ro, oo, so = po.port().residuals(nc, lay, threads=8)
    assert np.array_equal(r.residuals, ro) and np.array_equal(r.status, so)
    Ja, ra, _ = to_np(*engine.adjoint_jacobian_device(db, lay, nc, vs, x0))
    Jao, rao, _ = po.port().adjoint_jacobian(nc, lay, vs, x0, threads=8)
    assert np.array_equal(Ja, Jao) and np.array_equal(ra, rao)


@pytest.mark.skipif(not has_reference_build(), reason="reference build missing")
@pytest.mark.parametrize("method", ["adjoint", "fd"])
def test_lm_trajectories_bitwise_equal_reference(method):
    b, st, vs, x0, lay = batch(4)
    opt = engine.LmOptions(max_iterations=8,
                           jacobian=engine.JACOBIAN_ADJOINT if method == "adjoint"
                           else engine.JACOBIAN_FD, gram_exact=True, fail_weight_factor=1.0)
    g = engine.optimize_lm_gpu(b, lay, vs, x0, opt)
    r = po.reference().optimize_lm(b, lay, vs, x0, max_iterations=8, method=method,
                                   penalty_rounds=1, threads=4)
    for k in ("status", "iterations", "accepted", "x", "merit"):
        assert np.array_equal(g[k], r[k]), k
