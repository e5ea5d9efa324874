"""GPU parity with glass variables: the Buchdahl coordinates (n0, nu1, nu2) of one element's
glass among the configuration-2 variables (P = 32). Writing them recomputes the medium's index
at every wavelength on the device; the reverse sweeps carry each medium's index adjoint into
the glass columns. Precision FP64 reproduces the CPU oracle -- pinned bit for bit to the
reference here (tests/test_oracle.py) -- exactly: FD and adjoint Jacobians and the LM
trajectories of the reference's optimize_lm_cpu; the fused normal equations agree within the
tolerances of the coaxial tests. Those use NA 0.3: at the generator's NA 0.95 one of the first
six systems has a ray so close to grazing that its columns lose ~1e-4 (FP64_FMA, with or
without glass) of sqrt(A_ii A_jj) to the forward trace's rounding alone.
"""

import numpy as np
import pytest
import torch

from conftest import has_reference_build
from mikroptim_b200 import engine, workloads
from mikroptim_b200.batch import (PRECISION_FP64, PRECISION_FP64_FMA, PRECISION_MIXED,
                                  ResidualLayout)
import oracle.pyoracle as po

pytestmark = pytest.mark.gpu


def batch(n=4, precision=PRECISION_FP64, na=0.95):
    b, st, vs, x0 = workloads.objective(n, rings=3, spokes=6, glass=True, na=na)
    st.precision = precision
    return b, st, vs, x0, ResidualLayout(b.topology, st)


def to_np(*ts):
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in ts]


def test_fd_and_adjoint_jacobian_bitwise():
    b, st, vs, x0, lay = batch()
    db = engine.DeviceSystemBatch(b)
    Jf, rf, ch = to_np(*engine.fd_jacobian_device(db, lay, b, vs, x0))
    Jfo, rfo, cho = po.port().fd_jacobian(b, lay, vs, x0, threads=8)
    assert np.array_equal(Jf, Jfo) and np.array_equal(rf, rfo) and np.array_equal(ch, cho)
    Ja, ra, sa = to_np(*engine.adjoint_jacobian_device(db, lay, b, vs, x0))
    Jao, rao, sao = po.port().adjoint_jacobian(b, lay, vs, x0, threads=8)
    assert np.array_equal(Ja, Jao) and np.array_equal(ra, rao)
    assert np.any(Ja[:, -3:, :] != 0.0)


@pytest.mark.parametrize("precision,tol", [(PRECISION_FP64, 1e-10),
                                           (PRECISION_FP64_FMA, 1e-9)])
def test_fused_normal_equations_match_exact(precision, tol):
    b, st, vs, x0, lay = batch(16, na=0.3)
    db = engine.DeviceSystemBatch(b)
    J, r0, _ = engine.adjoint_jacobian_device(db, lay, b, vs, x0)
    ref = engine.normal_equations_device(J, r0, True)
    b2, st2, vs2, x02, lay2 = batch(16, precision=precision, na=0.3)
    fused = engine.adjoint_normal_equations_device(engine.DeviceSystemBatch(b2), lay2, b2, vs2,
                                                   x02)
    ref, fused = to_np(ref, fused)
    d = np.abs(np.diagonal(ref, axis1=1, axis2=2))
    d = np.maximum(d, 1e-20 * d.max(axis=1, keepdims=True) + 1e-300)
    err = np.abs(fused - ref) / np.sqrt(d[:, :, None] * d[:, None, :])
    assert err.max() <= tol, err.max()


def test_mixed_normal_equations_within_the_mixed_bar():
    """MIXED (FP32 reverse sweep, glass columns included): the bar of the coaxial MIXED tests,
    median relative entry error <= 1e-6 and every entry <= 1e-3 of sqrt(A_ii A_jj)."""
    b, st, vs, x0, lay = batch(16, na=0.3)
    db = engine.DeviceSystemBatch(b)
    J, r0, _ = engine.adjoint_jacobian_device(db, lay, b, vs, x0)
    ref = engine.normal_equations_device(J, r0, True)
    b2, st2, vs2, x02, lay2 = batch(16, precision=PRECISION_MIXED, na=0.3)
    fused = engine.adjoint_normal_equations_device(engine.DeviceSystemBatch(b2), lay2, b2, vs2,
                                                   x02)
    ref, fused = to_np(ref, fused)
    d = np.abs(np.diagonal(ref, axis1=1, axis2=2))
    d = np.maximum(d, 1e-20 * d.max(axis=1, keepdims=True) + 1e-300)
    err = np.abs(fused - ref) / np.sqrt(d[:, :, None] * d[:, None, :])
    assert np.median(err) <= 1e-6 and err.max() <= 1e-3, (np.median(err), err.max())


@pytest.mark.skipif(not has_reference_build(), reason="reference build missing")
@pytest.mark.parametrize("method", ["adjoint", "fd"])
def test_lm_trajectories_bitwise_equal_reference(method):
    b, st, vs, x0, lay = batch(3)
    opt = engine.LmOptions(max_iterations=5,
                           jacobian=engine.JACOBIAN_ADJOINT if method == "adjoint"
                           else engine.JACOBIAN_FD, gram_exact=True, fail_weight_factor=1.0)
    g = engine.optimize_lm_gpu(b, lay, vs, x0, opt)
    r = po.reference().optimize_lm(b, lay, vs, x0, max_iterations=5, method=method,
                                   penalty_rounds=1, threads=4)
    for k in ("status", "iterations", "accepted", "x", "merit"):
        assert np.array_equal(g[k], r[k]), k
