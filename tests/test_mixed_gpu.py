"""MIXED precision: the trace in FP64 (contracted), the adjoint reverse sweep in FP32.

The forward results (OPD, status, residuals, MERIT) are those of the FP64_FMA mode bit for bit,
so the OPD error against the FP64 oracle is the FP64-FMA one. The normal equations of the
fused adjoint carry the FP32 rounding of the reverse sweep; their error against the exact
FP64 normal equations is stated here per entry, relative to sqrt(A_ii A_jj):
  singlets (configuration 1): median <= 1e-6, every entry <= 1e-3.
"""

import dataclasses

import numpy as np
import pytest
import torch

from mikroptim_b200 import engine, workloads
from mikroptim_b200.batch import PRECISION_FP64, PRECISION_FP64_FMA, PRECISION_MIXED, ResidualLayout

pytestmark = pytest.mark.gpu


def _layout(b, st, precision):
    return ResidualLayout(b.topology, dataclasses.replace(st, precision=precision))


@pytest.mark.parametrize("make", [workloads.singlet, workloads.objective])
def test_mixed_forward_equals_fp64_fma(make):
    b, st, vs, x0 = make(24)
    db = engine.DeviceSystemBatch(b)
    r_mixed = engine.residuals_device(db, _layout(b, st, PRECISION_MIXED), b)
    r_fma = engine.residuals_device(db, _layout(b, st, PRECISION_FP64_FMA), b)
    m_mixed = engine.merit_device(db, _layout(b, st, PRECISION_MIXED), b)
    m_fma = engine.merit_device(db, _layout(b, st, PRECISION_FP64_FMA), b)
    torch.cuda.synchronize()
    assert torch.equal(r_mixed.residuals, r_fma.residuals)
    assert torch.equal(r_mixed.opd, r_fma.opd)
    assert torch.equal(r_mixed.status, r_fma.status)
    assert torch.equal(m_mixed.merit, m_fma.merit)


def _relative_gram_error(b, st, vs, x0, precision):
    db = engine.DeviceSystemBatch(b)
    ref = engine.adjoint_normal_equations_device(db, _layout(b, st, PRECISION_FP64), b, vs,
                                                 x0).cpu().numpy()
    got = engine.adjoint_normal_equations_device(db, _layout(b, st, precision), b, vs,
                                                 x0).cpu().numpy()
    d = np.abs(np.diagonal(ref, axis1=1, axis2=2))
    d = np.maximum(d, 1e-20 * d.max(axis=1, keepdims=True) + 1e-300)
    return got, np.abs(got - ref) / np.sqrt(d[:, :, None] * d[:, None, :])


def test_mixed_normal_equations_error_on_singlets():
    b, st, vs, x0 = workloads.singlet(128)
    got, err = _relative_gram_error(b, st, vs, x0, PRECISION_MIXED)
    assert np.isfinite(got).all()
    assert np.median(err) <= 1e-6, np.median(err)
    assert err.max() <= 1e-3, err.max()


def test_mixed_lm_reaches_fp64_optimum_on_singlets():
    """LM with the FP32 reverse sweep: the steps differ, the optimum does not."""
    b, st, vs, x0 = workloads.singlet(16)
    opt = engine.LmOptions(max_iterations=40, jacobian=engine.JACOBIAN_ADJOINT, gram_exact=False)
    mixed = engine.optimize_lm_gpu(b, _layout(b, st, PRECISION_MIXED), vs, x0, opt)
    fma = engine.optimize_lm_gpu(b, _layout(b, st, PRECISION_FP64_FMA), vs, x0, opt)
    assert np.all(mixed["merit"] < mixed["history"][:, 0])
    assert np.allclose(mixed["merit"], fma["merit"], rtol=1e-6, atol=1e-12)
