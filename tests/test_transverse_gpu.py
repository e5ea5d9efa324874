"""Transverse ray errors as residual rows (ResidualSettings.transverse_weight > 0; configuration
1 asks for "transverse ray errors plus OPD"). The reference's rows are OPD only, so these rows
have no reference counterpart: they are defined in include/mikroptim_b200.h
(mkb_residual_plan.transverse_weight) and checked bit for bit against the oracle's C
restatement of that definition; the OPD and penalty rows stay those of the reference. The FD
Jacobian and the LM with the FD Jacobian carry the rows; the materialised adjoint Jacobian
differentiates them too (the image-plane intercept's reverse step seeds the sweep) and agrees
with the central differences to their own error; the fused adjoint refuses them.
"""

import dataclasses

import numpy as np
import pytest
import torch

from mikroptim_b200 import engine, workloads
from mikroptim_b200.batch import FAILURE_HARD, PRECISION_FP64, ResidualLayout
import oracle.pyoracle as po

pytestmark = pytest.mark.gpu


def _cases():
    b, st, vs, x0 = workloads.singlet(16)
    yield "singlet", b, st, vs, x0
    b, st, vs, x0 = workloads.objective(6, rings=4, spokes=8)
    yield "objective", b, st, vs, x0
    b, st, vs, x0 = workloads.ghost(5)
    yield "ghost", b, st, vs, x0
    b, st, vs, x0 = workloads.tolerancing(4, elements=3, rings=4, spokes=8)
    yield "decentered", b, st, vs, x0


@pytest.mark.parametrize("failure", [0, FAILURE_HARD])
def test_transverse_rows_and_merit_bitwise_equal_oracle(failure):
    for name, b, st, vs, x0 in _cases():
        st = dataclasses.replace(st, failure=failure, precision=PRECISION_FP64,
                                 transverse_weight=4e4)
        lay = ResidualLayout(b.topology, st)
        db = engine.DeviceSystemBatch(b)
        r = engine.residuals_device(db, lay, b)
        m = engine.merit_device(db, lay, b)
        torch.cuda.synchronize()
        ro, oo, so = po.port().residuals(b, lay)
        mo, fo, ho = po.port().merit(b, lay)
        assert r.residuals.shape[1] == lay.trace_rows == lay.rays_per_variant * (
            2 + (1 if failure == 0 else 0) + 1)
        assert np.array_equal(r.residuals.cpu().numpy(), ro), name
        assert np.array_equal(m.merit.cpu().numpy(), mo), name
        # the OPD and penalty rows are unchanged by the transverse rows
        plain = ResidualLayout(b.topology, dataclasses.replace(st, transverse_weight=0.0))
        rp = engine.residuals_device(db, plain, b)
        assert torch.equal(r.residuals[:, :plain.trace_rows], rp.residuals)
        tr = r.residuals[:, plain.trace_rows:].cpu().numpy()
        assert np.abs(tr).max() > 0.0, name


def test_fd_jacobian_and_lm_carry_the_transverse_rows():
    b, st, vs, x0 = workloads.singlet(4)
    st = dataclasses.replace(st, transverse_weight=1e4)
    lay = ResidualLayout(b.topology, st)
    db = engine.DeviceSystemBatch(b)
    J, r0, _ = engine.fd_jacobian_device(db, lay, b, vs, x0)
    Jo, ro, _ = po.port().fd_jacobian(b, lay, vs, x0)
    assert np.array_equal(J.cpu().numpy(), Jo) and np.array_equal(r0.cpu().numpy(), ro)
    opt = engine.LmOptions(max_iterations=15, jacobian=engine.JACOBIAN_FD, gram_exact=True,
                           fail_weight_factor=1.0)
    res = engine.optimize_lm_gpu(b, lay, vs, x0, opt)
    assert np.all(res["merit"] < res["history"][:, 0])
    # the materialised adjoint carries them as well (the fused adjoint does not)
    ada = engine.optimize_lm_gpu(b, lay, vs, x0, dataclasses.replace(
        opt, jacobian=engine.JACOBIAN_ADJOINT))
    assert np.all(ada["merit"] < ada["history"][:, 0])
    with pytest.raises((ValueError, NotImplementedError), match="no fused adjoint"):
        engine.optimize_lm_gpu(b, lay, vs, x0, dataclasses.replace(
            opt, jacobian=engine.JACOBIAN_ADJOINT, gram_exact=False))


@pytest.mark.parametrize("case", ["singlet", "objective", "ghost", "decentered"])
def test_adjoint_transverse_rows_agree_with_central_differences(case):
    name, b, st, vs, x0 = next(c for c in _cases() if c[0] == case)
    st = dataclasses.replace(st, transverse_weight=1e4, precision=PRECISION_FP64)
    lay = ResidualLayout(b.topology, st)
    db = engine.DeviceSystemBatch(b)
    Jf, rf, sf = engine.fd_jacobian_device(db, lay, b, vs, x0)
    Ja, ra, sa = engine.adjoint_jacobian_device(db, lay, b, vs, x0)
    assert np.array_equal(ra.cpu().numpy(), rf.cpu().numpy())
    Jf, Ja = Jf.cpu().numpy(), Ja.cpu().numpy()
    t0 = lay.rays_per_variant + lay.penalty_rows  # the transverse rows
    tf, ta = Jf[:, :, t0:], Ja[:, :, t0:]
    assert np.abs(ta).max() > 0
    # per column relative to its largest entry (central differences: O(h^2), ~1e-10 on
    # smooth rays; rays near a soft boundary leave a few larger differences)
    scale = np.maximum(np.abs(tf).max(axis=2, keepdims=True), 1e-300)
    err = np.abs(ta - tf) / scale
    assert np.median(err) <= 1e-8 and np.quantile(err, 0.99) <= 1e-4, (
        np.median(err), np.quantile(err, 0.99), err.max())
