"""torch.autograd over the device path (mikroptim_b200.autograd): merit and residual rows of
run points as differentiable functions with adjoint gradients, and the device-side
VariableSet::apply they evaluate the points with."""

import numpy as np
import pytest
import torch

from mikroptim_b200 import autograd as ag
from mikroptim_b200 import engine, workloads
from mikroptim_b200.batch import ResidualLayout

pytestmark = pytest.mark.gpu


def _problem(runs=6, make=workloads.singlet):
    b, st, vs, x0 = make(runs)
    lay = ResidualLayout(b.topology, st)
    return b, lay, vs, x0, ag.AdjointProblem(b, lay, vs)


def test_device_apply_equals_host_apply():
    b, lay, vs, x0, prob = _problem()
    x = x0 * (1.0 + 1e-3 * np.arange(x0.size).reshape(x0.shape) / x0.size)
    host = b.subset(0, b.variants)
    for v in range(b.variants):
        vs.apply(host, v, x[v])
    want = engine.DeviceSystemBatch(host).records
    got = prob.records_at(torch.from_numpy(x)).records
    assert torch.equal(got, want)


def test_merit_forward_equals_trace_of_applied_batch():
    b, lay, vs, x0, prob = _problem()
    x = torch.from_numpy(x0 * 1.001).cuda()
    host = b.subset(0, b.variants)
    for v in range(b.variants):
        vs.apply(host, v, x0[v] * 1.001)
    want = engine.TraceEngine(0).run(host, engine.TraceMode.MERIT, lay.settings).merit.merit
    got = ag.merit(x, prob).cpu().numpy()
    assert np.array_equal(got, want)


def test_merit_gradient_matches_central_differences():
    b, lay, vs, x0, prob = _problem()
    x = torch.from_numpy(x0.copy()).cuda().requires_grad_(True)
    ag.merit(x, prob).sum().backward()
    grad = x.grad.cpu().numpy()
    fd = np.zeros_like(x0)
    for k in range(vs.size):
        h = 1e-6 * np.maximum(np.abs(x0[:, k]), 1e-3)
        xp, xm = x0.copy(), x0.copy()
        xp[:, k] += h
        xm[:, k] -= h
        mp = prob.merit(torch.from_numpy(xp)).cpu().numpy()
        mm = prob.merit(torch.from_numpy(xm)).cpu().numpy()
        fd[:, k] = (mp - mm) / (2 * h)
    scale = np.abs(grad).max(axis=1, keepdims=True)
    assert np.all(np.abs(grad - fd) <= 1e-4 * scale + 1e-12), np.abs(grad - fd).max()


def test_residual_vjp_agrees_with_merit_gradient_and_gram():
    b, lay, vs, x0, prob = _problem()
    x = torch.from_numpy(x0.copy()).cuda().requires_grad_(True)
    r = ag.residuals(x, prob)
    (r * r).sum().backward()
    g_res = x.grad.cpu().numpy()
    gram = prob.normal_equations(torch.from_numpy(x0)).cpu().numpy()
    P = vs.size
    assert np.allclose(g_res, 2 * gram[:, :P, P], rtol=1e-9, atol=1e-12)
    merit = prob.merit(torch.from_numpy(x0)).cpu().numpy()
    assert np.allclose(gram[:, P, P], merit, rtol=1e-11, atol=0)
