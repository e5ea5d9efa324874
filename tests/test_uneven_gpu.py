"""Uneven batches (configuration 3): variants with different surface counts share one table
(`variant_surfaces`) and LM runs with different variable sets run in one launch per kernel.

Every result of a run must be the one the run gets alone, as a batch of its own S_v surfaces
and its own variables -- bit for bit: the trace (FP64, checked against the oracle), and whole
LM trajectories with the fused adjoint (FP64 with FMA) and with finite differences.
"""

import numpy as np
import pytest
import torch

from mikroptim_b200 import engine, workloads
from mikroptim_b200.batch import ResidualLayout
import oracle.pyoracle as po

pytestmark = pytest.mark.gpu


def _small(n=10, precision=0):
    b, st, vss, x0 = workloads.uneven(n, rings=4, spokes=8, precision=precision)
    return b, st, vss, x0


def test_uneven_merit_and_residuals_equal_each_variant_alone_and_the_oracle():
    b, st, vss, x0 = _small()
    lay = ResidualLayout(b.topology, st)
    db = engine.DeviceSystemBatch(b)
    merit = engine.merit_device(db, lay, b)
    res = engine.residuals_device(db, lay, b)
    torch.cuda.synchronize()
    port = po.port()
    for v in range(b.variants):
        one = workloads.unpad(b, v)
        lone = ResidualLayout(one.topology, st)
        m_alone = engine.merit_device(engine.DeviceSystemBatch(one), lone, one).merit.cpu().numpy()
        assert merit.merit[v].item() == m_alone[0], v
        m_port, _, _ = port.merit(one, lone)
        assert merit.merit[v].item() == m_port[0], v
        r_alone = engine.residuals_device(engine.DeviceSystemBatch(one), lone, one)
        assert torch.equal(res.opd[v], r_alone.opd[0])
        assert torch.equal(res.residuals[v], r_alone.residuals[0])


@pytest.mark.parametrize("method", ["adjoint", "fd"])
def test_uneven_lm_equals_each_run_alone(method):
    b, st, vss, x0 = _small(8, precision=2)
    lay = ResidualLayout(b.topology, st)
    opt = engine.LmOptions(max_iterations=12, gram_exact=False,
                           jacobian=engine.JACOBIAN_ADJOINT if method == "adjoint"
                           else engine.JACOBIAN_FD)
    together = engine.optimize_lm_gpu(b, lay, vss, x0, opt)
    assert together["x"].shape == (b.variants, max(v.size for v in vss))
    for v in range(b.variants):
        one = workloads.unpad(b, v)
        lone = ResidualLayout(one.topology, st)
        vs_alone = type(vss[v])(one.topology, [
            type(var)(2 if (var.type == 1 and var.surface == one.surfaces - 1) else var.type,
                      var.surface, var.lower, var.upper, var.typical)
            for var in vss[v].variables])
        alone = engine.optimize_lm_gpu(one, lone, vs_alone, x0[v][None, :], opt)
        P = vss[v].size
        assert np.array_equal(together["x"][v, :P], alone["x"][0]), v
        assert together["merit"][v] == alone["merit"][0], v
        assert together["iterations"][v] == alone["iterations"][0], v
        assert together["status"][v] == alone["status"][0], v
    assert np.all(together["merit"] <= together["history"][:, 0])


def test_uneven_fused_normal_equations_equal_each_run_alone():
    b, st, vss, x0 = _small(8, precision=0)
    lay = ResidualLayout(b.topology, st)
    gram = engine.adjoint_normal_equations_runs_device(engine.DeviceSystemBatch(b), lay, b, vss,
                                                       x0)
    for v in range(b.variants):
        one = workloads.unpad(b, v)
        lone = ResidualLayout(one.topology, st)
        vs_alone = type(vss[v])(one.topology, [
            type(var)(2 if (var.type == 1 and var.surface == one.surfaces - 1) else var.type,
                      var.surface, var.lower, var.upper, var.typical)
            for var in vss[v].variables])
        alone = engine.adjoint_normal_equations_device(engine.DeviceSystemBatch(one), lone, one,
                                                       vs_alone, x0[v][None, :])
        assert torch.equal(engine.gram_block(gram, v, vss[v].size), alone[0]), v
