"""Uneven batches (configuration 3): variants with different surface counts share one table
(`variant_surfaces`) and LM runs with different variable sets run in one launch per kernel.

Every result of a run must be the one the run gets alone, as a batch of its own S_v surfaces
and its own variables -- bit for bit: the trace (FP64, checked against the oracle), and whole
LM trajectories with the fused adjoint (FP64 with FMA) and with finite differences.
"""

import dataclasses

import numpy as np
import pytest
import torch

from mikroptim_b200 import engine, workloads
from mikroptim_b200.batch import PRECISION_FP64, PRECISION_FP64_FMA, PRECISION_MIXED, ResidualLayout
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


def _gram_errors(ref, got):
    d = np.abs(np.diagonal(ref))
    d = np.maximum(d, 1e-20 * d.max() + 1e-300)
    return (np.abs(got - ref) / np.sqrt(d[:, None] * d[None, :])).ravel()


def test_uneven_mixed_fused_normal_equations_both_launches_against_fp64():
    """The headline kernel instance: the fused adjoint + normal equations in MIXED precision
    (FP64 trace, FP32 reverse sweep and FP32 derivative rows) on configuration-3 runs with full
    16 x 32 pupils, through both of its launches -- runs with <= 31 variables, and the launch
    sized for the widest run -- against the FP64 fused normal equations (separately rounded
    operations, within 1e-10 of the exact ones). Bar per entry, relative to sqrt(A_ii A_jj):
    median <= 1e-6 (narrow runs) and 1e-4 (wide runs: longer systems, 17 to 30 surfaces,
    accumulate more FP32 rounding in the sweep), every entry <= 2e-3. Measured on 256 runs:
    median 1.9e-7 / 2.5e-5, maximum 5.5e-4 / 7.1e-4."""
    b, st, vss, x0 = workloads.uneven(96)
    P = np.array([v.size for v in vss])
    assert (P > 31).sum() >= 16 and (P <= 31).sum() >= 16
    db = engine.DeviceSystemBatch(b)
    lay = {p: ResidualLayout(b.topology, dataclasses.replace(st, precision=p))
           for p in (PRECISION_FP64, PRECISION_MIXED)}
    ref = engine.adjoint_normal_equations_runs_device(db, lay[PRECISION_FP64], b, vss, x0)
    got = engine.adjoint_normal_equations_runs_device(db, lay[PRECISION_MIXED], b, vss, x0)
    torch.cuda.synchronize()
    errs = {"narrow": [], "wide": []}
    for v in range(b.variants):
        r = engine.gram_block(ref, v, vss[v].size).cpu().numpy()
        g = engine.gram_block(got, v, vss[v].size).cpu().numpy()
        assert np.isfinite(g).all(), v
        errs["wide" if vss[v].size > 31 else "narrow"].append(_gram_errors(r, g))
    for kind, bar in (("narrow", 1e-6), ("wide", 1e-4)):
        e = np.concatenate(errs[kind])
        assert np.median(e) <= bar, (kind, np.median(e))
        assert e.max() <= 2e-3, (kind, e.max())


def test_uneven_mixed_lm_ends_where_the_fp64_lm_does():
    """100 LM iterations on configuration-3 runs. Almost every run is still iterating at the
    limit in every precision (ill-conditioned thickness columns), so the end points are points
    on unconverged trajectories, and the FP32 sweep's slightly different steps put MIXED on a
    different trajectory after a few cycles. What holds is that MIXED ends as low as FP64 does:
    the geometric mean of merit_MIXED / merit_FP64 is at most 1.03 (measured 1.006 on plate-free
    systems, 0.969 with the zero-power ghost plate of configuration 3), MIXED
    ends at least as low in a third of the runs or more (measured 48 %), and every run
    decreases its merit. The FP64 reference is the fused kernel with separately rounded
    operations."""
    b, st, vss, x0 = workloads.uneven(48)
    opt = engine.LmOptions(max_iterations=100, jacobian=engine.JACOBIAN_ADJOINT, gram_exact=False)
    lay = {p: ResidualLayout(b.topology, dataclasses.replace(st, precision=p))
           for p in (PRECISION_FP64, PRECISION_MIXED)}
    mixed = engine.optimize_lm_gpu(b, lay[PRECISION_MIXED], vss, x0, opt)
    fp64 = engine.optimize_lm_gpu(b, lay[PRECISION_FP64], vss, x0, opt)
    assert np.all(mixed["merit"] < mixed["history"][:, 0])
    ratio = mixed["merit"] / fp64["merit"]
    assert np.mean(np.log(ratio)) <= 0.03, ratio  # MIXED may end lower, not 3 % higher
    assert np.mean(ratio <= 1.0 + 1e-9) >= 1.0 / 3.0, ratio


@pytest.mark.parametrize("precision", [PRECISION_MIXED, PRECISION_FP64_FMA, PRECISION_FP64])
def test_instance_without_the_plate_reverse_step_equals_the_full_one(precision):
    """Every run's variables lie behind the ghost plate at surface 1, so the launch takes the
    fused instance without the plate's reverse step; a thickness[0] variable in run 0 puts the
    plate on that run's sweep and the launch back on the full instance. The other runs'
    normal equations are the same bits either way."""
    from mikroptim_b200.batch import SURFACE_GHOST_PLATE, VAR_THICKNESS, Variable, VariableSet
    b, st, vss, x0 = _small(24, precision=precision)
    assert b.topology.ghost_plates == 1 and b.topology.type[1] == SURFACE_GHOST_PLATE
    lay = ResidualLayout(b.topology, st)
    db = engine.DeviceSystemBatch(b)
    g_cut = engine.adjoint_normal_equations_runs_device(db, lay, b, vss, x0)
    vss2, x2 = list(vss), list(x0)
    vss2[0] = VariableSet(vss[0].topology, list(vss[0].variables) +
                          [Variable(VAR_THICKNESS, 0, 0.1, 5.0, 1.0)])
    x2[0] = vss2[0].extract(b, 0)
    g_full = engine.adjoint_normal_equations_runs_device(db, lay, b, vss2, x2)
    torch.cuda.synchronize()
    for i in range(1, b.variants):
        P = vss[i].size
        assert np.array_equal(engine.gram_block(g_cut, i, P).cpu().numpy(),
                              engine.gram_block(g_full, i, P).cpu().numpy()), i
    # run 0 gained the column of thickness[0]: its block is one wider and not zero there
    blk = engine.gram_block(g_full, 0, vss2[0].size).cpu().numpy()
    assert blk[vss2[0].size - 1, vss2[0].size - 1] > 0
