"""GPU batched Levenberg-Marquardt against the reference's own optimize_lm_cpu.

With precision FP64 and the FMA-chain normal equations, every run's trajectory -- x, merit,
status, iteration and acceptance counts, damping and the merit history -- equals the
reference's host loop (compiled from its own sources, oracle/_ref) bit for bit, for the
adjoint and the finite-difference Jacobian. The DMMA normal equations reach the same optimum
within tolerance.
"""

import numpy as np
import pytest

from conftest import has_reference_build
from mikroptim_b200 import engine, workloads
from mikroptim_b200.batch import ResidualLayout
import oracle.pyoracle as po

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_reference_build(), reason="reference build missing")]


def run_both(method, runs=6, max_iterations=25, gram_exact=True, precision=0):
    b, st, vs, x0 = workloads.singlet(runs)
    lay = ResidualLayout(b.topology, st)
    lay_gpu = ResidualLayout(b.topology, type(st)(rings=st.rings, spokes=st.spokes,
                                                  failure=st.failure, precision=precision))
    opt = engine.LmOptions(max_iterations=max_iterations,
                           jacobian=engine.JACOBIAN_ADJOINT if method == "adjoint"
                           else engine.JACOBIAN_FD, gram_exact=gram_exact,
                           fail_weight_factor=1.0)
    g = engine.optimize_lm_gpu(b, lay_gpu, vs, x0, opt)
    r = po.reference().optimize_lm(b, lay, vs, x0, max_iterations=max_iterations,
                                   method=method, penalty_rounds=1, threads=4)
    return g, r


@pytest.mark.parametrize("method", ["adjoint", "fd"])
def test_lm_trajectories_bitwise_equal_reference(method):
    g, r = run_both(method)
    assert np.array_equal(g["status"], r["status"]), (g["status"], r["status"])
    assert np.array_equal(g["iterations"], r["iterations"])
    assert np.array_equal(g["accepted"], r["accepted"])
    assert np.array_equal(g["x"], r["x"])
    assert np.array_equal(g["merit"], r["merit"])
    assert np.array_equal(np.isnan(g["history"]), np.isnan(r["history"]))
    h = ~np.isnan(r["history"])
    assert np.array_equal(g["history"][h], r["history"][h])
    # the optimiser actually improves every run
    assert np.all(g["merit"] < g["history"][:, 0])


def test_lm_dmma_normal_equations_reach_same_optimum():
    g, r = run_both("adjoint", gram_exact=False)
    assert np.allclose(g["merit"], r["merit"], rtol=1e-6, atol=1e-12)
    assert np.allclose(g["x"], r["x"], rtol=1e-6, atol=1e-9)


def test_lm_fused_adjoint_fma_reaches_same_optimum():
    """FMA arithmetic with the fused adjoint + DMMA normal equations (the fast path)."""
    g, r = run_both("adjoint", gram_exact=False, precision=2)
    assert np.all(g["status"] > 0)
    assert np.allclose(g["merit"], r["merit"], rtol=1e-6, atol=1e-12)
    assert np.allclose(g["x"], r["x"], rtol=1e-6, atol=1e-9)


@pytest.mark.parametrize("method", ["adjoint", "fd"])
def test_lm_cycle_graph_replay_equals_direct_cycles(method):
    """A cycle is a fixed launch sequence with device masks: replaying its CUDA graph advances
    the runs exactly as calling the cycle does (bit for bit), FP64 exact path."""
    import torch
    b, st, vs, x0 = workloads.singlet(8)
    lay = ResidualLayout(b.topology, st)
    opt = engine.LmOptions(max_iterations=30, gram_exact=method == "fd",
                           jacobian=engine.JACOBIAN_ADJOINT if method == "adjoint"
                           else engine.JACOBIAN_FD)
    db = engine.DeviceSystemBatch(b)
    direct = engine.DeviceLm(db, lay, b, vs, opt, b.variants)
    direct.start(x0)
    for _ in range(12):
        direct.cycle()
    graphed = engine.DeviceLm(db, lay, b, vs, opt, b.variants)
    graphed.start(x0)
    graphed.cycle()
    graph = graphed.capture()
    for _ in range(11):
        graph.replay()
    torch.cuda.synchronize()
    a, g = direct.results(), graphed.results()
    for key in ("x", "merit", "status", "iterations", "accepted", "jacobians", "damping"):
        assert np.array_equal(a[key], g[key]), key
    h = ~np.isnan(a["history"])
    assert np.array_equal(np.isnan(a["history"]), np.isnan(g["history"]))
    assert np.array_equal(a["history"][h], g["history"][h])
    assert int(a["iterations"].sum()) > 0


def test_lm_penalty_rounds_bitwise_equal_reference():
    """Outer soft-failure penalty rounds (optimize_lm_rounds): objectives at NA 0.95 end with
    vignetted rays, so runs restart with w_fail x 10 up to 1e14; every run's end point, merit,
    status and summed counters equal the reference's optimize_lm_cpu with its default rounds."""
    b, st, vs, x0 = workloads.objective(4, rings=3, spokes=6)
    lay = ResidualLayout(b.topology, st)
    opt = engine.LmOptions(max_iterations=4, jacobian=engine.JACOBIAN_ADJOINT, gram_exact=True)
    g = engine.optimize_lm_gpu(b, lay, vs, x0, opt)
    r = po.reference().optimize_lm(b, lay, vs, x0, max_iterations=4, method="adjoint",
                                   penalty_rounds=2, threads=4)
    assert np.any(g["penalty_rounds"] > 1)
    for k in ("status", "iterations", "accepted", "x", "merit"):
        assert np.array_equal(g[k], r[k]), k
