"""GPU parity of the Jacobians and normal equations against the CPU oracle.

Precision FP64: the FD Jacobian, the adjoint Jacobian (checkpointed reverse sweep + piston
projection) and the FMA-chain normal equations reproduce the oracle -- which equals the
reference's fd_jacobian_cpu / adjoint_jacobian_cpu / normal_equations_host bit for bit --
exactly. The FMA-contracted and tensor-core (DMMA) variants are checked against tolerances.
"""

import numpy as np
import pytest
import torch

from mikroptim_b200 import engine, workloads
from mikroptim_b200.batch import PRECISION_FP64, PRECISION_FP64_FMA, ResidualLayout
import oracle.pyoracle as po

pytestmark = pytest.mark.gpu


def setup(make, n, precision=PRECISION_FP64, **kw):
    b, st, vs, x0 = make(n, **kw)
    st.precision = precision
    lay = ResidualLayout(b.topology, st)
    db = engine.DeviceSystemBatch(b)
    return b, st, vs, x0, lay, db


def to_np(*ts):
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in ts]


def test_fd_jacobian_bitwise_singlet():
    b, st, vs, x0, lay, db = setup(workloads.singlet, 24)
    J, r0, ch = to_np(*engine.fd_jacobian_device(db, lay, b, vs, x0))
    Jo, r0o, cho = po.port().fd_jacobian(b, lay, vs, x0, threads=8)
    assert np.array_equal(r0, r0o)
    assert np.array_equal(J, Jo)
    assert np.array_equal(ch, cho)


def test_fd_jacobian_bitwise_objective_chunked():
    b, st, vs, x0, lay, db = setup(workloads.objective, 5, rings=6, spokes=8)
    J, r0, ch = to_np(*engine.fd_jacobian_device(db, lay, b, vs, x0, chunk_runs=2))
    Jo, r0o, cho = po.port().fd_jacobian(b, lay, vs, x0, threads=8)
    assert np.array_equal(r0, r0o)
    assert np.array_equal(J, Jo)
    assert np.array_equal(ch, cho)


def test_fd_jacobian_one_template_for_all_runs():
    b, st, vs, x0, lay, db = setup(workloads.singlet, 1)
    xs = np.stack([x0[0], x0[0] * (1 + 1e-3), x0[0] * (1 - 2e-3)])
    J, r0, ch = to_np(*engine.fd_jacobian_device(db, lay, b, vs, xs))
    Jo, r0o, cho = po.port().fd_jacobian(b, lay, vs, xs)
    assert np.array_equal(J, Jo) and np.array_equal(r0, r0o)


def test_adjoint_jacobian_bitwise_singlet():
    b, st, vs, x0, lay, db = setup(workloads.singlet, 32)
    J, r0, s = to_np(*engine.adjoint_jacobian_device(db, lay, b, vs, x0))
    Jo, r0o, so = po.port().adjoint_jacobian(b, lay, vs, x0, threads=8)
    assert np.array_equal(r0, r0o) and np.array_equal(s, so)
    assert np.array_equal(J, Jo), np.argwhere(J != Jo)[:5]


def test_adjoint_jacobian_bitwise_objective_soft_failures():
    b, st, vs, x0, lay, db = setup(workloads.objective, 6)
    J, r0, s = to_np(*engine.adjoint_jacobian_device(db, lay, b, vs, x0))
    Jo, r0o, so = po.port().adjoint_jacobian(b, lay, vs, x0, threads=8)
    assert np.array_equal(r0, r0o) and np.array_equal(s, so)
    assert np.array_equal(J, Jo), np.argwhere(J != Jo)[:5]


def test_adjoint_fma_close_to_exact():
    b, st, vs, x0, lay, db = setup(workloads.singlet, 16, precision=PRECISION_FP64_FMA)
    J, r0, s = to_np(*engine.adjoint_jacobian_device(db, lay, b, vs, x0))
    Jo, r0o, so = po.port().adjoint_jacobian(b, lay, vs, x0, threads=8)
    scale = np.abs(Jo).max(axis=2, keepdims=True) + 1e-300
    assert np.max(np.abs(J - Jo) / scale) < 1e-10


def test_adjoint_matches_fd_to_truncation_error():
    b, st, vs, x0, lay, db = setup(workloads.singlet, 16)
    Ja, _, _ = to_np(*engine.adjoint_jacobian_device(db, lay, b, vs, x0))
    Jf, _, _ = to_np(*engine.fd_jacobian_device(db, lay, b, vs, x0))
    scale = np.abs(Jf).max(axis=2, keepdims=True)
    assert np.max(np.abs(Ja - Jf) / scale) < 1e-6


def test_normal_equations_exact_bitwise_and_dmma_close():
    b, st, vs, x0, lay, db = setup(workloads.objective, 3, rings=6, spokes=8)
    J, r0, s = engine.adjoint_jacobian_device(db, lay, b, vs, x0)
    g_exact, g_dmma = to_np(engine.normal_equations_device(J, r0, True),
                            engine.normal_equations_device(J, r0, False))
    Jn, r0n = to_np(J, r0)
    P = vs.size
    for i in range(3):
        A, g = po.port().normal_equations(Jn[i], r0n[i])
        assert np.array_equal(g_exact[i, :P, :P], A)
        assert np.array_equal(g_exact[i, :P, P], g)
        assert np.array_equal(g_exact[i], g_exact[i].T)
        M = np.concatenate([Jn[i], r0n[i][None, :]], axis=0)
        G = M @ M.T
        scale = np.sqrt(np.outer(np.diag(G), np.diag(G))) + 1e-300
        assert np.max(np.abs(g_dmma[i] - G) / scale) < 1e-12
        assert np.max(np.abs(g_exact[i] - G) / scale) < 1e-12


def gram_close(a, b, tol):
    """max |a - b| / sqrt(|b_ii b_jj|) <= tol, with the diagonal floored at 1e-20 max|diag|;
    reports the worst entry."""
    d = np.abs(np.diagonal(b, axis1=-2, axis2=-1))
    d = np.maximum(d, 1e-20 * d.max(axis=-1, keepdims=True) + 1e-300)
    scale = np.sqrt(d[..., :, None] * d[..., None, :])
    err = np.abs(a - b) / scale
    worst = np.unravel_index(np.argmax(err), err.shape)
    assert err.max() <= tol, (err.max(), worst, a[worst], b[worst])
    return True


def test_fused_adjoint_normal_equations_match_exact_on_singlets():
    """The fused kernel (tuple-centred rows, Chan merges, DMMA, FMA arithmetic) equals the exact
    materialised J^T J, J^T r and r^T r within rounding on well-conditioned systems."""
    b, st, vs, x0, lay, db = setup(workloads.singlet, 64)
    J, r0, s = engine.adjoint_jacobian_device(db, lay, b, vs, x0)
    ref = engine.normal_equations_device(J, r0, True)
    b2, st2, vs2, x02, lay2, db2 = setup(workloads.singlet, 64, precision=PRECISION_FP64_FMA)
    fused = engine.adjoint_normal_equations_device(db2, lay2, b2, vs2, x02)
    ref, fused = to_np(ref, fused)
    assert gram_close(fused, ref, 1e-9)


@pytest.mark.parametrize("kw", [{}, {"rings": 3, "spokes": 6}])
def test_fused_adjoint_normal_equations_exact_rows_match_exact_gram(kw):
    """Soft failures (objectives at NA 0.95): the fused kernel with exact-arithmetic rows
    against the exact materialised path -- the rows agree bit for bit, so the difference is
    only the summation order of the centred DMMA contraction."""
    b, st, vs, x0, lay, db = setup(workloads.objective, 6, **kw)
    J, r0, s = engine.adjoint_jacobian_device(db, lay, b, vs, x0)
    ref = engine.normal_equations_device(J, r0, True)
    fused = engine.adjoint_normal_equations_device(db, lay, b, vs, x0)
    ref, fused = to_np(ref, fused)
    assert gram_close(fused, ref, 1e-10)
