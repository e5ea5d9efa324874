"""Paraxial constraints evaluated on the device as the LM's extra rows (focal length, parfocal
length, working distance, paraxial focus, Petzval curvature).

* The rows and their central-difference Jacobian equal the reference's extra_rows_cpu with
  make_paraxial_residuals bit for bit (singlets; objectives with a Buchdahl glass variable,
  whose paraxial index follows the glass).
* The analytic adjoint Jacobian of the y-nu trace agrees with the central differences to the
  differences' own error.
* Ghost plates are thin elements of power -2 (n_G - n_m) t2 in the y-nu trace and the Petzval
  sum: the rows and the Jacobian's coefficient columns equal the reference's bit for bit too.
* LM trajectories with the constraints on the device equal the reference's optimize_lm_cpu
  with the same constraints bit for bit, with no host phase in the cycle: a cycle is one
  fixed launch sequence and replays from a CUDA graph.
"""

import copy

import numpy as np
import pytest
import torch

from conftest import has_reference_build
from mikroptim_b200 import engine, workloads
from mikroptim_b200.batch import ResidualLayout
import oracle.pyoracle as po

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_reference_build(), reason="reference build missing")]

SINGLET = [(0, 0, 4.0, 48.0), (2, 1, 1.0, 47.5), (4, 2, 1e4, 0.001), (3, 0, 0.5, 0.0),
           (1, 0, 0.25, 52.0)]
OBJECTIVE = [(0, 0, 2.0, 40.0), (2, 2, 1.0, 5.0), (4, 2, 1e3, 0.002), (3, 0, 1.0, 0.0)]


def _singlet(n=6):
    b, st, vs, x0 = workloads.singlet(n)
    return b, ResidualLayout(b.topology, st), vs, x0


def _objective(n=5):
    b, st, vs, x0 = workloads.objective(n, rings=3, spokes=6, glass=True)
    return b, ResidualLayout(b.topology, st), vs, x0


def _ghost(n=5):
    # coefficients ~ N(0, 2e-3) mm: the plate's power moves the rows well above rounding
    b, st, vs, x0 = workloads.ghost(n, rings=3, spokes=6, coeff_sigma=2e-3)
    return b, ResidualLayout(b.topology, st), vs, x0


CASES = [(_singlet, SINGLET), (_objective, OBJECTIVE), (_ghost, SINGLET)]


@pytest.mark.parametrize("make, cons", CASES)
def test_fd_rows_bitwise_equal_reference(make, cons):
    b, lay, vs, x0 = make()
    J, r = engine.paraxial_rows_device(engine.DeviceSystemBatch(b), lay, b, vs, x0,
                                       engine.ParaxialConstraints.of(cons))
    Jr, rr = po.reference().extra_rows(b, lay, vs, x0, cons)
    assert np.array_equal(r.cpu().numpy(), rr.reshape(r.shape))
    assert np.array_equal(J.cpu().numpy(), Jr.reshape(J.shape))


@pytest.mark.parametrize("make, cons", CASES)
def test_adjoint_rows_agree_with_central_differences(make, cons):
    b, lay, vs, x0 = make()
    db = engine.DeviceSystemBatch(b)
    Jf, rf = engine.paraxial_rows_device(db, lay, b, vs, x0, engine.ParaxialConstraints.of(cons))
    Ja, ra = engine.paraxial_rows_device(db, lay, b, vs, x0,
                                         engine.ParaxialConstraints.of(cons, derivative="adjoint"))
    Jf, Ja = Jf.cpu().numpy(), Ja.cpu().numpy()
    assert np.array_equal(rf.cpu().numpy(), ra.cpu().numpy())  # the same residuals
    # column-wise relative to the row's largest entry (central differences: O(h^2) ~ 1e-10)
    scale = np.maximum(np.abs(Jf).max(axis=1, keepdims=True), 1e-300)
    err = np.abs(Ja - Jf) / scale
    assert err.max() <= 1e-6, err.max()


def test_ghost_plates_change_the_rows():
    b, lay, vs, x0 = _ghost()
    cons = engine.ParaxialConstraints.of(SINGLET)
    _, r = engine.paraxial_rows_device(engine.DeviceSystemBatch(b), lay, b, vs, x0, cons)
    flat = copy.deepcopy(b)
    flat.ghost_coeff[:] = 0.0
    x_flat = np.stack([vs.extract(flat, v) for v in range(b.variants)])
    _, r0 = engine.paraxial_rows_device(engine.DeviceSystemBatch(flat), lay, flat, vs, x_flat,
                                        cons)
    # focal length, Petzval and paraxial focus follow the plate's power
    d = np.abs(r.cpu().numpy() - r0.cpu().numpy())
    assert d[:, [0, 3]].min() > 1e-6


def test_parfocal_reference_on_a_ghost_plate_is_refused():
    b, lay, vs, x0 = _ghost(2)
    cons = engine.ParaxialConstraints([engine.ParaxialConstraint(1, 0, 1.0, 50.0,
                                                                 reference_surface=3)])
    with pytest.raises(Exception, match="ghost plate"):
        engine.paraxial_rows_device(engine.DeviceSystemBatch(b), lay, b, vs, x0, cons)


@pytest.mark.parametrize("make", [_singlet, _ghost])
@pytest.mark.parametrize("method", ["adjoint", "fd"])
def test_lm_with_device_constraints_bitwise_equal_reference(method, make):
    b, lay, vs, x0 = make(4)
    cons = SINGLET[:3]
    opt = engine.LmOptions(max_iterations=8,
                           jacobian=engine.JACOBIAN_ADJOINT if method == "adjoint"
                           else engine.JACOBIAN_FD, gram_exact=True, fail_weight_factor=1.0,
                           paraxial=engine.ParaxialConstraints.of(cons))
    g = engine.optimize_lm_gpu(b, lay, vs, x0, opt)
    r = po.reference().optimize_lm(b, lay, vs, x0, max_iterations=8, method=method,
                                   penalty_rounds=1, threads=4, constraints=cons)
    for k in ("status", "iterations", "accepted", "x", "merit"):
        assert np.array_equal(g[k], r[k]), k
    assert np.array_equal(g["history"], r["history"], equal_nan=True)


def test_lm_with_device_constraints_replays_as_a_graph():
    b, lay, vs, x0 = _singlet(16)
    opt = engine.LmOptions(max_iterations=20, gram_exact=False, fail_weight_factor=1.0,
                           paraxial=engine.ParaxialConstraints.of(SINGLET[:3],
                                                                  derivative="adjoint"))
    db = engine.DeviceSystemBatch(b)
    direct = engine.DeviceLm(db, lay, b, vs, opt, 16)
    direct.start(x0)
    for _ in range(6):
        direct.cycle()
    graphed = engine.DeviceLm(db, lay, b, vs, opt, 16)
    graphed.start(x0)
    graphed.cycle()
    g = graphed.capture()
    for _ in range(5):
        g.replay()
    torch.cuda.synchronize()
    a, c = direct.results(), graphed.results()
    for k in ("x", "merit", "iterations", "status"):
        assert np.array_equal(a[k], c[k]), k
    # the constraints take part: a run optimised without them ends elsewhere
    plain = engine.optimize_lm_gpu(b, lay, vs, x0, engine.LmOptions(
        max_iterations=20, gram_exact=False, fail_weight_factor=1.0))
    assert not np.allclose(plain["x"], a["x"])
