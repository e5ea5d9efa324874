"""CPU tests: the oracle is pinned to the reference before anything is checked against it.

* the host quadrature equals the reference's generated Gauss-Legendre table bit for bit;
* the C restatement (liboracle.so) reproduces the golden fixtures, which were produced by the
  reference's own CPU code (tests/golden/make_golden.py), bit for bit;
* where the reference build is present, restatement and reference agree bit for bit on more
  variants, including every soft- and hard-failure branch;
* the adjoint Jacobian of the oracle agrees with its central finite differences.
"""

import json
import os

import numpy as np
import pytest

from conftest import has_reference_build
from mikroptim_b200 import workloads
from mikroptim_b200.batch import (ResidualLayout, STATUS_BACKWARD, STATUS_MISSED,
                                  STATUS_SOFT_MISSED, STATUS_SOFT_TIR)
from mikroptim_b200.quadrature import gauss_legendre_unit
import oracle.pyoracle as po

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def test_gauss_legendre_table_matches_reference():
    table = json.load(open(os.path.join(GOLDEN, "gauss_legendre.json")))["orders"]
    for n in range(1, 17):
        u, w = gauss_legendre_unit(n)
        assert list(u) == [float(x) for x in table[str(n)]["u"]], n
        assert list(w) == [float(x) for x in table[str(n)]["w"]], n


@pytest.mark.parametrize("n", [17, 24, 32])
def test_gauss_legendre_beyond_reference_is_exact_on_polynomials(n):
    u, w = gauss_legendre_unit(n)
    u, w = np.array(u), np.array(w)
    assert abs(w.sum() - 1) < 1e-15
    for k in range(2 * n):  # exact for degree <= 2n - 1
        assert abs((w * u ** k).sum() - 1.0 / (k + 1)) < 1e-14


def test_generator_reproduces_golden_inputs():
    g = load("singlet.npz")
    b, st, vs, x0 = workloads.singlet(1024)
    b = b.subset(0, 8)
    for name in ("curvature", "thickness", "index", "pupil_radius", "field_angle",
                 "field_target"):
        assert np.array_equal(getattr(b, name), g[name]), name
    assert np.array_equal(x0[:8], g["x0"])
    g = load("objective.npz")
    b, st, vs, x0 = workloads.objective(4096, rings=3, spokes=6)
    assert np.array_equal(b.subset(0, 2).curvature, g["curvature"])
    assert np.array_equal(b.subset(0, 2).thickness, g["thickness"])
    assert np.array_equal(b.subset(0, 2).index, g["index"])


def test_port_matches_golden_singlet_bitwise():
    g = load("singlet.npz")
    b, st, vs, x0 = workloads.singlet(1024)
    b = b.subset(0, 8)
    lay = ResidualLayout(b.topology, st)
    P = po.port()
    res, opd, status = P.residuals(b, lay)
    assert np.array_equal(res, g["residuals"])
    assert np.array_equal(opd, g["opd"])
    assert np.array_equal(status, g["status"])
    merit, failed, hard = P.merit(b, lay, threads=2)
    assert np.array_equal(merit, g["merit"])
    assert np.array_equal(failed, g["failed"]) and np.array_equal(hard, g["hard_failed"])
    J, r0, ch = P.fd_jacobian(b.subset(0, 2), lay, vs, x0[:2])
    assert np.array_equal(J, g["fd_jacobian"]) and np.array_equal(r0, g["fd_r0"])
    assert np.array_equal(ch, g["fd_changes"])
    J, r0, _ = P.adjoint_jacobian(b.subset(0, 2), lay, vs, x0[:2])
    assert np.array_equal(J, g["adjoint_jacobian"]) and np.array_equal(r0, g["adjoint_r0"])


def test_port_matches_golden_objective_bitwise():
    g = load("objective.npz")
    b, st, vs, x0 = workloads.objective(4096, rings=3, spokes=6)
    b = b.subset(0, 2)
    lay = ResidualLayout(b.topology, st)
    P = po.port()
    res, opd, status = P.residuals(b, lay)
    assert np.array_equal(res, g["residuals"]) and np.array_equal(status, g["status"])
    merit, failed, hard = P.merit(b, lay)
    assert np.array_equal(merit, g["merit"])
    one = b.subset(0, 1)
    J, r0, _ = P.adjoint_jacobian(one, lay, vs, x0[:1])
    assert np.array_equal(J, g["adjoint_jacobian"]) and np.array_equal(r0, g["adjoint_r0"])
    J, r0, ch = P.fd_jacobian(one, lay, vs, x0[:1])
    assert np.array_equal(J, g["fd_jacobian"]) and np.array_equal(ch, g["fd_changes"])


@pytest.mark.skipif(not has_reference_build(), reason="reference build not present")
def test_port_matches_reference_on_failure_branches():
    """64 objectives at the full 16 x 32 quadrature hit every soft and hard branch."""
    b, st, vs, x0 = workloads.objective(64)
    lay = ResidualLayout(b.topology, st)
    rp = po.port().residuals(b, lay, threads=8)
    rr = po.reference().residuals(b, lay, threads=8)
    for a, c in zip(rp, rr):
        assert np.array_equal(a, c)
    counts = np.bincount(rr[2].ravel(), minlength=7)
    for s in (STATUS_MISSED, STATUS_BACKWARD, STATUS_SOFT_MISSED, STATUS_SOFT_TIR):
        assert counts[s] > 0, s
    one = b.subset(3, 1)
    Jp = po.port().adjoint_jacobian(one, lay, vs, x0[3:4])
    Jr = po.reference().adjoint_jacobian(one, lay, vs, x0[3:4])
    assert np.array_equal(Jp[0], Jr[0]) and np.array_equal(Jp[1], Jr[1])


@pytest.mark.skipif(not has_reference_build(), reason="reference build not present")
def test_port_matches_reference_hard_mode():
    b, st, vs, x0 = workloads.singlet(1024)
    st.failure = 1  # hard
    b = b.subset(100, 32)
    lay = ResidualLayout(b.topology, st)
    for a, c in zip(po.port().residuals(b, lay), po.reference().residuals(b, lay)):
        assert np.array_equal(a, c)


def test_adjoint_matches_central_differences():
    """Criterion of the reference (tests/test_adjoint_jacobian.cpp:675): the adjoint and FD
    Jacobians agree to the FD truncation error on a smooth, failure-free case."""
    b, st, vs, x0 = workloads.singlet(16)
    lay = ResidualLayout(b.topology, st)
    P = po.port()
    Ja, r0a, _ = P.adjoint_jacobian(b.subset(0, 4), lay, vs, x0[:4])
    Jf, r0f, _ = P.fd_jacobian(b.subset(0, 4), lay, vs, x0[:4])
    assert np.array_equal(r0a, r0f)
    scale = np.abs(Jf).max(axis=2, keepdims=True)
    assert np.max(np.abs(Ja - Jf) / scale) < 1e-6


def test_normal_equations_fma_chain():
    rng = np.random.default_rng(5)
    J = rng.standard_normal((6, 40))
    r = rng.standard_normal(40)
    A, g = po.port().normal_equations(J, r)
    assert np.allclose(A, J @ J.T, rtol=1e-14, atol=1e-13)
    assert np.allclose(g, J @ r, rtol=1e-14, atol=1e-13)
    if has_reference_build():
        Ar, gr = po.reference().normal_equations(J, r)
        assert np.array_equal(A, Ar) and np.array_equal(g, gr)


@pytest.mark.skipif(not has_reference_build(), reason="reference CPU build not present")
def test_port_matches_reference_on_decentered_tilted_batch():
    """Non-coaxial batch (configuration-5 shape, small pupil): restatement and reference
    agree bit for bit on RESIDUALS, MERIT, the adjoint and the FD Jacobian."""
    b, st, vs, x0 = workloads.tolerancing(6, rings=6, spokes=12)
    assert np.any(b.decenter_tilt[:, 1:] != 0.0)
    lay = ResidualLayout(b.topology, st)
    P, R = po.port(), po.reference()
    for a, c in zip(P.residuals(b, lay), R.residuals(b, lay)):
        assert np.array_equal(a, c)
    for a, c in zip(P.merit(b, lay), R.merit(b, lay)):
        assert np.array_equal(a, c)
    two = b.subset(0, 2)
    for a, c in zip(P.adjoint_jacobian(two, lay, vs, x0[:2]),
                    R.adjoint_jacobian(two, lay, vs, x0[:2])):
        assert np.array_equal(a, c)
    for a, c in zip(P.fd_jacobian(two, lay, vs, x0[:2]), R.fd_jacobian(two, lay, vs, x0[:2])):
        assert np.array_equal(a, c)


def test_zero_transforms_trace_like_the_coaxial_batch():
    """A non-coaxial copy whose decenters and tilts are all zero traces bit for bit like the
    coaxial batch (surface_transform_of returns false for all-zero surfaces)."""
    from mikroptim_b200.batch import BatchTopology, SystemBatchHost, make_non_coaxial
    b, st, vs, x0 = workloads.tolerancing(3, rings=4, spokes=8)
    nc = b.subset(0, 3)
    nc.decenter_tilt[:] = 0.0
    t = b.topology
    co = SystemBatchHost(BatchTopology(t.surfaces, t.wavelengths, t.fields, list(t.type),
                                       list(t.pupil_mode)), 3)
    for name in ("curvature", "thickness", "index", "pupil_radius", "field_angle",
                 "field_target"):
        setattr(co, name, getattr(nc, name).copy())
    co.reference_wavelength_nm = nc.reference_wavelength_nm
    co.wavelength_weight, co.field_weight = nc.wavelength_weight, nc.field_weight
    assert make_non_coaxial(co).non_coaxial
    lay = ResidualLayout(b.topology, st)
    P = po.port()
    for a, c in zip(P.residuals(nc, lay), P.residuals(co, lay)):
        assert np.array_equal(a, c)


@pytest.mark.skipif(not has_reference_build(), reason="reference CPU build not present")
def test_port_matches_reference_with_ghost_plates():
    """Ghost plates with non-zero Legendre profiles (trace/ghost_plate.hpp): restatement and
    reference agree bit for bit on RESIDUALS, MERIT and the adjoint and FD Jacobians, whose
    columns include the plate's profile coefficients (GhostCoefficient variables)."""
    b, st, vs, x0 = workloads.ghost(8)
    assert np.any(b.ghost_coeff != 0.0)
    lay = ResidualLayout(b.topology, st)
    P, R = po.port(), po.reference()
    for a, c in zip(P.residuals(b, lay), R.residuals(b, lay)):
        assert np.array_equal(a, c)
    for a, c in zip(P.merit(b, lay), R.merit(b, lay)):
        assert np.array_equal(a, c)
    two = b.subset(0, 2)
    for a, c in zip(P.adjoint_jacobian(two, lay, vs, x0[:2]),
                    R.adjoint_jacobian(two, lay, vs, x0[:2])):
        assert np.array_equal(a, c)
    for a, c in zip(P.fd_jacobian(two, lay, vs, x0[:2]), R.fd_jacobian(two, lay, vs, x0[:2])):
        assert np.array_equal(a, c)


def test_port_adjoint_through_ghost_plates_matches_central_differences():
    """The restated reverse step of a ghost plate (ghost_step_backward): derivatives with
    respect to curvatures, thicknesses and the plate's profile coefficients agree with central
    differences of the pinned forward trace to 1e-6 of the column (steps 1e-5, thicknesses
    1e-4, where the OPL rounding of a smaller step dominates)."""
    b, st, vs, x0 = workloads.ghost(2)
    lay = ResidualLayout(b.topology, st)
    P = po.port()
    J, _, _ = P.adjoint_jacobian(b.subset(0, 1), lay, vs, x0[:1])
    for k in range(vs.size):
        h = 1e-4 if 4 <= k <= 6 else 1e-5
        bp, bm = b.subset(0, 1), b.subset(0, 1)
        xp, xm = x0[0].copy(), x0[0].copy()
        xp[k] += h
        xm[k] -= h
        vs.apply(bp, 0, xp)
        vs.apply(bm, 0, xm)
        fd = (P.residuals(bp, lay)[0][0] - P.residuals(bm, lay)[0][0]) / (2 * h)
        assert np.abs(J[0, k] - fd).max() <= 1e-6 * np.abs(fd).max(), k


def test_subset_owns_its_arrays():
    b, st, vs, x0 = workloads.ghost(3)
    sub = b.subset(0, 2)
    sub.curvature[0, 1] += 1.0
    sub.ghost_coeff[0, 0, 0] += 1.0
    assert b.curvature[0, 1] != sub.curvature[0, 1]
    assert b.ghost_coeff[0, 0, 0] != sub.ghost_coeff[0, 0, 0]


@pytest.mark.skipif(not has_reference_build(), reason="reference CPU build not present")
def test_port_matches_reference_with_glass_variables():
    """Glass variables (Buchdahl n0, nu1, nu2 of the medium after a surface; the reference's
    VariableType::Glass): applying x recomputes that medium's index at every wavelength, and the
    adjoint carries each medium's index adjoint into its glass columns with (1, w, w^2).
    Restatement and reference agree bit for bit on the adjoint and the FD Jacobians."""
    b, st, vs, x0 = workloads.objective(4, rings=3, spokes=6, glass=True)
    assert vs.size == 32
    lay = ResidualLayout(b.topology, st)
    P, R = po.port(), po.reference()
    two = b.subset(0, 2)
    for a, c in zip(P.adjoint_jacobian(two, lay, vs, x0[:2]),
                    R.adjoint_jacobian(two, lay, vs, x0[:2])):
        assert np.array_equal(a, c)
    for a, c in zip(P.fd_jacobian(two, lay, vs, x0[:2]), R.fd_jacobian(two, lay, vs, x0[:2])):
        assert np.array_equal(a, c)


@pytest.mark.skipif(not has_reference_build(), reason="reference CPU build not present")
def test_extra_rows_host_match_reference():
    """Extra residual rows (paraxial constraints evaluated by the reference's own
    paraxial_residuals): the host layer's central-difference rows, pattern and formula from the
    library's host entry points, equal the reference's extra_rows_cpu bit for bit."""
    from mikroptim_b200 import engine
    b, st, vs, x0 = workloads.singlet(3)
    lay = ResidualLayout(b.topology, st)
    R = po.reference()
    cons = [(0, 0, 4.0, 48.0), (2, 1, 1.0, 47.5), (4, 2, 1e4, 0.001)]
    extra = engine.ExtraResiduals(
        len(cons), lambda one, v, out: out.__setitem__(
            slice(None), R.paraxial_residuals(one, lay, v, cons)))
    J, r = engine.extra_rows_host(b, vs, x0[:3], extra)
    Jr, rr = R.extra_rows(b, lay, vs, x0[:3], cons)
    assert np.array_equal(r, rr) and np.array_equal(J, Jr)
    assert np.any(J != 0.0)
