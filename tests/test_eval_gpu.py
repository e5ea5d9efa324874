"""Mode EVAL on the dense pupil grid (TraceEngine::evaluate): OPD maps after the piston, spot
diagrams (image-plane intercepts relative to the ideal image point), statuses and the four
field rays per tuple, equal to the reference's eval_cpu bit for bit -- for the three reference
spheres (through the paraxial exit pupil, through the vertex of the last surface, infinite
radius), full and half pupils, singlets, objectives (with failed rays), ghost plates and
decentered systems.
"""

import numpy as np
import pytest

from conftest import has_reference_build
from mikroptim_b200 import engine, workloads
from mikroptim_b200.batch import ResidualLayout
import oracle.pyoracle as po

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_reference_build(), reason="reference build missing")]

KEYS = ("opd", "spot_x", "spot_y", "status", "field_rays", "field_status")


def _check(b, st, settings):
    lay = ResidualLayout(b.topology, st)
    got = engine.TraceEngine(0).evaluate(b, settings)
    want = po.reference().eval(b, lay, settings.grid, settings.half_pupil, settings.reference,
                               settings.field_ray_offset)
    for k in KEYS:
        assert np.array_equal(getattr(got, k), want[k], equal_nan=True), k
    kappa = np.asarray(got.reference_curvature)
    assert np.array_equal(kappa, want["kappa"], equal_nan=True)
    assert np.array_equal(got.exit_pupil_position, want["exit_pupil"], equal_nan=True)
    return got


@pytest.mark.parametrize("reference", [engine.EVAL_EXIT_PUPIL, engine.EVAL_VERTEX,
                                       engine.EVAL_INFINITE])
@pytest.mark.parametrize("half", [False, True])
def test_eval_singlets_bitwise_equal_reference(reference, half):
    b, st, _, _ = workloads.singlet(12)
    got = _check(b, st, engine.EvalSettings(grid=33, half_pupil=half, reference=reference))
    assert np.isfinite(got.opd).all()


def test_eval_objectives_with_failed_rays_bitwise_equal_reference():
    b, st, _, _ = workloads.objective(6, rings=3, spokes=6)
    got = _check(b, st, engine.EvalSettings(grid=48))
    assert (got.status != 0).any() and (got.status == 0).any()


def test_eval_ghost_plates_and_decentered_bitwise_equal_reference():
    b, st, _, _ = workloads.ghost(5)
    _check(b, st, engine.EvalSettings(grid=24, reference=engine.EVAL_VERTEX))
    # the exit pupil of systems with ghost plates: the plates' paraxial power in the chief ray
    _check(b, st, engine.EvalSettings(grid=24, reference=engine.EVAL_EXIT_PUPIL))
    strong, st2, _, _ = workloads.ghost(5, coeff_sigma=2e-2)
    _check(strong, st2, engine.EvalSettings(grid=24, reference=engine.EVAL_EXIT_PUPIL))
    b, st, _, _ = workloads.tolerancing(4, elements=3, rings=4, spokes=8)
    _check(b, st, engine.EvalSettings(grid=24))


def test_eval_contracted_close_to_exact():
    """EVAL in FP64 with contraction (the forward of the MIXED mode): the same statuses, and
    intercepts and OPD within 1e-9 mm of the bit-exact evaluation on the objectives."""
    b, st, _, _ = workloads.objective(6, rings=3, spokes=6)
    db = engine.DeviceSystemBatch(b)
    ex = engine.evaluate_device(db, b, engine.EvalSettings(grid=40))
    fm = engine.evaluate_device(db, b, engine.EvalSettings(grid=40, precision=2))
    assert np.array_equal(ex.status, fm.status)
    ok = ex.status == 0
    assert np.abs(fm.spot_x[ok] - ex.spot_x[ok]).max() <= 1e-9
    assert np.abs(fm.spot_y[ok] - ex.spot_y[ok]).max() <= 1e-9
    assert np.nanmax(np.abs(fm.opd - ex.opd)) <= 1e-9
