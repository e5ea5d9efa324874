"""An aperture stop inside the system (MKB_SURFACE_APERTURE_STOP), on the CPU: the packed
records carry the entrance pupil of paraxial ray aiming bit for bit as the oracle restates it,
a stop at the first vertex leaves the pupil as it is, and the checks refuse what is not built
(two stops, a stop at the last surfaces, thickness[0] as a variable, decentered systems)."""

import ctypes as C

import numpy as np
import pytest

from mikroptim_b200 import _capi, workloads
from mikroptim_b200.batch import (BatchTopology, SURFACE_APERTURE_STOP, SURFACE_SPHERE,
                                  SURFACE_STOP, VAR_THICKNESS, Variable, VariableSet)
from mikroptim_b200.quadrature import PUPIL_FULL
import oracle.pyoracle as po


def _packed(batch):
    lib = _capi.lib()
    view = batch.view()
    stride = lib.mkb_record_stride_ext(batch.surfaces, batch.wavelengths, batch.fields,
                                       0, 0, 0, int(batch.buchdahl_coeff is not None))
    rec = np.zeros((batch.variants, stride))
    rc = lib.mkb_pack_batch_host(C.byref(view), rec.ctypes.data_as(C.POINTER(C.c_double)))
    return rc, rec


def _layout(batch):
    S, L, F = batch.surfaces, batch.wavelengths, batch.fields
    pupil = 2 * S + S * L
    return pupil


@pytest.mark.parametrize("make,stop", [(lambda: workloads.objective(6, rings=4, spokes=8), 8),
                                       (lambda: workloads.objective(6, rings=4, spokes=8), 3),
                                       (lambda: workloads.singlet(5), 2)])
def test_packed_pupil_equals_the_oracle_aiming(make, stop):
    b, st, vs, _ = make()
    ab, _, avs, ax0 = workloads.with_aperture_stop(b, st, vs, stop)
    assert ab.type[stop] == SURFACE_APERTURE_STOP and ab.topology.stop_surface == stop
    assert all(not (v.type == VAR_THICKNESS and v.surface == 0) for v in avs.variables)
    rc, rec = _packed(ab)
    assert rc == 0, _capi.lib().mkb_last_error()
    a, t0 = po.port().aim(ab)
    pupil = _layout(ab)
    assert np.array_equal(rec[:, pupil], a)
    assert np.array_equal(rec[:, ab.surfaces], t0)  # thickness[0]
    # the stop's semi-aperture was chosen for the old pupil radius
    assert np.allclose(a, b.pupil_radius, rtol=1e-12)


def test_stop_at_the_first_vertex_keeps_the_pupil():
    b, st, vs, _ = workloads.singlet(4)
    ab, _, _, _ = workloads.with_aperture_stop(b, st, vs, 1)
    rc, rec = _packed(ab)
    assert rc == 0
    assert np.array_equal(rec[:, _layout(ab)], ab.curvature[:, 1])  # R / |1|
    assert np.all(rec[:, ab.surfaces] == 0.0)  # -0 / 1


def _topo(kinds, **kw):
    return BatchTopology(surfaces=len(kinds), wavelengths=1, fields=1, type=kinds,
                         pupil_mode=[PUPIL_FULL], **kw)


@pytest.mark.parametrize("kinds", [
    [SURFACE_STOP, SURFACE_APERTURE_STOP, SURFACE_SPHERE, SURFACE_APERTURE_STOP, SURFACE_SPHERE],
    [SURFACE_STOP, SURFACE_SPHERE, SURFACE_SPHERE, SURFACE_APERTURE_STOP]])
def test_topology_refuses_misplaced_stops(kinds):
    with pytest.raises(ValueError):
        _topo(kinds).validate()


def test_decentered_systems_with_an_interior_stop_are_refused():
    with pytest.raises(NotImplementedError):
        _topo([SURFACE_STOP, SURFACE_SPHERE, SURFACE_APERTURE_STOP, SURFACE_SPHERE],
              non_coaxial=True).validate()


def test_thickness0_is_no_variable_with_an_interior_stop():
    topo = _topo([SURFACE_STOP, SURFACE_SPHERE, SURFACE_APERTURE_STOP, SURFACE_SPHERE])
    with pytest.raises(ValueError):
        VariableSet(topo, [Variable(VAR_THICKNESS, 0, 0.0, 10.0, 1.0)])
    VariableSet(topo, [Variable(VAR_THICKNESS, 1, 0.0, 10.0, 1.0)])  # the others are fine


def test_pack_refuses_a_stop_imaged_at_infinity():
    b, st, vs, _ = workloads.singlet(2)
    ab, _, _, _ = workloads.with_aperture_stop(b, st, vs, 2)
    assert _packed(ab)[0] == 0
    # the first surface focuses the ray (y = 1, u = 0) exactly onto the stop: y_A = 0
    # (n' = 2, c = 0.5: u' = -0.25; t = 4: y = 1 - 1)
    ab.index[0, 1, 0] = 2.0
    ab.curvature[0, 1] = 0.5
    ab.thickness[0, 1] = 4.0
    rc, _ = _packed(ab)
    assert rc == _capi.MKB_ERR_ARGUMENT
    assert b"infinity" in _capi.lib().mkb_last_error()
