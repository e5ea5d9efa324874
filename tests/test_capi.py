"""CPU tests of the C-ABI library: it loads without a GPU, exports every function that
include/mikroptim_b200.h declares, and rejects bad arguments on the host before any device
work (the reference throws std::invalid_argument before a launch)."""

import ctypes as C
import os
import re

import numpy as np
import pytest

from mikroptim_b200 import _capi, workloads
from mikroptim_b200.batch import ResidualLayout

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                      "mikroptim_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mkb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _capi.lib()
    names = declared_functions()
    assert len(names) >= 10
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_record_stride_and_pack():
    lib = _capi.lib()
    b, st, vs, x0 = workloads.singlet(4)
    stride = lib.mkb_record_stride(3, 3, 3)
    assert stride % 2 == 0 and stride >= 2 * 3 + 9 + 1 + 9
    rec = np.zeros((4, stride))
    view = b.view()
    assert lib.mkb_pack_batch_host(C.byref(view), _capi.ptr(rec)) == 0
    assert np.array_equal(rec[:, 0:3], b.curvature)
    assert np.array_equal(rec[:, 3:6], b.thickness)
    assert np.array_equal(rec[:, 6:15], b.index.reshape(4, 9))
    assert np.array_equal(rec[:, 15], b.pupil_radius)
    assert np.array_equal(rec[:, 16:19], np.sin(b.field_angle))
    assert np.array_equal(rec[:, 19:22], np.cos(b.field_angle))
    assert np.array_equal(rec[:, 22:25], b.field_target)


def test_rays_and_rows_match_layout():
    lib = _capi.lib()
    for make in (workloads.singlet, workloads.objective):
        b, st, vs, x0 = make(2)
        lay = ResidualLayout(b.topology, st)
        plan = lay.plan(b)
        assert lib.mkb_rays_per_variant(C.byref(plan)) == lay.rays_per_variant
        assert lib.mkb_trace_rows(C.byref(plan)) == lay.trace_rows


def _bad_call(mutate):
    lib = _capi.lib()
    b, st, vs, x0 = workloads.singlet(2)
    lay = ResidualLayout(b.topology, st)
    plan = lay.plan(b)
    db = _capi.DeviceBatch()
    db.variants, db.surfaces, db.wavelengths, db.fields = 2, 3, 3, 3
    db.record_stride = lib.mkb_record_stride(3, 3, 3)
    db.records = C.c_void_p(0x10000)  # never dereferenced: the checks fail first
    types = np.array([0, 2, 2], dtype=np.uint8)
    db.type = _capi.ptr(types, C.c_uint8)
    mutate(db, plan, types)
    rc = lib.mkb_residuals_device(C.byref(db), C.byref(plan), C.c_void_p(0x10000),
                                  lay.trace_rows, None, None, None)
    return rc, lib.mkb_last_error().decode()


@pytest.mark.parametrize("mutate,expect", [
    (lambda b, p, t: setattr(p, "rings", 0), "rings"),
    (lambda b, p, t: setattr(p, "rings", 33), "rings"),
    (lambda b, p, t: setattr(p, "spokes", 0), "spokes"),
    (lambda b, p, t: setattr(p, "failure", 7), "failure"),
    (lambda b, p, t: setattr(p, "fail_weight", -1.0), "fail_weight"),
    (lambda b, p, t: setattr(b, "surfaces", 1), "surfaces"),
    (lambda b, p, t: setattr(b, "record_stride", 3), "record_stride"),
    (lambda b, p, t: setattr(b, "records", C.c_void_p(0x10008)), "aligned"),
    (lambda b, p, t: t.__setitem__(0, 2), "stop"),
    (lambda b, p, t: setattr(b, "fields", 2), "match"),
])
def test_bad_arguments_rejected_before_launch(mutate, expect):
    rc, msg = _bad_call(mutate)
    assert rc == _capi.MKB_ERR_ARGUMENT
    assert expect in msg


def test_ghost_plate_surface_without_plate_data_rejected():
    """A GhostPlate surface needs the batch to carry as many plates (ghost_plates) as the
    table has such surfaces."""
    rc, msg = _bad_call(lambda b, p, t: t.__setitem__(1, 3))
    assert rc == _capi.MKB_ERR_ARGUMENT and "ghost" in msg


def test_merit_workspace_checked():
    lib = _capi.lib()
    b, st, vs, x0 = workloads.singlet(2)
    lay = ResidualLayout(b.topology, st)
    plan = lay.plan(b)
    need = lib.mkb_merit_workspace_bytes(2, C.byref(plan))
    assert need >= 2 * 9 * 16
