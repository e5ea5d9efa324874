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


def test_usable_bytes_reserve():
    """usable = free - max(min, fraction * free), at least 0 (usable_bytes,
    batch_memory.hpp:125); a fraction outside [0, 1] is an argument error."""
    lib = _capi.lib()
    out = C.c_size_t(0)
    gib = 1 << 30
    assert lib.mkb_usable_bytes(10 * gib, 256 << 20, 0.05, C.byref(out)) == 0
    assert out.value == 10 * gib - int(0.05 * 10 * gib)
    assert lib.mkb_usable_bytes(gib, 256 << 20, 0.05, C.byref(out)) == 0
    assert out.value == gib - (256 << 20)
    assert lib.mkb_usable_bytes(100 << 20, 256 << 20, 0.05, C.byref(out)) == 0
    assert out.value == 0
    assert lib.mkb_usable_bytes(gib, 0, 1.5, C.byref(out)) == _capi.MKB_ERR_ARGUMENT


def _shape_and_plan(make=workloads.singlet):
    from mikroptim_b200.engine import TraceEngine
    b, st, vs, x0 = make(4)
    lay = ResidualLayout(b.topology, st)
    return b, lay, TraceEngine._shape(b.topology, False), lay.plan(b)


def test_trace_run_bytes_per_variant():
    lib = _capi.lib()
    b, lay, shape, plan = _shape_and_plan()
    per, fixed = C.c_size_t(0), C.c_size_t(0)
    rays, rows = lay.rays_per_variant, lay.trace_rows
    rec = 8 * shape.record_stride
    assert lib.mkb_trace_run_bytes(C.byref(shape), C.byref(plan), 0, 5, 1, 0, C.byref(per),
                                   C.byref(fixed)) == 0
    assert per.value == rec + 8 * (rows + 5) + rays + 8 * rays
    assert lib.mkb_trace_run_bytes(C.byref(shape), C.byref(plan), 0, 0, 0, 0, C.byref(per),
                                   C.byref(fixed)) == 0
    assert per.value == rec + 8 * rows + rays
    tuples = b.fields * b.wavelengths
    assert lib.mkb_trace_run_bytes(C.byref(shape), C.byref(plan), 1, 0, 0, 1, C.byref(per),
                                   C.byref(fixed)) == 0
    assert per.value == rec + 24 + int(lib.mkb_merit_workspace_bytes(1, C.byref(plan))) + 8
    assert per.value >= rec + 24 + 16 * tuples + 8
    assert lib.mkb_trace_run_bytes(C.byref(shape), C.byref(plan), 0, -1, 0, 0, C.byref(per),
                                   C.byref(fixed)) == _capi.MKB_ERR_ARGUMENT


def test_tranche_variants_fit_the_budget():
    """The tranche is the largest multiple of `granularity` whose buffers fit the usable bytes;
    0 when not even `granularity` variants fit."""
    lib = _capi.lib()
    b, lay, shape, plan = _shape_and_plan()
    per, fixed = C.c_size_t(0), C.c_size_t(0)
    lib.mkb_trace_run_bytes(C.byref(shape), C.byref(plan), 0, 0, 1, 0, C.byref(per),
                            C.byref(fixed))
    opts = _capi.TraceOptions()

    def tranche(usable, g=1):
        return lib.mkb_trace_tranche_variants(usable, C.byref(shape), C.byref(plan),
                                              C.byref(opts), 0, 0, 1, 0, g)
    assert tranche(fixed.value + 300 * per.value) == 300
    assert tranche(fixed.value + 300 * per.value - 1) == 299
    assert tranche(fixed.value + 300 * per.value, 7) == 294
    assert tranche(fixed.value + 6 * per.value, 7) == 0
    assert tranche(fixed.value) == 0
    assert 0 < tranche(1 << 50) <= (2**31 - 1)  # capped by the CTA count of one launch
    assert tranche(1 << 30, 0) == _capi.MKB_ERR_ARGUMENT
    opts.pack_rays = -1
    assert tranche(1 << 30) == _capi.MKB_ERR_ARGUMENT


def test_engine_settings_mirror_the_reference():
    from mikroptim_b200 import engine
    ts = engine.TraceSettings()
    assert (ts.opd, ts.status, ts.extra_residuals, ts.extrema, ts.pack_rays) == \
        (False, True, 0, False, 512)
    r = engine.MemoryReserve()
    assert (r.min_bytes, r.fraction) == (256 << 20, 0.05)
    assert engine.EngineOptions().memory_limit_bytes is None
