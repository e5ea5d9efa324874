"""Failure paths of the kernels' bounded waits, driven without a fault or a hang.

Every kernel stages its variant's record into shared memory with one bulk copy and waits on an
mbarrier for at most a fixed number of polls. When the wait gives up the block records
MKB_ERR_TIMEOUT in a device error word, drains the copy still in flight (with the full limit)
and returns without writing its outputs. mkb_set_wait_limit(0) makes every first wait give up
at once, so the give-up path runs deterministically while every copy still completes.

A record pointer that is not 16-byte aligned would make the bulk copy fault; the host rejects
it with MKB_ERR_ARGUMENT before anything is enqueued.
"""

import ctypes as C

import numpy as np
import pytest
import torch

from mikroptim_b200 import _capi, engine, workloads
from mikroptim_b200.batch import ResidualLayout

pytestmark = pytest.mark.gpu

SENTINEL = 7.25


def _residuals(db, lay, b, fill: float):
    lib = _capi.lib()
    V = db.variants
    res = torch.full((V, lay.trace_rows), fill, dtype=torch.float64, device=db.device)
    opd = torch.full((V, lay.rays_per_variant), fill, dtype=torch.float64, device=db.device)
    st = torch.full((V, lay.rays_per_variant), 99, dtype=torch.uint8, device=db.device)
    s, plan = db.c_struct(), lay.plan(b)
    rc = lib.mkb_residuals_device(C.byref(s), C.byref(plan), C.c_void_p(res.data_ptr()),
                                  lay.trace_rows, C.c_void_p(opd.data_ptr()),
                                  C.c_void_p(st.data_ptr()),
                                  C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return rc, res, opd, st


def test_wait_that_gives_up_records_timeout_and_writes_nothing():
    lib = _capi.lib()
    b, st, vs, x0 = workloads.singlet(64)
    lay = ResidualLayout(b.topology, st)
    db = engine.DeviceSystemBatch(b)
    torch.cuda.synchronize()
    assert lib.mkb_device_status() == _capi.MKB_OK  # nothing pending from earlier tests
    assert lib.mkb_set_wait_limit(0) == _capi.MKB_OK
    try:
        rc, res, opd, stt = _residuals(db, lay, b, SENTINEL)
        torch.cuda.synchronize()
    finally:
        assert lib.mkb_set_wait_limit(_capi.MKB_WAIT_POLLS_DEFAULT) == _capi.MKB_OK
    assert rc == _capi.MKB_OK  # the launch itself succeeded
    assert lib.mkb_device_status() == _capi.MKB_ERR_TIMEOUT
    assert "wait gave up" in lib.mkb_last_error().decode()
    # every block gave up before touching its outputs
    assert torch.all(res == SENTINEL) and torch.all(opd == SENTINEL) and torch.all(stt == 99)
    # the status word was cleared by the read; the next call runs normally and is correct
    assert lib.mkb_device_status() == _capi.MKB_OK
    rc, res, opd, stt = _residuals(db, lay, b, SENTINEL)
    torch.cuda.synchronize()
    assert rc == _capi.MKB_OK and lib.mkb_device_status() == _capi.MKB_OK
    ref = engine.residuals_device(db, lay, b)
    assert torch.equal(res, ref.residuals) and torch.equal(opd, ref.opd)
    assert torch.equal(stt, ref.status)


def test_fused_adjoint_wait_that_gives_up_records_timeout():
    """The persistent fused kernel: its blocks leave the run queue on a give-up."""
    lib = _capi.lib()
    b, st, vs, x0 = workloads.singlet(16)
    lay = ResidualLayout(b.topology, st)
    db = engine.DeviceSystemBatch(b)
    good = engine.adjoint_normal_equations_device(db, lay, b, vs, x0)
    torch.cuda.synchronize()
    assert lib.mkb_device_status() == _capi.MKB_OK
    assert lib.mkb_set_wait_limit(0) == _capi.MKB_OK
    try:
        engine.adjoint_normal_equations_device(db, lay, b, vs, x0)
        torch.cuda.synchronize()
    finally:
        assert lib.mkb_set_wait_limit(_capi.MKB_WAIT_POLLS_DEFAULT) == _capi.MKB_OK
    assert lib.mkb_device_status() == _capi.MKB_ERR_TIMEOUT
    again = engine.adjoint_normal_equations_device(db, lay, b, vs, x0)
    torch.cuda.synchronize()
    assert lib.mkb_device_status() == _capi.MKB_OK
    assert torch.equal(again, good)


def test_unaligned_records_rejected_before_any_launch():
    lib = _capi.lib()
    b, st, vs, x0 = workloads.singlet(4)
    lay = ResidualLayout(b.topology, st)
    db = engine.DeviceSystemBatch(b)
    s = db.c_struct()
    s.records = db.records.data_ptr() + 8  # inside the allocation, 8 B off
    plan = lay.plan(b)
    out = torch.full((4, lay.trace_rows), SENTINEL, dtype=torch.float64, device=db.device)
    opd = torch.empty((4, lay.rays_per_variant), dtype=torch.float64, device=db.device)
    stt = torch.empty((4, lay.rays_per_variant), dtype=torch.uint8, device=db.device)
    l0 = lib.mkb_launch_count()
    rc = lib.mkb_residuals_device(C.byref(s), C.byref(plan), C.c_void_p(out.data_ptr()),
                                  lay.trace_rows, C.c_void_p(opd.data_ptr()),
                                  C.c_void_p(stt.data_ptr()), None)
    assert rc == _capi.MKB_ERR_ARGUMENT
    assert "16-byte aligned" in lib.mkb_last_error().decode()
    assert lib.mkb_launch_count() == l0
    torch.cuda.synchronize()
    assert torch.all(out == SENTINEL)
    assert lib.mkb_device_status() == _capi.MKB_OK
