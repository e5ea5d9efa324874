"""GPU test of the MERIT entry point that allocates nothing (mkb_merit_noalloc_device).

It exists for callers that may not call cudaMalloc -- a host that owns all device memory,
or a loop that must not wait on an allocation -- and keeps its partial sums in an array
inside the library. Through the C ABI, two calls in a row must give exactly what the
workspace entry point (mkb_merit_device) gives; a batch beyond the built-in limit must be
rejected before any work. The file is named so that pytest collects it last.
"""

import ctypes as C

import numpy as np
import pytest
import torch

from mikroptim_b200 import _capi, engine, workloads
from mikroptim_b200.batch import (PRECISION_FP64, PRECISION_FP64_FMA, PRECISION_MIXED,
                                  ResidualLayout)

pytestmark = pytest.mark.gpu

MAX_SLOTS = 262144  # MKB_NOALLOC_MERIT_MAX_SLOTS


def outputs(V, dev):
    return (torch.empty(V, dtype=torch.float64, device=dev),
            torch.empty(V, dtype=torch.int64, device=dev),
            torch.empty(V, dtype=torch.int64, device=dev))


def with_workspace(db, plan, dev):
    lib = _capi.lib()
    m, f, h = outputs(db.variants, dev)
    ws = torch.empty(int(lib.mkb_merit_workspace_bytes(db.variants, C.byref(plan))),
                     dtype=torch.uint8, device=dev)
    b = db.c_struct()
    rc = lib.mkb_merit_device(C.byref(b), C.byref(plan), C.c_void_p(m.data_ptr()),
                              C.c_void_p(f.data_ptr()), C.c_void_p(h.data_ptr()),
                              C.c_void_p(ws.data_ptr()), ws.numel(),
                              C.c_void_p(torch.cuda.current_stream().cuda_stream))
    _capi.check(rc, "mkb_merit_device")
    torch.cuda.synchronize()
    return m.cpu().numpy(), f.cpu().numpy(), h.cpu().numpy()


def without_allocation(db, plan, dev):
    lib = _capi.lib()
    m, f, h = outputs(db.variants, dev)
    b = db.c_struct()
    rc = lib.mkb_merit_noalloc_device(C.byref(b), C.byref(plan), C.c_void_p(m.data_ptr()),
                                      C.c_void_p(f.data_ptr()), C.c_void_p(h.data_ptr()),
                                      C.c_void_p(torch.cuda.current_stream().cuda_stream))
    _capi.check(rc, "mkb_merit_noalloc_device")
    torch.cuda.synchronize()
    return m.cpu().numpy(), f.cpu().numpy(), h.cpu().numpy()


@pytest.mark.parametrize("precision", [PRECISION_FP64, PRECISION_FP64_FMA, PRECISION_MIXED])
def test_no_alloc_merit_matches_workspace_entry_point_twice(precision):
    dev = torch.device("cuda", 0)
    for b, st, vs, x0 in (workloads.singlet(1024), workloads.objective(96)):
        st.precision = precision
        lay = ResidualLayout(b.topology, st)
        plan = lay.plan(b)
        db = engine.DeviceSystemBatch(b, dev)
        ref = with_workspace(db, plan, dev)
        first = without_allocation(db, plan, dev)
        second = without_allocation(db, plan, dev)
        for got in (first, second):
            for x, y in zip(got, ref):
                # the same kernels with the same inputs: equal bit for bit (stricter than the
                # 1e-13 relative bound the other merit tests use)
                assert np.array_equal(x, y)
    assert _capi.lib().mkb_device_status() == 0


def test_no_alloc_merit_rejects_batches_beyond_the_limit():
    dev = torch.device("cuda", 0)
    b, st, vs, x0 = workloads.singlet(4)
    lay = ResidualLayout(b.topology, st)
    plan = lay.plan(b)
    db = engine.DeviceSystemBatch(b, dev)
    s = db.c_struct()
    tuples = b.fields * b.wavelengths
    s.variants = MAX_SLOTS // tuples + 1  # never traced: the size check fails first
    m = torch.empty(4, dtype=torch.float64, device=dev)
    rc = _capi.lib().mkb_merit_noalloc_device(C.byref(s), C.byref(plan),
                                              C.c_void_p(m.data_ptr()),
                                              C.c_void_p(m.data_ptr()),
                                              C.c_void_p(m.data_ptr()), None)
    assert rc == _capi.MKB_ERR_ARGUMENT
    assert "limit" in _capi.lib().mkb_last_error().decode()


def test_no_alloc_merit_rejects_null_outputs_before_any_work():
    dev = torch.device("cuda", 0)
    b, st, vs, x0 = workloads.singlet(4)
    lay = ResidualLayout(b.topology, st)
    plan = lay.plan(b)
    db = engine.DeviceSystemBatch(b, dev)
    s = db.c_struct()
    m = torch.full((4,), -1.0, dtype=torch.float64, device=dev)
    f = torch.full((4,), -1, dtype=torch.int64, device=dev)
    lib = _capi.lib()
    for ptrs in ((None, f.data_ptr(), f.data_ptr()), (m.data_ptr(), None, f.data_ptr()),
                 (m.data_ptr(), f.data_ptr(), None)):
        rc = lib.mkb_merit_noalloc_device(C.byref(s), C.byref(plan),
                                          *[C.c_void_p(p) if p else None for p in ptrs], None)
        assert rc == _capi.MKB_ERR_ARGUMENT
        assert "null" in lib.mkb_last_error().decode()
    torch.cuda.synchronize()
    assert torch.all(m == -1.0) and torch.all(f == -1)
