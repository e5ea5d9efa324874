"""Device-side engine mirroring the reference's CUDA host API.

  DeviceSystemBatch  include/mikroptim/cuda/device_system_batch.hpp (upload of a batch)
  TraceEngine        include/mikroptim/cuda/trace_engine.hpp (run RESIDUALS / MERIT)
  TraceMode          trace_engine.hpp:31

PyTorch only provides device memory and streams here; every computation is a kernel of
libmikroptim_b200.so called through its C ABI. There is no CPU fallback: without a CUDA device
or without the built library the calls raise.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
import enum

import numpy as np
import torch

from . import _capi
from .batch import ResidualLayout, ResidualSettings, SystemBatchHost


class TraceMode(enum.Enum):
    RESIDUALS = "RESIDUALS"
    MERIT = "MERIT"


def _stream_handle(stream: torch.cuda.Stream | None) -> C.c_void_p:
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _require_cuda(device) -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("mikroptim_b200: no CUDA device (there is no CPU fallback)")
    _capi.lib()
    return torch.device(device)


class DeviceSystemBatch:
    """A batch resident in device memory as packed per-variant records (16-byte aligned)."""

    def __init__(self, batch: SystemBatchHost, device="cuda", stream=None):
        self.device = _require_cuda(device)
        lib = _capi.lib()
        batch.validate_values()
        self.topology = batch.topology
        self.variants = batch.variants
        self.stride = int(lib.mkb_record_stride(batch.surfaces, batch.wavelengths,
                                                batch.fields))
        host = np.zeros((max(batch.variants, 1), self.stride))
        view = batch.view()
        _capi.check(lib.mkb_pack_batch_host(C.byref(view), _capi.ptr(host)), "pack batch")
        self.host_records = torch.from_numpy(host[:batch.variants]).pin_memory()
        self.records = torch.empty((max(batch.variants, 1), self.stride), dtype=torch.float64,
                                   device=self.device)
        if batch.variants:
            with torch.cuda.stream(stream) if stream is not None else _nullcontext():
                self.records[:batch.variants].copy_(self.host_records, non_blocking=True)
        self.type = np.ascontiguousarray(batch.type, dtype=np.uint8)

    def c_struct(self, first: int = 0, count: int | None = None) -> _capi.DeviceBatch:
        count = self.variants - first if count is None else count
        b = _capi.DeviceBatch()
        b.variants = count
        b.surfaces = self.topology.surfaces
        b.wavelengths = self.topology.wavelengths
        b.fields = self.topology.fields
        b.record_stride = self.stride
        b.records = C.c_void_p(self.records.data_ptr() + first * self.stride * 8)
        b.type = _capi.ptr(self.type, C.c_uint8)
        b._keep = self.type
        return b


class _nullcontext:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


@dataclass
class ResidualOutput:
    residuals: np.ndarray | torch.Tensor  # [V][trace_rows]
    opd: np.ndarray | torch.Tensor        # [V][rays]
    status: np.ndarray | torch.Tensor     # [V][rays] uint8


@dataclass
class MeritOutput:
    merit: np.ndarray | torch.Tensor      # [V]
    failed: np.ndarray | torch.Tensor     # [V] int64
    hard_failed: np.ndarray | torch.Tensor


def residuals_device(dbatch: DeviceSystemBatch, layout: ResidualLayout, host: SystemBatchHost,
                     stream=None) -> ResidualOutput:
    """RESIDUALS on an uploaded batch; outputs stay on the device."""
    lib = _capi.lib()
    V = dbatch.variants
    res = torch.empty((V, layout.trace_rows), dtype=torch.float64, device=dbatch.device)
    opd = torch.empty((V, layout.rays_per_variant), dtype=torch.float64, device=dbatch.device)
    st = torch.empty((V, layout.rays_per_variant), dtype=torch.uint8, device=dbatch.device)
    b = dbatch.c_struct()
    plan = layout.plan(host)
    rc = lib.mkb_residuals_device(C.byref(b), C.byref(plan), C.c_void_p(res.data_ptr()),
                                  layout.trace_rows, C.c_void_p(opd.data_ptr()),
                                  C.c_void_p(st.data_ptr()), _stream_handle(stream))
    _capi.check(rc, "residuals")
    return ResidualOutput(res, opd, st)


def merit_device(dbatch: DeviceSystemBatch, layout: ResidualLayout, host: SystemBatchHost,
                 stream=None, workspace: torch.Tensor | None = None) -> MeritOutput:
    """MERIT on an uploaded batch; outputs stay on the device."""
    lib = _capi.lib()
    V = dbatch.variants
    plan = layout.plan(host)
    need = int(lib.mkb_merit_workspace_bytes(V, C.byref(plan)))
    if workspace is None or workspace.numel() < need:
        workspace = torch.empty(need, dtype=torch.uint8, device=dbatch.device)
    merit = torch.empty(V, dtype=torch.float64, device=dbatch.device)
    failed = torch.empty(V, dtype=torch.int64, device=dbatch.device)
    hard = torch.empty(V, dtype=torch.int64, device=dbatch.device)
    b = dbatch.c_struct()
    rc = lib.mkb_merit_device(C.byref(b), C.byref(plan), C.c_void_p(merit.data_ptr()),
                              C.c_void_p(failed.data_ptr()), C.c_void_p(hard.data_ptr()),
                              C.c_void_p(workspace.data_ptr()), workspace.numel(),
                              _stream_handle(stream))
    _capi.check(rc, "merit")
    return MeritOutput(merit, failed, hard)


class TraceEngine:
    """TraceEngine(device): host batch in, host results out (TraceEngine::run)."""

    def __init__(self, device: int = 0):
        self.device = _require_cuda(f"cuda:{device}")
        self._workspace = None

    def run(self, batch: SystemBatchHost, mode: TraceMode,
            settings: ResidualSettings | None = None):
        layout = ResidualLayout(batch.topology, settings or ResidualSettings())
        with torch.cuda.device(self.device):
            dbatch = DeviceSystemBatch(batch, self.device)
            if mode == TraceMode.RESIDUALS:
                out = residuals_device(dbatch, layout, batch)
                torch.cuda.synchronize()
                _device_status()
                return ResidualOutput(out.residuals.cpu().numpy(), out.opd.cpu().numpy(),
                                      out.status.cpu().numpy())
            if self._workspace is None:
                self._workspace = torch.empty(0, dtype=torch.uint8, device=self.device)
            need = int(_capi.lib().mkb_merit_workspace_bytes(batch.variants,
                                                            C.byref(layout.plan(batch))))
            if self._workspace.numel() < need:
                self._workspace = torch.empty(need, dtype=torch.uint8, device=self.device)
            out = merit_device(dbatch, layout, batch, workspace=self._workspace)
            torch.cuda.synchronize()
            _device_status()
            return MeritOutput(out.merit.cpu().numpy(), out.failed.cpu().numpy(),
                               out.hard_failed.cpu().numpy())


def _device_status() -> None:
    lib = _capi.lib()
    lib.mkb_device_status.restype = C.c_int
    _capi.check(lib.mkb_device_status(), "device status")
