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
import dataclasses
import math
from dataclasses import dataclass
import enum

import numpy as np
import torch

from . import _capi
from .batch import FAILURE_SOFT, ResidualLayout, ResidualSettings, SystemBatchHost


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
    """A batch resident in device memory as packed per-variant records (16-byte aligned).

    `storage` (a uint8 device tensor) lets a caller that keeps its buffers across calls, like
    TraceEngine, place the records in memory it already holds when it is large enough."""

    def __init__(self, batch: SystemBatchHost, device="cuda", stream=None,
                 storage: torch.Tensor | None = None, staging: torch.Tensor | None = None,
                 validated: bool = False):
        self.device = _require_cuda(device)
        lib = _capi.lib()
        if not validated:  # a caller that has just validated the batch skips the second pass
            batch.validate_values()
        self.topology = batch.topology
        self.variants = batch.variants
        self.non_coaxial = 1 if batch.non_coaxial else 0
        self.ghost_plates = batch.topology.ghost_plates
        self.ghost_terms = batch.topology.ghost_terms
        self.glass = 1 if batch.buchdahl_coeff is not None else 0
        self.wavelength_nm = np.ascontiguousarray(batch.wavelength_nm, dtype=np.float64)
        self.stride = int(lib.mkb_record_stride_ext(batch.surfaces, batch.wavelengths,
                                                    batch.fields, self.non_coaxial,
                                                    self.ghost_plates, self.ghost_terms,
                                                    self.glass))
        n_host = max(batch.variants, 1) * self.stride
        if staging is not None and staging.numel() >= n_host and staging.is_pinned():
            # a caller's pinned buffer, reused across calls (pinning memory is slow)
            self.host_records = staging[:n_host].view(-1, self.stride)
            host = self.host_records.numpy()
            host.fill(0.0)
        else:
            host = np.zeros((max(batch.variants, 1), self.stride))
            self.host_records = None
        view = batch.view()
        _capi.check(lib.mkb_pack_batch_host(C.byref(view), _capi.ptr(host)), "pack batch")
        if self.host_records is None:
            self.host_records = torch.from_numpy(host).pin_memory()
        self.host_records = self.host_records[:batch.variants]
        n = max(batch.variants, 1) * self.stride
        if storage is not None and storage.numel() >= 8 * n and storage.device == self.device:
            self.records = storage[:8 * n].view(torch.float64).view(-1, self.stride)
        else:
            self.records = torch.empty((max(batch.variants, 1), self.stride),
                                       dtype=torch.float64, device=self.device)
        if batch.variants:
            with torch.cuda.stream(stream) if stream is not None else _nullcontext():
                self.records[:batch.variants].copy_(self.host_records, non_blocking=True)
        self.type = np.ascontiguousarray(batch.type, dtype=np.uint8)
        self.variant_surfaces = None
        if batch.variant_surfaces is not None:
            self.variant_surfaces = torch.from_numpy(
                np.ascontiguousarray(batch.variant_surfaces, dtype=np.uint8)).to(self.device)

    def c_struct(self, first: int = 0, count: int | None = None) -> _capi.DeviceBatch:
        count = self.variants - first if count is None else count
        b = _capi.DeviceBatch()
        b.variants = count
        b.surfaces = self.topology.surfaces
        b.wavelengths = self.topology.wavelengths
        b.fields = self.topology.fields
        b.record_stride = self.stride
        b.non_coaxial = self.non_coaxial
        b.ghost_plates = self.ghost_plates
        b.ghost_terms = self.ghost_terms
        b.glass = self.glass
        b.wavelength_nm = _capi.ptr(self.wavelength_nm)
        b.records = C.c_void_p(self.records.data_ptr() + first * self.stride * 8)
        b.type = _capi.ptr(self.type, C.c_uint8)
        b._keep = (self.type, self.wavelength_nm)
        b.variant_surfaces = (C.c_void_p(self.variant_surfaces.data_ptr() + first)
                              if self.variant_surfaces is not None else None)
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


def _trace_options(pack_rays: int = 0, extra_merit: torch.Tensor | None = None,
                   extrema: torch.Tensor | None = None, variants_per_cta: int = 0):
    o = _capi.TraceOptions()
    o.pack_rays = int(pack_rays)
    o.variants_per_cta = int(variants_per_cta)
    o.extra_merit = C.c_void_p(extra_merit.data_ptr()) if extra_merit is not None else None
    o.extrema = C.c_void_p(extrema.data_ptr()) if extrema is not None else None
    return o


def residuals_device(dbatch: DeviceSystemBatch, layout: ResidualLayout, host: SystemBatchHost,
                     stream=None, pack_rays: int = 0,
                     variants_per_cta: int = 0) -> ResidualOutput:
    """RESIDUALS on an uploaded batch; outputs stay on the device."""
    lib = _capi.lib()
    V = dbatch.variants
    res = torch.empty((V, layout.trace_rows), dtype=torch.float64, device=dbatch.device)
    opd = torch.empty((V, layout.rays_per_variant), dtype=torch.float64, device=dbatch.device)
    st = torch.empty((V, layout.rays_per_variant), dtype=torch.uint8, device=dbatch.device)
    b = dbatch.c_struct()
    plan = layout.plan(host)
    opts = _trace_options(pack_rays, variants_per_cta=variants_per_cta)
    rc = lib.mkb_residuals_ex_device(C.byref(b), C.byref(plan), C.byref(opts),
                                     C.c_void_p(res.data_ptr()), layout.trace_rows,
                                     C.c_void_p(opd.data_ptr()), C.c_void_p(st.data_ptr()),
                                     _stream_handle(stream))
    _capi.check(rc, "residuals")
    return ResidualOutput(res, opd, st)


def merit_device(dbatch: DeviceSystemBatch, layout: ResidualLayout, host: SystemBatchHost,
                 stream=None, workspace: torch.Tensor | None = None, pack_rays: int = 0,
                 extra_merit: torch.Tensor | None = None,
                 variants_per_cta: int = 0) -> MeritOutput:
    """MERIT on an uploaded batch; outputs stay on the device. extra_merit: device [V] added to
    each variant's merit after its tuple sums."""
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
    if extra_merit is not None:
        extra_merit = extra_merit.to(device=dbatch.device, dtype=torch.float64).contiguous()
        if extra_merit.numel() != V:
            raise ValueError(f"extra_merit must hold {V} values")
    opts = _trace_options(pack_rays, extra_merit, variants_per_cta=variants_per_cta)
    rc = lib.mkb_merit_ex_device(C.byref(b), C.byref(plan), C.byref(opts),
                                 C.c_void_p(merit.data_ptr()), C.c_void_p(failed.data_ptr()),
                                 C.c_void_p(hard.data_ptr()), C.c_void_p(workspace.data_ptr()),
                                 workspace.numel(), _stream_handle(stream))
    _capi.check(rc, "merit")
    return MeritOutput(merit, failed, hard)


# ---- TraceEngine (include/mikroptim/cuda/trace_engine.hpp) ---------------------------------
@dataclass
class MemoryReserve:
    """MemoryReserve (include/mikroptim/batch/batch_memory.hpp:119): the engine leaves
    max(min_bytes, fraction * free) of the device memory it sees as free untouched."""

    min_bytes: int = 256 << 20
    fraction: float = 0.05


@dataclass
class EngineOptions:
    """EngineOptions (trace_engine.hpp:44). memory_limit_bytes caps the memory the engine
    regards as available (tranche tests, sharing a GPU); None: the device's free memory."""

    memory_limit_bytes: int | None = None
    reserve: MemoryReserve = dataclasses.field(default_factory=MemoryReserve)


@dataclass
class TraceSettings:
    """TraceSettings (trace_engine.hpp:52). opd / status / extra_residuals apply to RESIDUALS
    (the extra rows follow the ray and penalty rows and are set to 0); extra_merit (host [V] or
    None) to MERIT, added to each variant's merit after its tuple sums. precision None: the
    quadrature's. pack_rays changes only the run time (bit-identical results for every value).
    extrema: per variant and surface the largest ray height and the smallest cos I of the valid
    rays (SurfaceExtremaResult, hard maxima; a tilted surface's in its own frame) in the
    result's `extrema` [V][S][2]."""

    quadrature: ResidualSettings = dataclasses.field(default_factory=ResidualSettings)
    opd: bool = False
    status: bool = True
    extra_residuals: int = 0
    extrema: bool = False
    extra_merit: np.ndarray | None = None
    precision: int | None = None
    pack_rays: int = 512


@dataclass
class TraceRunInfo:
    """TraceRunInfo (trace_engine.hpp:93)."""

    variants: int = 0
    tranches: int = 0
    tranche_variants: int = 0
    budget_bytes: int = 0
    device_bytes: int = 0


@dataclass
class ResidualResult:
    """ResidualResult (batch_residuals.hpp): residuals [V][stride], opd / status [V][rays]
    (empty when not requested)."""

    variants: int = 0
    rays_per_variant: int = 0
    penalty_rows: int = 0
    stride: int = 0
    residuals: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 0)))
    opd: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 0)))
    status: np.ndarray = dataclasses.field(
        default_factory=lambda: np.zeros((0, 0), dtype=np.uint8))
    extrema: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 0, 2)))


@dataclass
class MeritResult:
    """MeritResult (batch_merit.hpp:32)."""

    variants: int = 0
    rays_per_variant: int = 0
    merit: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0))
    failed: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0, dtype=np.int64))
    hard_failed: np.ndarray = dataclasses.field(
        default_factory=lambda: np.zeros(0, dtype=np.int64))
    extrema: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 0, 2)))


@dataclass
class TraceOutput:
    """TraceOutput (trace_engine.hpp:103): the result of the run's mode; the other is empty."""

    mode: TraceMode = TraceMode.RESIDUALS
    layout: ResidualLayout | None = None
    residuals: ResidualResult = dataclasses.field(default_factory=ResidualResult)
    merit: MeritResult = dataclasses.field(default_factory=MeritResult)
    info: TraceRunInfo = dataclasses.field(default_factory=TraceRunInfo)


@dataclass
class DeviceTranche:
    """DeviceTranche (trace_engine.hpp:117): one tranche's RESIDUALS on the device, views of
    the engine's buffers valid during the callback only."""

    first: int
    count: int
    rays_per_variant: int
    penalty_rows: int
    stride: int
    residuals: torch.Tensor            # [count][stride]
    status: torch.Tensor               # [count][rays]
    opd: torch.Tensor | None           # [count][rays] when settings.opd
    extrema: torch.Tensor | None = None  # [count][S][2] when settings.extrema


def _as_trace_settings(settings) -> TraceSettings:
    if settings is None:
        return TraceSettings()
    if isinstance(settings, TraceSettings):
        return settings
    if isinstance(settings, ResidualSettings):
        return TraceSettings(quadrature=settings)
    raise TypeError("settings must be TraceSettings or ResidualSettings")


class TraceEngine:
    """TraceEngine(device, options) (include/mikroptim/cuda/trace_engine.hpp:145): host batch
    in, host results out. Splits a batch into tranches that fit the device memory it sees
    (free memory plus its own buffers, at most options.memory_limit_bytes, less the reserve)
    and keeps its buffers across calls; every variant's results are bit-identical whatever the
    split (the kernels do not depend on a variant's position in the batch)."""

    def __init__(self, device: int = 0, options: EngineOptions | None = None):
        self.device = _require_cuda(f"cuda:{device}")
        self.options = options or EngineOptions()
        self._usable(0)  # checks the reserve (ValueError for a fraction outside [0, 1])
        self.device_name = torch.cuda.get_device_name(self.device)
        self._buffers: dict[str, torch.Tensor] = {}
        self._staging: torch.Tensor | None = None  # pinned host records, grown on demand
        self._last_usable = 0

    def _host_staging(self, doubles: int) -> torch.Tensor:
        if self._staging is None or self._staging.numel() < doubles:
            self._staging = torch.empty(max(int(doubles), 1), dtype=torch.float64).pin_memory()
        return self._staging

    # ---- memory ---------------------------------------------------------------------------
    def device_bytes(self) -> int:
        """Device memory the engine holds now (batch and outputs) [bytes]."""
        return sum(t.numel() for t in self._buffers.values())

    def release(self) -> None:
        """Frees every device buffer (the next run allocates them again)."""
        self._buffers.clear()
        self._last_usable = 0

    def _usable(self, available: int) -> int:
        out = C.c_size_t(0)
        r = self.options.reserve
        _capi.check(_capi.lib().mkb_usable_bytes(int(available), int(r.min_bytes),
                                                  float(r.fraction), C.byref(out)),
                    "memory reserve")
        return int(out.value)

    def _available(self) -> int:
        free, _ = torch.cuda.mem_get_info(self.device)
        cached = (torch.cuda.memory_reserved(self.device) -
                  torch.cuda.memory_allocated(self.device))
        available = int(free) + int(cached) + self.device_bytes()
        if self.options.memory_limit_bytes is not None:
            available = min(available, int(self.options.memory_limit_bytes))
        return available

    def _buffer(self, name: str, nbytes: int) -> torch.Tensor:
        buf = self._buffers.get(name)
        if buf is None or buf.numel() < nbytes:
            self._buffers.pop(name, None)  # the old buffer goes before the new one comes
            buf = torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=self.device)
            self._buffers[name] = buf
        return buf

    @staticmethod
    def _shape(topology, glass: bool, variant_surfaces: bool = False) -> _capi.DeviceBatch:
        lib = _capi.lib()
        b = _capi.DeviceBatch()
        b.variants = 0
        b.surfaces, b.wavelengths, b.fields = (topology.surfaces, topology.wavelengths,
                                                topology.fields)
        b.non_coaxial = 1 if topology.non_coaxial else 0
        b.ghost_plates, b.ghost_terms = topology.ghost_plates, topology.ghost_terms
        b.glass = 1 if glass else 0
        b.record_stride = int(lib.mkb_record_stride_ext(b.surfaces, b.wavelengths, b.fields,
                                                        b.non_coaxial, b.ghost_plates,
                                                        b.ghost_terms, b.glass))
        t = np.ascontiguousarray(topology.type, dtype=np.uint8)
        b.type = _capi.ptr(t, C.c_uint8)
        b.records = None
        b.variant_surfaces = C.c_void_p(1) if variant_surfaces else None  # never dereferenced
        b._keep = (t,)
        return b

    @staticmethod
    def _layout(topology, ts: TraceSettings) -> ResidualLayout:
        q = ts.quadrature
        if ts.precision is not None:
            q = dataclasses.replace(q, precision=ts.precision)
        return ResidualLayout(topology, q)

    @staticmethod
    def _check(ts: TraceSettings) -> None:
        if ts.extra_residuals < 0:
            raise ValueError("TraceEngine: extra_residuals must be >= 0")
        if ts.pack_rays < 1:
            raise ValueError("TraceEngine: pack_rays must be >= 1")

    def _tranche(self, shape, layout: ResidualLayout, plan, ts: TraceSettings, merit: bool,
                 granularity: int, usable: int) -> int:
        opts = _trace_options(ts.pack_rays)
        n = int(_capi.lib().mkb_trace_tranche_variants(
            int(usable), C.byref(shape), C.byref(plan), C.byref(opts), 1 if merit else 0,
            int(ts.extra_residuals), 1 if ts.opd else 0,
            1 if (merit and ts.extra_merit is not None) else 0, int(granularity)))
        if n < 0:
            _capi.check(n, "tranche plan")
        return n

    def max_variants(self, topology, mode: TraceMode, settings=None, glass: bool = False) -> int:
        """Largest tranche for batches of this topology (TraceEngine::max_variants): the free
        device memory plus the engine's own buffers, at most memory_limit_bytes, less the
        reserve and the fixed per-run buffers. 0 when not one variant fits."""
        ts = _as_trace_settings(settings)
        self._check(ts)
        layout = self._layout(topology, ts)
        host = _UnitWeights(topology)
        return self._tranche(self._shape(topology, glass), layout, layout.plan(host), ts,
                             mode == TraceMode.MERIT, 1, self._usable(self._available()))

    def _plan(self, batch: SystemBatchHost, layout: ResidualLayout, ts: TraceSettings,
              merit: bool, granularity: int, plan=None) -> tuple[int, int]:
        shape = self._shape(batch.topology, batch.buchdahl_coeff is not None,
                            batch.variant_surfaces is not None)
        plan = plan if plan is not None else layout.plan(batch)
        # A batch whose whole run fits the buffers this mode already holds reuses them without
        # asking the device (cudaMemGetInfo costs about a millisecond): the previous plan
        # reserved them within the same limits.
        per, fixed = C.c_size_t(0), C.c_size_t(0)
        _capi.check(_capi.lib().mkb_trace_run_bytes(
            C.byref(shape), C.byref(plan), 1 if merit else 0, int(ts.extra_residuals),
            1 if ts.opd else 0, 1 if (merit and ts.extra_merit is not None) else 0,
            C.byref(per), C.byref(fixed)), "run bytes")
        mine = ("records", "merit", "failed", "hard", "ws", "extra") if merit else \
            ("records", "res", "status", "opd")
        held_mine = sum(self._buffers[k].numel() for k in mine if k in self._buffers)
        if self._last_usable and held_mine >= batch.variants * per.value and \
                self._last_usable >= fixed.value + batch.variants * per.value:
            return batch.variants, self._last_usable
        # the other mode's buffers stay while the tranche does not shrink because of them
        other = ("res", "status", "opd") if merit else ("merit", "failed", "hard", "ws", "extra")
        held = sum(self._buffers[k].numel() for k in other if k in self._buffers)
        available = self._available()
        usable = self._usable(available - min(held, available))
        tranche = self._tranche(shape, layout, plan, ts, merit, granularity, usable)
        if held and tranche < batch.variants:
            usable_all = self._usable(available)
            tranche_all = self._tranche(shape, layout, plan, ts, merit, granularity, usable_all)
            if tranche_all > tranche:
                for k in other:
                    self._buffers.pop(k, None)
                tranche, usable = tranche_all, usable_all
        if tranche < 1:
            what = ("one variant fits" if granularity == 1
                    else f"{granularity} variants that belong together fit")
            raise RuntimeError(f"TraceEngine: not even {what} into the device memory "
                               f"(available {available / 2**20:.1f} MiB, after the reserve "
                               f"{usable / 2**20:.1f} MiB)")
        self._last_usable = usable
        return min(tranche, batch.variants), usable

    # ---- runs -----------------------------------------------------------------------------
    def run(self, batch: SystemBatchHost, mode: TraceMode, settings=None,
            out: TraceOutput | None = None) -> TraceOutput:
        """TraceEngine::run: validate, plan the tranches, then per tranche upload, kernel and
        download into the host result at the tranche's first variant. Synchronous."""
        ts = _as_trace_settings(settings)
        self._check(ts)
        if not isinstance(mode, TraceMode):
            raise ValueError("TraceEngine: unknown mode")
        layout = self._layout(batch.topology, ts)
        batch.validate_values()
        V = batch.variants
        merit = mode == TraceMode.MERIT
        extra = None
        if merit and ts.extra_merit is not None:
            extra = np.ascontiguousarray(ts.extra_merit, dtype=np.float64).reshape(-1)
            if extra.size != V:
                raise ValueError(f"TraceEngine: extra_merit must be empty or hold {V} values")
        reuse = out is not None
        out = out if out is not None else TraceOutput()
        rays = layout.rays_per_variant
        stride = layout.trace_rows + ts.extra_residuals
        out.mode, out.layout = mode, layout
        out.info = TraceRunInfo(variants=V)
        # A loop that passes its `out` back gets its results in pinned memory that `out` keeps
        # (downloaded straight into, the reference keeps its vectors' capacity likewise); a
        # call without `out` gets fresh arrays.
        pin = out.__dict__.setdefault("_pinned", {})

        def host(name, shape, dtype):
            n = int(np.prod(shape))
            if not reuse:
                return torch.empty(shape, dtype=dtype)
            t = pin.get(name)
            if t is None or t.numel() < n or t.dtype != dtype:
                t = torch.empty(max(n, 1), dtype=dtype).pin_memory()
                pin[name] = t
            return t[:n].view(*shape)

        hp = {}
        S = batch.surfaces
        if ts.extrema:
            hp["extrema"] = host("extrema", (V, S, 2), torch.float64)
        if merit:
            hp["merit"] = host("merit", (V,), torch.float64)
            hp["failed"] = host("failed", (V,), torch.int64)
            hp["hard"] = host("hard", (V,), torch.int64)
            out.residuals = ResidualResult()
            out.merit = MeritResult(V, rays, hp["merit"].numpy(), hp["failed"].numpy(),
                                    hp["hard"].numpy())
            if ts.extrema:
                out.merit.extrema = hp["extrema"].numpy()
        else:
            hp["res"] = host("res", (V, stride), torch.float64)
            if ts.opd:
                hp["opd"] = host("opd", (V, rays), torch.float64)
            if ts.status:
                hp["status"] = host("status", (V, rays), torch.uint8)
            out.merit = MeritResult()
            out.residuals = ResidualResult(
                V, rays, layout.penalty_rows, stride, hp["res"].numpy(),
                hp["opd"].numpy() if ts.opd else np.zeros((0, 0)),
                hp["status"].numpy() if ts.status else np.zeros((0, 0), dtype=np.uint8))
            if ts.extrema:
                out.residuals.extrema = hp["extrema"].numpy()
        if V == 0:
            out.info.device_bytes = self.device_bytes()
            return out
        with torch.cuda.device(self.device):
            plan = layout.plan(batch)  # one plan per call (the tranches share its weights)
            tranche, usable = self._plan(batch, layout, ts, merit, 1, plan)
            for first in range(0, V, tranche):
                count = min(tranche, V - first)
                part = batch.subset(first, count) if (first, count) != (0, V) else batch
                sl = slice(first, first + count)
                if merit:
                    m = self._merit_tranche(part, layout, ts,
                                            None if extra is None else extra[first:first + count],
                                            plan)
                    hp["merit"][sl].copy_(m.merit, non_blocking=True)
                    hp["failed"][sl].copy_(m.failed, non_blocking=True)
                    hp["hard"][sl].copy_(m.hard_failed, non_blocking=True)
                    if ts.extrema:
                        hp["extrema"][sl].copy_(self._last_extrema, non_blocking=True)
                else:
                    t = self._residual_tranche(part, layout, ts, first, plan)
                    hp["res"][sl].copy_(t.residuals, non_blocking=True)
                    if ts.status:
                        hp["status"][sl].copy_(t.status, non_blocking=True)
                    if ts.opd:
                        hp["opd"][sl].copy_(t.opd, non_blocking=True)
                    if ts.extrema:
                        hp["extrema"][sl].copy_(t.extrema, non_blocking=True)
                torch.cuda.current_stream(self.device).synchronize()
                _device_status()
                out.info.tranches += 1
            out.info.tranche_variants = tranche
            out.info.budget_bytes = usable
            out.info.device_bytes = self.device_bytes()
        return out

    def prefilter_variants(self, batch: SystemBatchHost,
                           settings: "PrefilterSettings | None" = None) -> "PrefilterResult":
        """FP32 prefilter of all variants (TraceEngine::prefilter_variants,
        include/mikroptim/cuda/trace_engine.hpp:188): the float trace with margins on the device,
        then the conservative decision on the host. The values only bound the FP64 merit for
        the selection; kept variants are evaluated again with run()."""
        settings = settings or PrefilterSettings()
        layout = ResidualLayout(batch.topology, settings.quadrature)
        stats = prefilter_device(DeviceSystemBatch(batch, self.device), layout, batch,
                                 settings.options.boundary)
        return prefilter_decide(stats, layout, batch, settings.options, settings.extra_merit)

    def evaluate(self, batch: SystemBatchHost, settings: "EvalSettings | None" = None):
        """Mode EVAL (TraceEngine::evaluate, include/mikroptim/cuda/trace_engine.hpp:193): OPD
        maps, spots and field rays of every variant on the dense pupil grid."""
        return evaluate_device(DeviceSystemBatch(batch, self.device), batch, settings)

    def run_on_device(self, batch: SystemBatchHost, settings, granularity: int,
                      consume) -> TraceRunInfo:
        """TraceEngine::run_on_device: RESIDUALS without the download. After each tranche's
        kernel the engine calls consume(DeviceTranche) with views of its device buffers; the
        tranche size is a multiple of `granularity` (only the last may be smaller)."""
        ts = _as_trace_settings(settings)
        self._check(ts)
        if granularity < 1:
            raise ValueError("TraceEngine: granularity must be >= 1")
        if consume is None:
            raise ValueError("TraceEngine: run_on_device without a callback")
        layout = self._layout(batch.topology, ts)
        batch.validate_values()
        V = batch.variants
        info = TraceRunInfo(variants=V)
        if V == 0:
            info.device_bytes = self.device_bytes()
            return info
        with torch.cuda.device(self.device):
            plan = layout.plan(batch)
            tranche, usable = self._plan(batch, layout, ts, False, granularity, plan)
            for first in range(0, V, tranche):
                count = min(tranche, V - first)
                part = batch.subset(first, count) if (first, count) != (0, V) else batch
                t = self._residual_tranche(part, layout, ts, first, plan)
                torch.cuda.synchronize()
                _device_status()
                consume(t)
                torch.cuda.synchronize()
                info.tranches += 1
            info.tranche_variants = tranche
            info.budget_bytes = usable
            info.device_bytes = self.device_bytes()
        return info

    def _residual_tranche(self, part: SystemBatchHost, layout: ResidualLayout,
                          ts: TraceSettings, first: int, plan=None) -> DeviceTranche:
        """One tranche's RESIDUALS on the device; `part` was validated by the caller and `plan`
        (or None) is the run's plan, whose weights every tranche shares."""
        lib = _capi.lib()
        n = part.variants
        rays = layout.rays_per_variant
        stride = layout.trace_rows + ts.extra_residuals
        sv = n * self._stride_of(part)
        db = DeviceSystemBatch(part, self.device, storage=self._buffer("records", 8 * sv),
                               staging=self._host_staging(sv), validated=True)
        res = self._buffer("res", 8 * n * stride)[:8 * n * stride].view(torch.float64)
        res = res.view(n, stride)
        st = self._buffer("status", n * rays)[:n * rays].view(n, rays)
        opd = None
        if ts.opd:
            opd = self._buffer("opd", 8 * n * rays)[:8 * n * rays].view(torch.float64)
            opd = opd.view(n, rays)
        if ts.extra_residuals:
            res[:, layout.trace_rows:].zero_()
        b = db.c_struct()
        plan = plan if plan is not None else layout.plan(part)
        ext = self._extrema_buffer(part, ts)
        opts = _trace_options(ts.pack_rays, None, ext)
        rc = lib.mkb_residuals_ex_device(C.byref(b), C.byref(plan), C.byref(opts),
                                         C.c_void_p(res.data_ptr()), stride,
                                         C.c_void_p(opd.data_ptr()) if opd is not None else None,
                                         C.c_void_p(st.data_ptr()), _stream_handle(None))
        _capi.check(rc, "residuals")
        return DeviceTranche(first, n, rays, layout.penalty_rows, stride, res, st, opd,
                             ext)

    def _merit_tranche(self, part: SystemBatchHost, layout: ResidualLayout, ts: TraceSettings,
                       extra: np.ndarray | None, plan=None) -> MeritOutput:
        """One tranche's MERIT on the device (`part` validated by the caller, `plan` as in
        _residual_tranche)."""
        lib = _capi.lib()
        n = part.variants
        sv = n * self._stride_of(part)
        db = DeviceSystemBatch(part, self.device, storage=self._buffer("records", 8 * sv),
                               staging=self._host_staging(sv), validated=True)
        plan = plan if plan is not None else layout.plan(part)
        ws = self._buffer("ws", int(lib.mkb_merit_workspace_bytes(n, C.byref(plan))))
        merit = self._buffer("merit", 8 * n)[:8 * n].view(torch.float64)
        failed = self._buffer("failed", 8 * n)[:8 * n].view(torch.int64)
        hard = self._buffer("hard", 8 * n)[:8 * n].view(torch.int64)
        extra_dev = None
        if extra is not None:
            extra_dev = self._buffer("extra", 8 * n)[:8 * n].view(torch.float64)
            extra_dev.copy_(torch.from_numpy(np.ascontiguousarray(extra)))
        b = db.c_struct()
        ext = self._extrema_buffer(part, ts)
        self._last_extrema = ext
        opts = _trace_options(ts.pack_rays, extra_dev, ext)
        rc = lib.mkb_merit_ex_device(C.byref(b), C.byref(plan), C.byref(opts),
                                     C.c_void_p(merit.data_ptr()), C.c_void_p(failed.data_ptr()),
                                     C.c_void_p(hard.data_ptr()), C.c_void_p(ws.data_ptr()),
                                     ws.numel(), _stream_handle(None))
        _capi.check(rc, "merit")
        return MeritOutput(merit, failed, hard)

    def _extrema_buffer(self, part: SystemBatchHost, ts: TraceSettings):
        if not ts.extrema:
            return None
        n = part.variants * part.surfaces * 2
        return self._buffer("extrema", 8 * n)[:8 * n].view(torch.float64).view(
            part.variants, part.surfaces, 2)

    @staticmethod
    def _stride_of(batch: SystemBatchHost) -> int:
        return int(_capi.lib().mkb_record_stride_ext(
            batch.surfaces, batch.wavelengths, batch.fields, 1 if batch.non_coaxial else 0,
            batch.topology.ghost_plates, batch.topology.ghost_terms,
            1 if batch.buchdahl_coeff is not None else 0))


@dataclass
class PrefilterOptions:
    """PrefilterCriteria + PrefilterMargins (include/mikroptim/batch/batch_prefilter.hpp:35,52)
    with the reference's defaults."""

    max_failed_fraction: float = 0.5
    max_merit: float = float("inf")
    max_merit_factor: float = float("inf")
    boundary: float = 0.15
    opl_error_factor: float = 32.0
    merit_relative: float = 0.01

    def c_struct(self) -> _capi.PrefilterOptions:
        return _capi.PrefilterOptions(self.max_failed_fraction, self.max_merit,
                                      self.max_merit_factor, self.boundary,
                                      self.opl_error_factor, self.merit_relative)


@dataclass
class PrefilterSettings:
    """PrefilterSettings (trace_engine.hpp:80): the quadrature of the later FP64 run, the
    options, and an optional FP64 merit share per variant added to both bounds."""

    quadrature: ResidualSettings = dataclasses.field(default_factory=ResidualSettings)
    options: PrefilterOptions = dataclasses.field(default_factory=PrefilterOptions)
    extra_merit: np.ndarray | None = None


@dataclass
class PrefilterStats:
    """PrefilterStats (batch_prefilter.hpp:66): float results per variant, stored as double."""

    variants: int = 0
    rays_per_variant: int = 0
    merit: np.ndarray = None
    optical_length: np.ndarray = None
    failed: np.ndarray = None
    uncertain_ok: np.ndarray = None
    uncertain_failed: np.ndarray = None

    def uncertain(self, v: int) -> int:
        return int(self.uncertain_ok[v] + self.uncertain_failed[v])


@dataclass
class PrefilterResult:
    """PrefilterResult (batch_prefilter.hpp:94): bounds of the FP64 merit, the reason mask per
    variant (0 = keep), the best-merit bound criterion (c) used and its variant, the count
    kept."""

    stats: PrefilterStats
    merit_lower: np.ndarray
    merit_upper: np.ndarray
    reject: np.ndarray
    reference_merit: float
    reference_variant: int
    kept: int

    def keep(self, v: int) -> bool:
        return self.reject[v] == _capi.MKB_PREFILTER_KEEP


def prefilter_device(dbatch: DeviceSystemBatch, layout: ResidualLayout, host: SystemBatchHost,
                     boundary: float = 0.15, stream=None) -> PrefilterStats:
    """The FP32 prefilter kernel on an uploaded batch (DevicePrefilter::run + download,
    include/mikroptim/cuda/prefilter.hpp): per-variant raw results, bit-identical to the
    reference's prefilter_stats_cpu."""
    lib = _capi.lib()
    V = dbatch.variants
    dev = dbatch.device
    view = host.view()
    trig = np.zeros((max(V, 1), host.fields, 2), dtype=np.float32)
    _capi.check(lib.mkb_prefilter_field_trig_host(C.byref(view), trig.ctypes.data),
                "prefilter field table")
    trig_d = torch.from_numpy(trig).to(dev)
    plan = layout.plan(host)
    outs = [torch.empty(max(V, 1), dtype=t, device=dev)
            for t in (torch.float64, torch.float64, torch.int64, torch.int64, torch.int64)]
    need = int(lib.mkb_prefilter_workspace_bytes(V, C.byref(plan)))
    ws = torch.empty(max(need, 1), dtype=torch.uint8, device=dev)
    b = dbatch.c_struct()
    rc = lib.mkb_prefilter_device(C.byref(b), C.byref(plan), C.c_void_p(trig_d.data_ptr()),
                                  float(boundary), *[C.c_void_p(o.data_ptr()) for o in outs],
                                  C.c_void_p(ws.data_ptr()), ws.numel(), _stream_handle(stream))
    _capi.check(rc, "prefilter")
    host_outs = [o[:V].cpu().numpy() for o in outs]
    return PrefilterStats(V, layout.rays_per_variant, *host_outs)


def prefilter_decide(stats: PrefilterStats, layout: ResidualLayout, host: SystemBatchHost,
                     options: PrefilterOptions | None = None,
                     extra_merit=None) -> PrefilterResult:
    """prefilter_decide (src/batch/batch_prefilter.cpp): the conservative decision from the raw
    results (mkb_prefilter_decide_host)."""
    lib = _capi.lib()
    options = options or PrefilterOptions()
    V = stats.variants
    if extra_merit is not None:
        extra_merit = np.ascontiguousarray(extra_merit, dtype=np.float64)
        if extra_merit.shape != (V,):
            raise ValueError(f"prefilter: extra_merit must have {V} values")
    arrs = [np.ascontiguousarray(a, dtype=t) for a, t in (
        (stats.merit, np.float64), (stats.optical_length, np.float64),
        (stats.failed, np.int64), (stats.uncertain_ok, np.int64),
        (stats.uncertain_failed, np.int64))]
    lower, upper = np.zeros(V), np.zeros(V)
    reject = np.zeros(V, dtype=np.uint8)
    ref_m, ref_v, kept = C.c_double(), C.c_int32(), C.c_int32()
    plan = layout.plan(host)
    opts = options.c_struct()
    rc = lib.mkb_prefilter_decide_host(
        C.byref(plan), C.byref(opts), V, *[a.ctypes.data for a in arrs],
        extra_merit.ctypes.data if extra_merit is not None else None, lower.ctypes.data,
        upper.ctypes.data, reject.ctypes.data, C.addressof(ref_m), C.addressof(ref_v),
        C.addressof(kept))
    _capi.check(rc, "prefilter decide")
    stats = dataclasses.replace(stats, merit=arrs[0], optical_length=arrs[1], failed=arrs[2],
                                uncertain_ok=arrs[3], uncertain_failed=arrs[4])
    return PrefilterResult(stats, lower, upper, reject, ref_m.value, ref_v.value, kept.value)


def prefilter_decide_exact(merit, failed, rays_per_variant: int,
                           options: PrefilterOptions | None = None, extra_merit=None):
    """prefilter_decide_exact: the same rule without margins on FP64 merits (the truth)."""
    lib = _capi.lib()
    options = options or PrefilterOptions()
    merit = np.ascontiguousarray(merit, dtype=np.float64)
    failed = np.ascontiguousarray(failed, dtype=np.int64)
    ex = None if extra_merit is None else np.ascontiguousarray(extra_merit, dtype=np.float64)
    reject = np.zeros(len(merit), dtype=np.uint8)
    opts = options.c_struct()
    rc = lib.mkb_prefilter_decide_exact_host(C.byref(opts), len(merit), rays_per_variant,
                                             merit.ctypes.data, failed.ctypes.data,
                                             ex.ctypes.data if ex is not None else None,
                                             reject.ctypes.data)
    _capi.check(rc, "prefilter decide exact")
    return reject


EVAL_EXIT_PUPIL, EVAL_VERTEX, EVAL_INFINITE = 0, 1, 2


@dataclass
class EvalSettings:
    """EvalSettings (include/mikroptim/eval/eval.hpp:27): grid edge N, half pupil (x >= 0),
    the reference sphere (EVAL_EXIT_PUPIL, EVAL_VERTEX, EVAL_INFINITE), the field-ray offset;
    paraxial_column: the wavelength column holding the paraxial index (exit-pupil position)."""

    grid: int = 64
    half_pupil: bool = False
    reference: int = EVAL_EXIT_PUPIL
    field_ray_offset: float = 1e-3
    paraxial_column: int = 0
    precision: int = 0  # PRECISION_FP64 (the reference's arithmetic) or PRECISION_FP64_FMA


@dataclass
class EvalResult:
    """EvalResult (eval.hpp:96): ray (v, f, l, k) at ((v F + f) L + l) n + k; field ray j at
    ((v F + f) L + l) 4 + j with values (x, y, d_x, d_y, d_z). OPD and spot in mm (spot
    relative to the ideal image point); failed rays NaN with their status."""

    variants: int
    fields: int
    wavelengths: int
    grid: np.ndarray              # [n][3] x, y, weight
    reference_curvature: np.ndarray
    exit_pupil_position: np.ndarray
    opd: np.ndarray
    spot_x: np.ndarray
    spot_y: np.ndarray
    status: np.ndarray
    field_rays: np.ndarray
    field_status: np.ndarray
    grid_size: int = 0        # N
    half_pupil: bool = False
    field_ray_offset: float = 1e-3

    @property
    def samples(self) -> int:
        return self.grid.shape[0]


def eval_grid(size: int, half_pupil: bool = False) -> np.ndarray:
    """make_eval_grid: cell centres inside the unit pupil with their weights, [n][3]."""
    lib = _capi.lib()
    n = C.c_int64()
    _capi.check(lib.mkb_eval_grid_host(size, int(half_pupil), None, C.byref(n)), "eval grid")
    pts = np.zeros((n.value, 3))
    _capi.check(lib.mkb_eval_grid_host(size, int(half_pupil), pts.ctypes.data, C.byref(n)),
                "eval grid")
    return pts


def evaluate_device(dbatch: "DeviceSystemBatch", host: SystemBatchHost,
                    settings: EvalSettings | None = None, stream=None) -> EvalResult:
    """EVAL on an uploaded batch (TraceEngine::evaluate, the kernel EVAL): bit-identical to
    the reference's eval_cpu."""
    settings = settings or EvalSettings()
    pts, kappa, z_ap, out = evaluate_device_tensors(dbatch, host, settings, stream)
    h = {k: v.cpu().numpy() for k, v in out.items()}
    return EvalResult(host.variants, host.fields, host.wavelengths, pts, kappa.reshape(-1), z_ap,
                      h["opd"], h["sx"], h["sy"], h["st"], h["fr"], h["fs"], settings.grid,
                      settings.half_pupil, settings.field_ray_offset)


def evaluate_device_tensors(dbatch: "DeviceSystemBatch", host: SystemBatchHost,
                            settings: EvalSettings | None = None, stream=None):
    """EVAL leaving its outputs on the device: grid points [n][3], kappa [V][F], exit-pupil
    positions [V] (host) and the device tensors opd, sx, sy, st [V F L n], fr [V F L 4 5],
    fs [V F L 4]."""
    lib = _capi.lib()
    settings = settings or EvalSettings()
    if settings.half_pupil and host.non_coaxial:
        raise ValueError("EVAL: half pupil only for coaxial systems")
    dev = dbatch.device
    V, F, L = host.variants, host.fields, host.wavelengths
    pts = eval_grid(settings.grid, settings.half_pupil)
    n = pts.shape[0]
    kappa = np.zeros((V, F))
    z_ap = np.zeros(V)
    view = host.view()
    _capi.check(lib.mkb_eval_reference_host(C.byref(view), settings.reference,
                                            settings.paraxial_column, kappa.ctypes.data,
                                            z_ap.ctypes.data), "eval reference")
    T = V * F * L
    out = dict(opd=torch.empty(T * n, dtype=torch.float64, device=dev),
               sx=torch.empty(T * n, dtype=torch.float64, device=dev),
               sy=torch.empty(T * n, dtype=torch.float64, device=dev),
               st=torch.empty(T * n, dtype=torch.uint8, device=dev),
               fr=torch.empty(T * 20, dtype=torch.float64, device=dev),
               fs=torch.empty(T * 4, dtype=torch.uint8, device=dev))
    grid_d = torch.from_numpy(pts).to(dev)
    kappa_d = torch.from_numpy(kappa).to(dev)
    b = dbatch.c_struct()
    ws = torch.empty(int(lib.mkb_eval_workspace_bytes(C.byref(b))), dtype=torch.uint8,
                     device=dev)
    rc = lib.mkb_eval_device(C.byref(b), settings.reference, settings.field_ray_offset,
                             settings.precision, C.c_void_p(grid_d.data_ptr()), n, C.c_void_p(kappa_d.data_ptr()),
                             *[C.c_void_p(out[k].data_ptr()) for k in
                               ("opd", "sx", "sy", "st", "fr", "fs")],
                             C.c_void_p(ws.data_ptr()), ws.numel(), _stream_handle(stream))
    _capi.check(rc, "eval")
    return pts, kappa, z_ap, out


class _UnitWeights:
    """The weights a plan reads, for sizing a run of a topology alone (sizes do not depend on
    the weights)."""

    def __init__(self, topology):
        self.field_weight = np.ones(topology.fields)
        self.wavelength_weight = np.ones(topology.wavelengths)
        self.reference_wavelength_nm = 587.56


def _device_status() -> None:
    lib = _capi.lib()
    lib.mkb_device_status.restype = C.c_int
    _capi.check(lib.mkb_device_status(), "device status")


# ---- Jacobians and normal equations (device) --------------------------------------------
def _dev_f64(a, device):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).to(device)


def _x_rows(x0, P: int, device):
    """Variable rows [runs][P] on the device: a device tensor is used in place (no copy when
    it is already contiguous FP64), host arrays are copied."""
    if isinstance(x0, torch.Tensor):
        return x0.to(device=device, dtype=torch.float64).reshape(-1, P).contiguous()
    return _dev_f64(np.asarray(x0).reshape(-1, P), device)


def fd_jacobian_device(templates: DeviceSystemBatch, layout: ResidualLayout,
                       host: SystemBatchHost, variables, x0, chunk_runs: int | None = None,
                       stream=None):
    """Central-difference Jacobian of runs x0 [runs][P] (DeviceFdJacobian::compute).
    Returns device tensors J [runs][P][R], r0 [runs][R], status_changes [runs][P]."""
    lib = _capi.lib()
    dev = templates.device
    x0 = _x_rows(x0, variables.size, dev)
    runs, P = x0.shape
    R = layout.trace_rows
    b = templates.c_struct()
    plan = layout.plan(host)
    chunk = runs if chunk_runs is None else chunk_runs
    need = int(lib.mkb_fd_jacobian_workspace_bytes(C.byref(b), C.byref(plan), P, runs, chunk))
    ws = torch.empty(max(need, 1), dtype=torch.uint8, device=dev)
    J = torch.empty((runs, P, R), dtype=torch.float64, device=dev)
    r0 = torch.empty((runs, R), dtype=torch.float64, device=dev)
    ch = torch.empty((runs, P), dtype=torch.int64, device=dev)
    vs = variables.c_struct()
    rc = lib.mkb_fd_jacobian_device(C.byref(b), C.byref(plan), C.byref(vs),
                                    C.c_void_p(x0.data_ptr()), runs, C.c_void_p(J.data_ptr()),
                                    C.c_void_p(r0.data_ptr()), C.c_void_p(ch.data_ptr()),
                                    C.c_void_p(ws.data_ptr()), ws.numel(), _stream_handle(stream))
    _capi.check(rc, "fd jacobian")
    return J, r0, ch


def adjoint_jacobian_device(templates: DeviceSystemBatch, layout: ResidualLayout,
                            host: SystemBatchHost, variables, x0, stream=None):
    """Adjoint Jacobian of runs x0 [runs][P] (DeviceAdjointJacobian::compute).
    Returns device tensors J [runs][P][R], r0 [runs][R], status [runs][rays]."""
    lib = _capi.lib()
    dev = templates.device
    x0 = _x_rows(x0, variables.size, dev)
    runs, P = x0.shape
    R = layout.trace_rows
    b = templates.c_struct()
    plan = layout.plan(host)
    need = int(lib.mkb_adjoint_jacobian_workspace_bytes(C.byref(b), runs))
    ws = torch.empty(max(need, 1), dtype=torch.uint8, device=dev)
    J = torch.empty((runs, P, R), dtype=torch.float64, device=dev)
    r0 = torch.empty((runs, R), dtype=torch.float64, device=dev)
    st = torch.empty((runs, layout.rays_per_variant), dtype=torch.uint8, device=dev)
    vs = variables.c_struct()
    rc = lib.mkb_adjoint_jacobian_device(C.byref(b), C.byref(plan), C.byref(vs),
                                         C.c_void_p(x0.data_ptr()), runs,
                                         C.c_void_p(J.data_ptr()), C.c_void_p(r0.data_ptr()),
                                         C.c_void_p(st.data_ptr()), C.c_void_p(ws.data_ptr()),
                                         ws.numel(), _stream_handle(stream))
    _capi.check(rc, "adjoint jacobian")
    return J, r0, st


def normal_equations_device(J: torch.Tensor, r: torch.Tensor, exact: bool = True, stream=None):
    """gram [runs][P+1][P+1] = [J r]^T [J r] (DeviceNormalEquations::compute)."""
    lib = _capi.lib()
    runs, P, R = J.shape
    gram = torch.empty((runs, P + 1, P + 1), dtype=torch.float64, device=J.device)
    rc = lib.mkb_normal_equations_device(C.c_void_p(J.data_ptr()), C.c_void_p(r.data_ptr()),
                                         runs, P, R, C.c_void_p(gram.data_ptr()), int(exact),
                                         _stream_handle(stream))
    _capi.check(rc, "normal equations")
    return gram


# ---- batched Levenberg-Marquardt (device) -------------------------------------------------
JACOBIAN_FD, JACOBIAN_ADJOINT = 0, 1
LM_STATUS = {0: "running", 1: "converged_merit", 2: "converged_step", 3: "converged_gradient",
             4: "converged_stall", 5: "max_iterations", 6: "damping_limit",
             7: "numerical_error"}


class ExtraResiduals:
    """ExtraResiduals (include/mikroptim/optim/extra_residuals.hpp): `count` residual rows per
    variant after the trace rows (paraxial constraints and the like). evaluate(batch, v, out)
    writes variant v's rows of a SystemBatchHost into out (float64 [count]). The LM takes
    their Jacobian by central differences on the host, with the FD Jacobian's pattern, and adds
    sum_e r_e^2 to every merit (extra_rows_untraced, src/optim/adjoint_jacobian.cpp:245;
    extra_merit_values, src/optim/levenberg_marquardt.cpp:659)."""

    def __init__(self, count: int = 0, evaluate=None):
        if count < 0 or (count > 0 and evaluate is None):
            raise ValueError("ExtraResiduals: count >= 0 and an evaluate function needed")
        self.count = count
        self.evaluate = evaluate


class TraceExtraResiduals:
    """TraceExtraResiduals (include/mikroptim/optim/trace_extra_residuals.hpp): `count` rows per
    variant after the ExtraResiduals rows, computed from the per-surface extrema of the same
    trace (largest ray height, smallest cos I: semi-diameter and incidence-angle constraints).
    evaluate(batch, v, extrema, out) gets variant v's extrema [S][2] (hard maxima). The LM
    traces every FD point with extrema to differentiate them and adds sum t^2 to each merit
    after the MERIT kernel's sum (GpuLmBackend::merit, src/cuda/levenberg_marquardt.cpp:235)."""

    def __init__(self, count: int = 0, evaluate=None):
        if count < 0 or (count > 0 and evaluate is None):
            raise ValueError("TraceExtraResiduals: count >= 0 and an evaluate function needed")
        self.count = count
        self.evaluate = evaluate


def extra_rows_host(host: SystemBatchHost, variables, x0, extra: ExtraResiduals):
    """The caller's extra rows at run points x0 [runs][P] on the host (extra_rows_untraced,
    src/optim/adjoint_jacobian.cpp:245): per run, a one-variant copy of its template (`host`
    holds 1 variant or one per run), the values r at x and J [P][E] by central differences with
    the FD Jacobian's pattern (each point applied in full, as the reference does). Returns
    J [runs][P][E], r [runs][E]."""
    lib = _capi.lib()
    P, E = variables.size, extra.count
    x0 = np.ascontiguousarray(x0, dtype=np.float64).reshape(-1, P)
    runs = x0.shape[0]
    J = np.zeros((runs, P, E))
    R = np.zeros((runs, E))
    vc = variables.c_struct()
    for i in range(runs):
        one = host.subset(0 if host.variants == 1 else i, 1)

        def evaluate(y):
            variables.apply(one, 0, y)
            out = np.zeros(E)
            extra.evaluate(one, 0, out)
            return out

        x = x0[i].copy()
        xp, xm, dp, dm = (np.zeros(P) for _ in range(4))
        st = np.zeros(P, dtype=np.int32)
        _capi.check(lib.mkb_fd_pattern_host(C.byref(vc), _capi.ptr(x), 1, _capi.ptr(xp),
                                            _capi.ptr(xm), _capi.ptr(dp), _capi.ptr(dm),
                                            _capi.ptr(st, C.c_int32)), "fd pattern")
        y = x.copy()
        r0 = evaluate(y)
        R[i] = r0
        for k in range(P):
            y[k] = xp[k]
            ra = evaluate(y)
            y[k] = xm[k]
            rb = evaluate(y)
            y[k] = x[k]
            col = np.zeros(E)
            _capi.check(lib.mkb_fd_derivative_host(int(st[k]), float(dp[k]), float(dm[k]), E,
                                                   _capi.ptr(r0), _capi.ptr(ra), _capi.ptr(rb),
                                                   _capi.ptr(col)), "fd derivative")
            J[i, k] = col
    return J, R


CONSTRAINT_FOCAL_LENGTH, CONSTRAINT_PARFOCAL_LENGTH, CONSTRAINT_WORKING_DISTANCE = 0, 1, 2
CONSTRAINT_PARAXIAL_FOCUS, CONSTRAINT_PETZVAL = 3, 4
MODE_EQUAL, MODE_MIN, MODE_MAX = 0, 1, 2


@dataclass
class ParaxialConstraint:
    """ParaxialConstraint (include/mikroptim/optim/paraxial_residuals.hpp:67): type and mode
    as ConstraintType / ConstraintMode, r = sqrt(weight) * mode(q + shift)."""

    type: int
    mode: int = MODE_EQUAL
    weight: float = 1.0
    target: float = 0.0
    reference_surface: int = 0
    offset: float = 0.0
    shift: float = 0.0


@dataclass
class ParaxialConstraints:
    """Paraxial constraints evaluated on the device as the LM's extra rows (no host phase):
    `column` is the wavelength column holding the paraxial index (the batch's paraxial_index),
    `derivative` "fd" (central differences with the FD pattern, the reference's extra rows bit
    for bit) or "adjoint" (analytic reverse sweep of the y-nu trace)."""

    items: list = dataclasses.field(default_factory=list)
    column: int = 0
    derivative: str = "fd"

    @staticmethod
    def of(tuples, column: int = 0, derivative: str = "fd") -> "ParaxialConstraints":
        """From (type, mode, weight, target) tuples."""
        return ParaxialConstraints([ParaxialConstraint(int(t[0]), int(t[1]), float(t[2]),
                                                       float(t[3])) for t in tuples],
                                   column, derivative)

    def c_array(self):
        arr = (_capi.ParaxialConstraint * len(self.items))()
        for i, c in enumerate(self.items):
            arr[i] = _capi.ParaxialConstraint(c.type, c.mode, c.weight, c.target,
                                               c.reference_surface, 0, c.offset, c.shift)
        return arr


def paraxial_rows_device(templates: DeviceSystemBatch, layout: ResidualLayout,
                         host: SystemBatchHost, variables, x0,
                         constraints: ParaxialConstraints, stream=None):
    """The paraxial constraint rows of every run at x0 on the device: (Jacobian [runs][P][E],
    residuals [runs][E]), by central differences with the FD pattern or by the analytic adjoint
    (constraints.derivative)."""
    lib = _capi.lib()
    dev = templates.device
    x = _x_rows(x0, variables.size, dev)
    runs, P = x.shape
    E = len(constraints.items)
    je = torch.zeros((runs, P, E), dtype=torch.float64, device=dev)
    re = torch.zeros((runs, E), dtype=torch.float64, device=dev)
    opt = LmOptions(paraxial=constraints).c_struct()
    b = templates.c_struct()
    plan = layout.plan(host)
    vs = variables.c_struct()
    rc = lib.mkb_paraxial_rows_device(C.byref(b), C.byref(plan), C.byref(vs), C.byref(opt),
                                      C.c_void_p(x.data_ptr()), runs, C.c_void_p(je.data_ptr()),
                                      C.c_void_p(re.data_ptr()), _stream_handle(stream))
    _capi.check(rc, "paraxial rows")
    return je, re


@dataclass
class LmOptions:
    """LmOptions (include/mikroptim/optim/levenberg_marquardt.hpp:85). fail_weight_factor and
    max_fail_weight drive the outer soft-failure penalty rounds of optimize_lm_gpu
    (optimize_lm_rounds, src/optim/levenberg_marquardt.cpp:891); a factor <= 1 gives one pass.
    extra / trace_extra: the caller's extra residual rows (LmOptions::jacobian.extra and
    ::jacobian.trace_extra), or None."""

    max_iterations: int = 100
    ftol: float = 1e-10
    xtol: float = 1e-10
    gtol: float = 1e-10
    initial_damping: float = 1e-3
    max_damping: float = 1e16
    diag_floor: float = 1e-12
    reject_new_failures: bool = True
    jacobian: int = JACOBIAN_ADJOINT
    gram_exact: bool = True
    fail_weight_factor: float = 10.0
    max_fail_weight: float = 1e14
    extra: ExtraResiduals | None = None
    trace_extra: TraceExtraResiduals | None = None
    paraxial: "ParaxialConstraints | None" = None

    def c_struct(self) -> "_capi.LmOptions":
        o = _capi.LmOptions()
        o.max_iterations = self.max_iterations
        o.reject_new_failures = int(self.reject_new_failures)
        o.ftol, o.xtol, o.gtol = self.ftol, self.xtol, self.gtol
        o.initial_damping, o.max_damping = self.initial_damping, self.max_damping
        o.diag_floor = self.diag_floor
        o.jacobian = self.jacobian
        o.gram_exact = int(self.gram_exact)
        o.per_run_variables = 0
        if self.paraxial is not None and self.paraxial.items:
            arr = self.paraxial.c_array()
            o._keep_paraxial = arr
            o.paraxial_count = len(self.paraxial.items)
            o.paraxial = C.cast(arr, C.POINTER(_capi.ParaxialConstraint))
            o.paraxial_column = self.paraxial.column
            o.paraxial_derivative = (_capi.MKB_PARAXIAL_ADJOINT
                                     if self.paraxial.derivative == "adjoint"
                                     else _capi.MKB_PARAXIAL_FD)
        return o


def pad_rows(x, runs: int, width: int) -> np.ndarray:
    """[runs][width] float64 rows: a 2-D array as it is, or a list of rows padded with zeros."""
    if isinstance(x, (list, tuple)):
        out = np.zeros((runs, width))
        for i, row in enumerate(x):
            out[i, :len(row)] = row
        return out
    return np.asarray(x, dtype=np.float64).reshape(runs, width)


def check_start_points(variables, x0: np.ndarray, run_variables=None) -> None:
    """The reference rejects a start value outside its variable's bounds before any work
    (VariableSet validation in levenberg_marquardt, std::invalid_argument): ValueError. With
    run_variables (the RunVariables of a per-run list) the check runs on whole arrays."""
    if run_variables is not None:
        lo, up = run_variables.bounds()
        x = np.asarray(x0, dtype=np.float64)[:, :run_variables.pmax]
        bad = (x < lo) | (x > up)
        if bad.any():
            i = int(np.nonzero(bad.any(axis=1))[0][0])
            k = int(np.nonzero(bad[i])[0][0])
            raise ValueError(f"lm: run {i}, variable {k}: start value {x[i, k]!r} outside "
                             f"[{lo[i, k]!r}, {up[i, k]!r}]")
        return
    sets = variables if isinstance(variables, (list, tuple)) else [variables] * len(x0)
    for i, (vs, row) in enumerate(zip(sets, x0)):
        lo, up = vs.lower(), vs.upper()
        x = row[:vs.size]
        bad = np.nonzero((x < lo) | (x > up))[0]
        if bad.size:
            k = int(bad[0])
            raise ValueError(f"lm: run {i}, variable {k}: start value {x[k]!r} outside "
                             f"[{lo[k]!r}, {up[k]!r}]")


class DeviceLm:
    """Batched LM state on the device: start(x0), cycle(), results(). One object per problem;
    the workspace is allocated once and reused by every cycle.

    `variables` is one VariableSet for all runs, or a list of one VariableSet per run (uneven
    batches: the counts may differ; x0 / x rows are then padded to the largest count)."""

    def __init__(self, templates: DeviceSystemBatch, layout: ResidualLayout,
                 host: SystemBatchHost, variables, options: LmOptions, runs: int,
                 stream=None):
        self.lib = _capi.lib()
        self.templates, self.layout, self.host = templates, layout, host
        self.variables, self.options, self.runs = variables, options, runs
        self.stream = stream
        self._b = templates.c_struct()
        self._plan = layout.plan(host)
        self._opt = options.c_struct()
        if isinstance(variables, (list, tuple)):
            if len(variables) != runs:
                raise ValueError("DeviceLm: one VariableSet per run needed")
            self._run_vars = RunVariables(variables)
            self.P = self._run_vars.pmax
            self._vars = self._run_vars.pointer.contents
            self._opt.per_run_variables = 1
        else:
            self._run_vars = None
            self.P = variables.size
            self._vars = variables.c_struct()
        need = int(self.lib.mkb_lm_workspace_bytes(C.byref(self._b), C.byref(self._plan),
                                                   C.byref(self._vars), C.byref(self._opt),
                                                   runs))
        if need == 0:
            raise ValueError(f"lm: {self.lib.mkb_last_error().decode()}")
        self.workspace = torch.empty(need, dtype=torch.uint8, device=templates.device)
        self.cycles = 0

    def _args(self):
        return (C.byref(self._b), C.byref(self._plan), C.byref(self._vars), C.byref(self._opt))

    def start(self, x0) -> None:
        rows = pad_rows(x0, self.runs, self.P)
        check_start_points(self.variables, rows, self._run_vars)
        x0 = _dev_f64(rows, self.templates.device)
        self._x0 = x0
        extra = tmerit = None
        if self._plain_rows():
            extra = _dev_f64([self._extra_merit(i, rows[i]) for i in range(self.runs)],
                             self.templates.device)
        if self._trace_rows():
            tmerit = _dev_f64(self._trace_merits([(i, rows[i]) for i in range(self.runs)]),
                              self.templates.device)
        rc = self.lib.mkb_lm_start_ex_device(
            *self._args(), C.c_void_p(x0.data_ptr()),
            C.c_void_p(extra.data_ptr()) if extra is not None else None,
            C.c_void_p(tmerit.data_ptr()) if tmerit is not None else None, self.runs,
            C.c_void_p(self.workspace.data_ptr()), self.workspace.numel(),
            _stream_handle(self.stream))
        _capi.check(rc, "lm start")

    def cycle(self) -> None:
        if self._extra_rows():
            self._cycle_with_extra_rows()
            return
        rc = self.lib.mkb_lm_cycle_device(*self._args(), self.runs,
                                          C.c_void_p(self.workspace.data_ptr()),
                                          self.workspace.numel(), _stream_handle(self.stream))
        _capi.check(rc, "lm cycle")
        self.cycles += 1

    # ---- the caller's extra rows (evaluated on the host) ----------------------------------
    def _plain_rows(self) -> int:
        e = self.options.extra
        return e.count if e is not None else 0

    def _trace_rows(self) -> int:
        t = self.options.trace_extra
        return t.count if t is not None else 0

    def _extra_rows(self) -> int:
        return self._plain_rows() + self._trace_rows()

    def _var_set(self, i: int):
        return self.variables[i] if isinstance(self.variables, (list, tuple)) else self.variables

    def _template(self, i: int) -> int:
        return 0 if self.host.variants == 1 else i

    def _work_batch(self, i: int) -> SystemBatchHost:
        """A one-variant copy of run i's template (the reference's working variant)."""
        cache = self.__dict__.setdefault("_work", {})
        t = self._template(i)
        if t not in cache:
            cache[t] = self.host.subset(t, 1)
        return cache[t]

    def _evaluate(self, i: int, y) -> np.ndarray:
        one = self._work_batch(i)
        self._var_set(i).apply(one, 0, np.asarray(y, dtype=np.float64))
        out = np.zeros(self.options.extra.count)
        self.options.extra.evaluate(one, 0, out)
        return out

    @staticmethod
    def _sum_squares(values) -> float:
        s = 0.0
        for e in values:
            s = s + e * e
        return s

    def _extra_merit(self, i: int, x_row) -> float:
        """sum_e r_e^2 in row order, each product and sum rounded (extra_merit_values)."""
        if not self._plain_rows():
            return 0.0
        return self._sum_squares(self._evaluate(i, x_row[:self._var_set(i).size]))

    def _points_extrema(self, pts, invalid=None) -> tuple[SystemBatchHost, np.ndarray]:
        """The batch of the points [(run, y)] and their extrema [n][S][2] from one MERIT trace
        (FD points and trial points alike). A point whose system is not valid (a glass step
        that drives an index to <= 0, say) is traced at its template instead and marked in
        `invalid` (a bool array the caller passes), so one bad trial point cannot stop the
        batch."""
        multi = self.host.take([self._template(i) for i, _ in pts])
        keep = self.host.take([self._template(i) for i, _ in pts])
        for j, (i, y) in enumerate(pts):
            vs = self._var_set(i)
            vs.apply(multi, j, np.asarray(y[:vs.size], dtype=np.float64))
        bad = ~np.all(multi.index.reshape(len(pts), -1) > 0, axis=1)
        bad |= ~np.all(np.isfinite(multi.curvature) & np.isfinite(multi.thickness), axis=1)
        if np.any(bad):
            for name in ("curvature", "thickness", "index", "pupil_radius"):
                getattr(multi, name)[bad] = getattr(keep, name)[bad]
            if multi.buchdahl_coeff is not None:
                multi.buchdahl_coeff[bad] = keep.buchdahl_coeff[bad]
        if invalid is not None:
            invalid[:] = bad
        elif np.any(bad):
            raise ValueError("LM: a difference point of the trace-dependent rows is not a valid "
                             "system")
        eng = self.__dict__.setdefault("_engine", TraceEngine(self.templates.device.index or 0))
        out = eng.run(multi, TraceMode.MERIT, TraceSettings(self.layout.settings, extrema=True))
        return multi, out.merit.extrema

    def _trace_values(self, multi, ext, j: int) -> np.ndarray:
        out = np.zeros(self._trace_rows())
        self.options.trace_extra.evaluate(multi, j, ext[j], out)
        return out

    def _trace_merits(self, pts) -> np.ndarray:
        """sum_i t_i^2 at the points [(run, y)] (trace_extra_merit)."""
        if not pts:
            return np.zeros(0)
        invalid = np.zeros(len(pts), dtype=bool)
        multi, ext = self._points_extrema(pts, invalid)
        # an invalid trial point gets an infinite merit: the LM rejects the step
        return np.array([math.inf if invalid[j] else
                         self._sum_squares(self._trace_values(multi, ext, j))
                         for j in range(len(pts))])

    def _extra_jacobian(self, i: int, x_row) -> tuple[np.ndarray, np.ndarray]:
        """J [P][E + E_t] and r [E + E_t] of run i at x: the ExtraResiduals rows, then the
        trace-dependent rows, by central differences with the FD Jacobian's pattern
        (extra_rows_cpu, src/optim/adjoint_jacobian.cpp:300)."""
        vs = self._var_set(i)
        P = vs.size
        x = np.ascontiguousarray(x_row[:P], dtype=np.float64)
        parts_J, parts_r = [], []
        if self._plain_rows():
            J, r = extra_rows_host(self.host.subset(self._template(i), 1), vs, x,
                                   self.options.extra)
            parts_J.append(J[0])
            parts_r.append(r[0])
        Et = self._trace_rows()
        if Et:
            xp, xm, dp, dm = (np.zeros(P) for _ in range(4))
            st = np.zeros(P, dtype=np.int32)
            vc = vs.c_struct()
            _capi.check(self.lib.mkb_fd_pattern_host(
                C.byref(vc), _capi.ptr(x), 1, _capi.ptr(xp), _capi.ptr(xm), _capi.ptr(dp),
                _capi.ptr(dm), _capi.ptr(st, C.c_int32)), "fd pattern")
            pts = [(i, x)]
            for k in range(P):
                for val in (xp[k], xm[k]):
                    y = x.copy()
                    y[k] = val
                    pts.append((i, y))
            multi, ext = self._points_extrema(pts)
            vals = [self._trace_values(multi, ext, j) for j in range(len(pts))]
            J = np.zeros((P, Et))
            for k in range(P):
                col = np.zeros(Et)
                _capi.check(self.lib.mkb_fd_derivative_host(
                    int(st[k]), float(dp[k]), float(dm[k]), Et, _capi.ptr(vals[0]),
                    _capi.ptr(vals[1 + 2 * k]), _capi.ptr(vals[2 + 2 * k]), _capi.ptr(col)),
                    "fd derivative")
                J[k] = col
            parts_J.append(J)
            parts_r.append(vals[0])
        return np.concatenate(parts_J, axis=1), np.concatenate(parts_r)

    def _points(self, want: bool):
        flags = np.zeros(self.runs, dtype=np.int32)
        rows = np.zeros((self.runs, self.P))
        torch.cuda.synchronize(self.templates.device)
        args = [None] * 4
        if want:
            args[0], args[1] = _capi.ptr(flags, C.c_int32), _capi.ptr(rows)
        else:
            args[2], args[3] = _capi.ptr(flags, C.c_int32), _capi.ptr(rows)
        rc = self.lib.mkb_lm_points_device(*self._args(), self.runs,
                                           C.c_void_p(self.workspace.data_ptr()), *args,
                                           _stream_handle(self.stream))
        _capi.check(rc, "lm points")
        torch.cuda.synchronize(self.templates.device)
        return flags, rows

    def _cycle_with_extra_rows(self) -> None:
        E = self._extra_rows()
        ws = (C.c_void_p(self.workspace.data_ptr()), self.workspace.numel())
        h = _stream_handle(self.stream)
        dev = self.templates.device
        _capi.check(self.lib.mkb_lm_cycle_jacobian_device(*self._args(), self.runs, *ws, h),
                    "lm cycle (Jacobian)")
        want, x = self._points(True)
        je = np.zeros((self.runs, self.P, E))
        re = np.zeros((self.runs, E))
        for i in np.nonzero(want)[0]:
            J, r = self._extra_jacobian(int(i), x[i])
            je[i, :J.shape[0]] = J
            re[i] = r
        je_d, re_d = _dev_f64(je, dev), _dev_f64(re, dev)
        _capi.check(self.lib.mkb_lm_extra_rows_device(
            *self._args(), self.runs, *ws, C.c_void_p(je_d.data_ptr()),
            C.c_void_p(re_d.data_ptr()), E, h), "lm extra rows")
        _capi.check(self.lib.mkb_lm_cycle_step_device(*self._args(), self.runs, *ws, h),
                    "lm cycle (step)")
        evaluate, trial = self._points(False)
        em = np.zeros(self.runs)
        for i in np.nonzero(evaluate)[0]:
            em[i] = self._extra_merit(int(i), trial[i])
        em_d = _dev_f64(em, dev)
        if not self._trace_rows():
            _capi.check(self.lib.mkb_lm_cycle_accept_device(*self._args(), self.runs, *ws,
                                                            C.c_void_p(em_d.data_ptr()), h),
                        "lm cycle (acceptance)")
        else:
            # the trace-dependent share needs the trial points' own extrema (the reference
            # takes them from the trial MERIT); they are traced here with the engine
            _capi.check(self.lib.mkb_lm_cycle_trial_device(
                *self._args(), self.runs, *ws, C.c_void_p(em_d.data_ptr()), None, h),
                "lm cycle (trial merit)")
            idx = [int(i) for i in np.nonzero(evaluate)[0]]
            tm = np.zeros(self.runs)
            tm[idx] = self._trace_merits([(i, trial[i]) for i in idx])
            tm_d = _dev_f64(tm, dev)
            _capi.check(self.lib.mkb_lm_cycle_decide_device(
                *self._args(), self.runs, *ws, C.c_void_p(tm_d.data_ptr()), h),
                "lm cycle (acceptance)")
        torch.cuda.synchronize(dev)
        self.cycles += 1

    def capture(self) -> "torch.cuda.CUDAGraph":
        """One LM cycle captured as a CUDA graph: a cycle is a fixed launch sequence whose
        per-run decisions live in device masks, so replaying the graph advances every run by
        one cycle exactly as cycle() does. Call cycle() at least once first (it sets kernel
        attributes outside the capture)."""
        if self._extra_rows():
            raise NotImplementedError("DeviceLm.capture: extra rows are evaluated on the host")
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            rc = self.lib.mkb_lm_cycle_device(*self._args(), self.runs,
                                              C.c_void_p(self.workspace.data_ptr()),
                                              self.workspace.numel(),
                                              _stream_handle(None))
        _capi.check(rc, "lm cycle capture")
        return graph

    def iterations(self) -> np.ndarray:
        """Per-run iteration counters (synchronising)."""
        out = np.zeros(self.runs, dtype=np.int32)
        torch.cuda.synchronize(self.templates.device)
        rc = self.lib.mkb_lm_results_device(*self._args(), self.runs,
                                            C.c_void_p(self.workspace.data_ptr()), None, None,
                                            None, _capi.ptr(out, C.c_int32), *([None] * 7),
                                            _stream_handle(self.stream))
        _capi.check(rc, "lm results")
        torch.cuda.synchronize(self.templates.device)
        return out

    def running(self) -> int:
        out = np.zeros(1, dtype=np.int32)
        torch.cuda.synchronize(self.templates.device)
        rc = self.lib.mkb_lm_results_device(*self._args(), self.runs,
                                            C.c_void_p(self.workspace.data_ptr()),
                                            *([None] * 10), _capi.ptr(out, C.c_int32),
                                            _stream_handle(self.stream))
        _capi.check(rc, "lm results")
        torch.cuda.synchronize(self.templates.device)
        return int(out[0])

    def results(self) -> dict:
        R, P, H = self.runs, self.P, self.options.max_iterations + 1
        out = dict(x=np.zeros((R, P)), merit=np.zeros(R), status=np.zeros(R, np.int32),
                   iterations=np.zeros(R, np.int32), accepted=np.zeros(R, np.int32),
                   jacobians=np.zeros(R, np.int32), damping=np.zeros(R),
                   history=np.zeros((R, H)), failed=np.zeros(R, np.int64),
                   hard_failed=np.zeros(R, np.int64))
        torch.cuda.synchronize(self.templates.device)
        rc = self.lib.mkb_lm_results_device(
            *self._args(), self.runs, C.c_void_p(self.workspace.data_ptr()),
            _capi.ptr(out["x"]), _capi.ptr(out["merit"]), _capi.ptr(out["status"], C.c_int32),
            _capi.ptr(out["iterations"], C.c_int32), _capi.ptr(out["accepted"], C.c_int32),
            _capi.ptr(out["jacobians"], C.c_int32), _capi.ptr(out["damping"]),
            _capi.ptr(out["history"]), _capi.ptr(out["failed"], C.c_int64),
            _capi.ptr(out["hard_failed"], C.c_int64), None, _stream_handle(self.stream))
        _capi.check(rc, "lm results")
        torch.cuda.synchronize(self.templates.device)
        return out


def _lm_pass(batch, layout, variables, x0, options, dev) -> dict:
    """One LM pass of every run on the device (levenberg_marquardt with GpuLmBackend)."""
    if isinstance(variables, (list, tuple)):
        runs = len(variables)
        x0 = pad_rows(x0, runs, max(v.size for v in variables))
    else:
        x0 = np.asarray(x0, dtype=np.float64).reshape(-1, variables.size)
        runs = x0.shape[0]
    with torch.cuda.device(dev):
        templates = DeviceSystemBatch(batch, dev)
        lm = DeviceLm(templates, layout, batch, variables, options, runs)
        lm.start(x0)
        if lm._extra_rows():
            while lm.running() > 0:
                lm.cycle()
            cycles = lm.cycles
        else:
            cycles = _run_to_end(lm, options.max_iterations + 1)
        res = lm.results()
        res["cycles"] = cycles
        _device_status()
        return res


def _run_to_end(lm: DeviceLm, max_cycles: int) -> int:
    """Cycles until no run is running (or max_cycles): the first cycle directly (it sets kernel
    attributes outside any capture), the rest as replays of one captured cycle. The count of
    running runs after cycle k is copied to pinned memory and read while cycle k + 1 runs, so the
    host never waits for an idle GPU; the one cycle that may run past the end changes nothing
    (a run that stopped is masked out of every kernel). Returns the cycles that had a running
    run."""
    if lm.running() == 0:
        return 0
    lm.cycle()
    done = 1
    if max_cycles <= 1:
        return done
    stream = torch.cuda.current_stream(lm.templates.device)
    count = torch.zeros(2, dtype=torch.int32).pin_memory()
    ready = [torch.cuda.Event(), torch.cuda.Event()]

    def read_count(slot: int) -> None:
        rc = lm.lib.mkb_lm_results_device(*lm._args(), lm.runs,
                                          C.c_void_p(lm.workspace.data_ptr()),
                                          *([None] * 10),
                                          C.c_void_p(count.data_ptr() + 4 * slot),
                                          _stream_handle(stream))
        _capi.check(rc, "lm results")
        ready[slot].record(stream)

    read_count(0)
    graph = lm.capture()
    try:
        pending = 0  # slot holding the count after the last cycle enqueued before this one
        while done < max_cycles:
            graph.replay()
            lm.cycles += 1
            read_count(1 - pending)
            ready[pending].synchronize()
            if int(count[pending]) == 0:
                break  # the cycle just enqueued found nothing running
            done += 1
            pending = 1 - pending
        torch.cuda.synchronize(lm.templates.device)
    finally:
        del graph
    return done


LM_NUMERICAL_ERROR = 7  # LmStatus::NumericalError


def optimize_lm_gpu(batch: SystemBatchHost, layout: ResidualLayout, variables, x0,
                    options: LmOptions | None = None, device: int = 0) -> dict:
    """optimize_lm_gpu (include/mikroptim/cuda/levenberg_marquardt.hpp): batched LM of the runs
    x0 [runs][P] on `batch` (1 variant for all runs or one per run). `variables` may be a list
    of one VariableSet per run (uneven batches; x0 rows padded).

    In soft-failure mode the outer penalty rounds follow (optimize_lm_rounds,
    src/optim/levenberg_marquardt.cpp:891): runs that end with failed rays (and not in
    NumericalError) restart together from their end point with fail_weight times
    fail_weight_factor, as long as the weight stays <= max_fail_weight. Per run: x, merit,
    failed rays, status and damping of the last round; iterations, accepted steps and Jacobians
    summed; the merit histories of the rounds joined (padded with NaN); fail_weight and
    penalty_rounds."""
    options = options or LmOptions()
    dev = _require_cuda(f"cuda:{device}")
    res = _lm_pass(batch, layout, variables, x0, options, dev)
    runs = res["x"].shape[0]
    weight = layout.settings.fail_weight
    res["fail_weight"] = np.full(runs, weight)
    res["penalty_rounds"] = np.ones(runs, np.int32)
    histories = [[h[~np.isnan(h)]] for h in res["history"]]
    if not (layout.settings.failure == FAILURE_SOFT and options.fail_weight_factor > 1.0 and
            weight > 0.0):
        return res
    per_run = isinstance(variables, (list, tuple))
    while True:
        weight *= options.fail_weight_factor
        if not weight <= options.max_fail_weight:
            break
        again = [i for i in range(runs)
                 if res["failed"][i] > 0 and res["status"][i] != LM_NUMERICAL_ERROR]
        if not again:
            break
        tmpl = batch if batch.variants == 1 else batch.take(again)
        lay = ResidualLayout(layout.topology, dataclasses.replace(layout.settings,
                                                                  fail_weight=weight))
        vars_again = [variables[i] for i in again] if per_run else variables
        part = _lm_pass(tmpl, lay, vars_again, res["x"][again], options, dev)
        for j, i in enumerate(again):
            for k in ("x", "merit", "failed", "hard_failed", "status", "damping"):
                res[k][i] = part[k][j]
            for k in ("iterations", "accepted", "jacobians"):
                res[k][i] += part[k][j]
            h = part["history"][j]
            histories[i].append(h[~np.isnan(h)])
            res["fail_weight"][i] = weight
            res["penalty_rounds"][i] += 1
        res["cycles"] += part["cycles"]
    joined = [np.concatenate(h) for h in histories]
    width = max(res["history"].shape[1], max(len(h) for h in joined))
    res["history"] = np.full((runs, width), np.nan)
    for i, h in enumerate(joined):
        res["history"][i, :len(h)] = h
    return res


def adjoint_normal_equations_device(templates: DeviceSystemBatch, layout: ResidualLayout,
                                    host: SystemBatchHost, variables, x0, stream=None):
    """Fused adjoint + normal equations (FP64_FMA, DMMA): gram [runs][P+1][P+1]."""
    lib = _capi.lib()
    dev = templates.device
    x0 = _x_rows(x0, variables.size, dev)
    runs, P = x0.shape
    b = templates.c_struct()
    plan = layout.plan(host)
    need = int(lib.mkb_adjoint_jacobian_workspace_bytes(C.byref(b), runs))
    ws = torch.empty(max(need, 1), dtype=torch.uint8, device=dev)
    gram = torch.empty((runs, P + 1, P + 1), dtype=torch.float64, device=dev)
    vs = variables.c_struct()
    rc = lib.mkb_adjoint_normal_equations_device(C.byref(b), C.byref(plan), C.byref(vs),
                                                 C.c_void_p(x0.data_ptr()), runs,
                                                 C.c_void_p(gram.data_ptr()),
                                                 C.c_void_p(ws.data_ptr()), ws.numel(),
                                                 _stream_handle(stream))
    _capi.check(rc, "adjoint normal equations")
    return gram


class RunVariables:
    """One VariableSet per run as the C array the ABI takes (built once, reused): every run's
    variable fields in flat arrays, and one mkb_variables record per run pointing into them (a
    structured array laid out as the C struct), so thousands of runs take milliseconds."""

    def __init__(self, variable_sets):
        self.sets = list(variable_sets)
        self.runs = len(self.sets)
        counts = np.fromiter((v.size for v in self.sets), dtype=np.int64, count=self.runs)
        self.pmax = int(counts.max()) if self.runs else 0
        flat = [var for v in self.sets for var in v.variables]
        n = len(flat)

        def column(attr, dtype):
            return np.fromiter((getattr(x, attr) for x in flat), dtype=dtype, count=n)
        self.fields = {"type": column("type", np.int32), "surface": column("surface", np.int32),
                       "lower": column("lower", np.float64), "upper": column("upper", np.float64),
                       "typical": column("typical", np.float64),
                       "ghost_plate": column("plate", np.int32),
                       "ghost_order": column("order", np.int32),
                       "glass_component": column("component", np.int32)}
        starts = np.zeros(self.runs, dtype=np.int64)
        if self.runs > 1:
            starts[1:] = np.cumsum(counts)[:-1]
        self.counts, self.starts = counts, starts
        rec = _capi.Variables
        names = [f[0] for f in rec._fields_]
        layout = np.dtype({"names": names,
                           "formats": [np.int32] + [np.uint64] * (len(names) - 1),
                           "offsets": [getattr(rec, f).offset for f in names],
                           "itemsize": C.sizeof(rec)})
        self._array = np.zeros(max(self.runs, 1), dtype=layout)
        self._array["count"][:self.runs] = counts
        for name, a in self.fields.items():
            self._array[name][:self.runs] = a.ctypes.data + starts * a.itemsize
        self.pointer = C.cast(self._array.ctypes.data, C.POINTER(rec))

    def bounds(self):
        """(lower, upper) padded to [runs][pmax] with -inf / +inf past each run's count."""
        k = np.arange(self.pmax)[None, :]
        valid = k < self.counts[:, None]
        idx = np.where(valid, self.starts[:, None] + k, 0)
        if self.fields["lower"].size == 0:
            full = np.zeros((self.runs, self.pmax))
            return full - np.inf, full + np.inf
        lo = np.where(valid, self.fields["lower"][idx], -np.inf)
        up = np.where(valid, self.fields["upper"][idx], np.inf)
        return lo, up


def adjoint_normal_equations_runs_device(templates: DeviceSystemBatch, layout: ResidualLayout,
                                         host: SystemBatchHost, variable_sets, x0,
                                         stream=None, workspace: torch.Tensor | None = None):
    """Fused adjoint + normal equations of an uneven batch: one VariableSet per run (a list or
    a RunVariables), x0 rows padded to the largest P. Returns gram [runs][Pmax+1][Pmax+1]; run
    i's (P_i+1)^2 matrix is dense at the start of its slot (see gram_block)."""
    lib = _capi.lib()
    dev = templates.device
    rv = variable_sets if isinstance(variable_sets, RunVariables) else RunVariables(variable_sets)
    runs, pmax = rv.runs, rv.pmax
    x = x0 if isinstance(x0, torch.Tensor) else _dev_f64(pad_rows(x0, runs, pmax), dev)
    b = templates.c_struct()
    plan = layout.plan(host)
    pv = rv.pointer
    need = int(lib.mkb_adjoint_normal_equations_runs_workspace_bytes(C.byref(b), pv, runs))
    ws = workspace if workspace is not None and workspace.numel() >= need else \
        torch.empty(max(need, 1), dtype=torch.uint8, device=dev)
    gram = torch.zeros((runs, pmax + 1, pmax + 1), dtype=torch.float64, device=dev)
    rc = lib.mkb_adjoint_normal_equations_runs_device(C.byref(b), C.byref(plan), pv,
                                                      C.c_void_p(x.data_ptr()), runs,
                                                      C.c_void_p(gram.data_ptr()),
                                                      C.c_void_p(ws.data_ptr()), ws.numel(),
                                                      _stream_handle(stream))
    _capi.check(rc, "adjoint normal equations (runs)")
    return gram


def gram_block(gram: torch.Tensor, run: int, P: int) -> torch.Tensor:
    """Run `run`'s (P+1) x (P+1) matrix from a gram of stride (Pmax+1)^2 per run."""
    return gram[run].reshape(-1)[:(P + 1) * (P + 1)].reshape(P + 1, P + 1)
