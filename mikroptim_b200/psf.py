"""Scalar PSF, MTF and Strehl from EVAL OPD maps (include/mikroptim/eval/psf.hpp and
include/mikroptim/cuda/psf.hpp of the reference).

The device work -- pupil function, 2-D FFT, intensity, centred PSF, MTF cuts -- runs in
``mkb_psf_device`` (csrc/psf.cu, this library's own shared-memory FFT); the pupil maps, the NA
of the pupil imaging and the per-tuple figures (``finish_psf``) are host steps as in the
reference (make_psf_pupil, finish_psf, src/eval/psf.cpp:196,290), the latter two through the
C ABI so that the Python and C++ layers share them. ``psf_from_eval_device`` keeps the whole
EVAL -> PSF chain on the device (maps built from EVAL's device outputs).
"""

from __future__ import annotations

import ctypes as C
import os
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass

import numpy as np
import torch

from . import _capi
from .batch import SystemBatchHost
from .engine import EngineOptions, EvalResult, _require_cuda, _stream_handle

MAX_PSF_FFT = 8192
BESSEL_J1_FIRST_ZERO = 3.8317059702075123


@dataclass
class PsfSettings:
    """PsfSettings (psf.hpp:33): zero-padding factor Q (M = smallest power of two >= max(2N,
    ceil(Q N))) and a given NA of the pupil imaging (> 0), or 0: from the field rays."""

    padding: float = 4.0
    numerical_aperture: float = 0.0


def check_psf_settings(s: PsfSettings) -> None:
    if not (s.padding >= 2.0) or not np.isfinite(s.padding):
        raise ValueError("PSF: zero-padding factor must be >= 2")
    if not (s.numerical_aperture >= 0.0) or not np.isfinite(s.numerical_aperture):
        raise ValueError("PSF: the given NA must be >= 0 (0: from the field rays)")


def psf_fft_size(grid: int, padding: float) -> int:
    """psf_fft_size (src/eval/psf.cpp:168)."""
    m = C.c_int32(0)
    _capi.check(_capi.lib().mkb_psf_fft_size_host(int(grid), float(padding), C.byref(m)),
                "psf fft size")
    return int(m.value)


@dataclass
class PsfPupil:
    """PsfPupil (psf.hpp:57): the tuple's OPD map after piston [N*N] (opd[j N + i], NaN: no
    transmission), the NA of the pupil imaging per axis and the mirror flags of a divergent
    wave."""

    field: int
    wavelength: int
    grid: int
    full_count: int
    wavelength_nm: float
    na_x: float
    na_y: float
    flip_x: bool
    flip_y: bool
    opd: np.ndarray

    @property
    def wavelength_mm(self) -> float:
        return self.wavelength_nm * 1e-6


@dataclass
class PsfResult:
    """PsfResult (psf.hpp:95): psf [M*M] (psf[j M + i] at ((i - M/2) dx, (j - M/2) dy) from the
    ideal image point, 1 = peak of the unaberrated full pupil), MTF cuts k = 0 .. N at
    f = k f_c / N, and the figures of finish_psf."""

    field: int
    wavelength: int
    grid: int
    fft_size: int
    wavelength_nm: float
    na_x: float
    na_y: float
    dx: float = 0.0
    dy: float = 0.0
    airy_radius: float = 0.0
    psf: np.ndarray | None = None
    mtf_sagittal: np.ndarray | None = None
    mtf_tangential: np.ndarray | None = None
    transmitted: int = 0
    energy: float = float("nan")
    strehl_fft: float = float("nan")
    strehl_origin: float = float("nan")
    strehl: float = float("nan")
    reference_x: float = float("nan")
    reference_y: float = float("nan")
    peak: float = float("nan")
    peak_x: float = float("nan")
    peak_y: float = float("nan")

    def psf_at(self, i: int, j: int) -> float:
        return float(self.psf[j * self.fft_size + i])

    def cutoff_x(self) -> float:
        return 2.0 * self.na_x / (self.wavelength_nm * 1e-6)

    def cutoff_y(self) -> float:
        return 2.0 * self.na_y / (self.wavelength_nm * 1e-6)

    @staticmethod
    def _mtf_at(mtf: np.ndarray, nu: float) -> float:
        if mtf is None or len(mtf) == 0 or not (nu >= 0.0):
            return float("nan")
        n = float(len(mtf) - 1)
        x = nu * n
        if x >= n:
            return 0.0 if nu > 1.0 else float(mtf[-1])
        k = int(x)
        t = x - k
        return (1.0 - t) * float(mtf[k]) + t * float(mtf[k + 1])

    def mtf_sagittal_at(self, nu: float) -> float:
        return self._mtf_at(self.mtf_sagittal, nu)

    def mtf_tangential_at(self, nu: float) -> float:
        return self._mtf_at(self.mtf_tangential, nu)


def grid_cells(result: EvalResult) -> tuple[np.ndarray, np.ndarray, int, bool]:
    """Column i and row j of every grid point of an EVAL result (x = (2i + 1 - N)/N), the
    number of points of the full pupil and whether the grid is a half pupil."""
    pts = result.grid
    n = _grid_size(result)
    col = np.rint((pts[:, 0] * n + n - 1) / 2.0).astype(np.int32)
    row = np.rint((pts[:, 1] * n + n - 1) / 2.0).astype(np.int32)
    a = 2 * np.arange(n, dtype=np.int64) + 1 - n
    full = int(np.count_nonzero(a[:, None] ** 2 + a[None, :] ** 2 <= n * n))
    return col, row, full, bool(result.half_pupil)


def _grid_size(result: EvalResult) -> int:
    if not result.grid_size:
        raise ValueError("PSF: the EVAL result carries no grid edge")
    return int(result.grid_size)


def eval_opd_map(result: EvalResult, v: int, f: int, l: int) -> np.ndarray:
    """eval_opd_map with piston removal (src/eval/eval.cpp:512): the N*N map, NaN outside the
    pupil and for rays whose status is not Ok, the half pupil mirrored to x < 0."""
    if not (0 <= v < result.variants):
        raise IndexError(f"EVAL: variant {v} does not exist")
    if not (0 <= f < result.fields and 0 <= l < result.wavelengths):
        raise IndexError(f"EVAL: tuple ({f}, {l}) does not exist")
    col, row, _, half = grid_cells(result)
    n = _grid_size(result)
    k = result.samples
    t = (v * result.fields + f) * result.wavelengths + l
    opd = result.opd[t * k:(t + 1) * k]
    ok = result.status[t * k:(t + 1) * k] == 0
    m = np.full(n * n, np.nan)
    m[row[ok].astype(np.int64) * n + col[ok]] = opd[ok]
    if half:
        m[row[ok].astype(np.int64) * n + (n - 1 - col[ok])] = opd[ok]
    return m


def make_psf_pupil(batch: SystemBatchHost, result: EvalResult, v: int, f: int, l: int,
                   settings: PsfSettings | None = None) -> PsfPupil:
    """make_psf_pupil (src/eval/psf.cpp:196): the map, and the NA from the field rays with the
    image-space index n' = index[v][S - 1][l] (or the given NA)."""
    settings = settings or PsfSettings()
    check_psf_settings(settings)
    if (batch.variants, batch.fields, batch.wavelengths) != (result.variants, result.fields,
                                                             result.wavelengths):
        raise ValueError("PSF: batch does not match the EVAL result")
    opd = eval_opd_map(result, v, f, l)
    _, _, full, _ = grid_cells(result)
    t = (v * result.fields + f) * result.wavelengths + l
    fr = np.ascontiguousarray(result.field_rays[t * 20:(t + 1) * 20], dtype=np.float64)
    fs = np.ascontiguousarray(result.field_status[t * 4:(t + 1) * 4], dtype=np.uint8)
    na_x, na_y = C.c_double(), C.c_double()
    flip_x, flip_y = C.c_int32(), C.c_int32()
    n_image = float(batch.index[v, batch.surfaces - 1, l])
    _capi.check(_capi.lib().mkb_psf_aperture_host(
        fr.ctypes.data, fs.ctypes.data, n_image, float(result.field_ray_offset),
        float(settings.numerical_aperture), C.byref(na_x), C.byref(na_y), C.byref(flip_x),
        C.byref(flip_y)), f"psf aperture (field {f}, wavelength {l})")
    return PsfPupil(f, l, _grid_size(result), full, float(batch.wavelength_nm[l]), na_x.value,
                    na_y.value, bool(flip_x.value), bool(flip_y.value), opd)


def make_psf_pupils(batch: SystemBatchHost, result: EvalResult, v: int,
                    settings: PsfSettings | None = None) -> list[PsfPupil]:
    """All tuples of variant v, [f L + l]."""
    return [make_psf_pupil(batch, result, v, f, l, settings)
            for f in range(result.fields) for l in range(result.wavelengths)]


def prepare_psf_result(p: PsfPupil, fft_size: int) -> PsfResult:
    if fft_size < 2 * p.grid or fft_size > MAX_PSF_FFT or fft_size & (fft_size - 1):
        raise ValueError(f"PSF: FFT size {fft_size} must be a power of two in [2N, "
                         f"{MAX_PSF_FFT}] (N = {p.grid})")
    if p.opd.size != p.grid * p.grid or p.full_count < 1:
        raise ValueError("PSF: the pupil map does not hold N*N values")
    if not (p.wavelength_nm > 0.0) or not (p.na_x > 0.0 and p.na_y > 0.0):
        raise ValueError("PSF: wavelength and NA must be positive")
    return PsfResult(p.field, p.wavelength, p.grid, fft_size, p.wavelength_nm, p.na_x, p.na_y)


def finish_psf(r: PsfResult, p: PsfPupil) -> None:
    """finish_psf (src/eval/psf.cpp:290) with prepare_psf_result's geometry, on the host."""
    m = _capi.PsfMetrics()
    opd = np.ascontiguousarray(p.opd, dtype=np.float64)
    psf = np.ascontiguousarray(r.psf, dtype=np.float64)
    _capi.check(_capi.lib().mkb_psf_finish_host(
        p.grid, r.fft_size, opd.ctypes.data, p.full_count, p.wavelength_nm, p.na_x, p.na_y,
        int(p.flip_x), int(p.flip_y), psf.ctypes.data, C.byref(m)), "psf finish")
    r.transmitted = int(m.transmitted)
    for k in ("energy", "strehl_fft", "strehl_origin", "strehl", "reference_x", "reference_y",
              "peak", "peak_x", "peak_y", "dx", "dy", "airy_radius"):
        setattr(r, k, float(getattr(m, k)))


def psf_device(maps: torch.Tensor, params: np.ndarray, grid: int, fft_size: int,
               stream=None) -> tuple[torch.Tensor, torch.Tensor]:
    """mkb_psf_device on device maps [T][N][N]: returns psf [T][M][M] and mtf [T][2][N + 1]
    (device tensors). params: host structured array or list of PsfPupilParams."""
    lib = _capi.lib()
    dev = maps.device
    T = maps.shape[0]
    pa = (_capi.PsfPupilParams * max(T, 1))(*params)
    pd = torch.frombuffer(bytearray(pa), dtype=torch.uint8).to(dev)
    psf = torch.empty((T, fft_size, fft_size), dtype=torch.float64, device=dev)
    mtf = torch.empty((T, 2, grid + 1), dtype=torch.float64, device=dev)
    nbytes = int(lib.mkb_psf_workspace_bytes(T, grid, fft_size))
    ws = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=dev)
    _capi.check(lib.mkb_psf_device(T, grid, fft_size, C.c_void_p(maps.data_ptr()),
                                   C.c_void_p(pd.data_ptr()), C.c_void_p(psf.data_ptr()),
                                   C.c_void_p(mtf.data_ptr()), C.c_void_p(ws.data_ptr()),
                                   nbytes, _stream_handle(stream)), "psf")
    return psf, mtf


def pupil_params(p: PsfPupil) -> _capi.PsfPupilParams:
    full = float(p.full_count)
    return _capi.PsfPupilParams(p.wavelength_mm, 1.0 / (full * full), -1 if p.flip_x else 1,
                                -1 if p.flip_y else 1)


@dataclass
class PsfRunInfo:
    """PsfRunInfo (include/mikroptim/cuda/psf.hpp:22); work_bytes: the FFT workspace."""

    pupils: int = 0
    tranche: int = 0
    tranches: int = 0
    work_bytes: int = 0
    device_bytes: int = 0
    budget_bytes: int = 0


class PsfEngine:
    """PsfEngine (include/mikroptim/cuda/psf.hpp:37): PSF, MTF and figures of all pupils of one
    grid edge N with FFT size M, in tranches sized against the device memory (EngineOptions);
    per tranche the maps are uploaded, one mkb_psf_device call runs, PSF and MTF come back and
    finish_psf runs on the host. Buffers are kept across calls."""

    def __init__(self, device: int = 0, options: EngineOptions | None = None):
        self.device = _require_cuda(device)
        self.options = options or EngineOptions()
        self._buf: dict[str, torch.Tensor] = {}
        self.last_run = PsfRunInfo()

    def device_bytes(self) -> int:
        return sum(t.numel() * t.element_size() for t in self._buf.values())

    def release(self) -> None:
        self._buf.clear()

    def _take(self, name: str, count: int, dtype) -> torch.Tensor:
        t = self._buf.get(name)
        if t is None or t.dtype != dtype or t.numel() < count:
            self._buf.pop(name, None)
            t = torch.empty(max(count, 1), dtype=dtype, device=self.device)
            self._buf[name] = t
        return t[:count]

    def _usable(self) -> int:
        free, _ = torch.cuda.mem_get_info(self.device)
        cached = torch.cuda.memory_reserved(self.device) - torch.cuda.memory_allocated(self.device)
        available = int(free) + int(cached) + self.device_bytes()
        if self.options.memory_limit_bytes is not None:
            available = min(available, int(self.options.memory_limit_bytes))
        out = C.c_size_t(0)
        r = self.options.reserve
        _capi.check(_capi.lib().mkb_usable_bytes(int(available), int(r.min_bytes),
                                                  float(r.fraction), C.byref(out)), "reserve")
        return int(out.value)

    @staticmethod
    def tranche_bytes(tuples: int, grid: int, fft_size: int) -> int:
        """Device bytes of a tranche: maps, params, PSF, MTF and the FFT workspace."""
        lib = _capi.lib()
        return (tuples * (grid * grid * 8 + 32 + fft_size * fft_size * 8 + 2 * (grid + 1) * 8) +
                int(lib.mkb_psf_workspace_bytes(tuples, grid, fft_size)))

    def compute(self, pupils, fft_size=None, v: int | None = None,
                settings: PsfSettings | None = None) -> list[PsfResult]:
        """compute(pupils, fft_size) or compute(batch, eval_result, v, settings) (the reference's
        two overloads)."""
        if isinstance(pupils, SystemBatchHost):
            batch, result = pupils, fft_size
            settings = settings or PsfSettings()
            ps = make_psf_pupils(batch, result, v, settings)
            return self.compute(ps, psf_fft_size(_grid_size(result), settings.padding))
        pupils = list(pupils)
        out = []
        for p in pupils:
            if p.grid != pupils[0].grid:
                raise ValueError("PsfEngine: every pupil needs the same grid edge")
            out.append(prepare_psf_result(p, fft_size))
        self.last_run = PsfRunInfo(pupils=len(pupils))
        if not pupils:
            return out
        n, m, count = pupils[0].grid, int(fft_size), len(pupils)
        usable = self._usable()
        tranche = count
        while tranche >= 1 and self.tranche_bytes(tranche, n, m) > usable:
            tranche = max(1, tranche * 3 // 4) if tranche > 1 else 0
        if tranche < 1:
            raise RuntimeError(f"PsfEngine: not one pupil fits the device memory (M = {m})")
        with torch.cuda.device(self.device):
            for first in range(0, count, tranche):
                used = min(tranche, count - first)
                part = pupils[first:first + used]
                host = np.concatenate([np.asarray(p.opd, dtype=np.float64) for p in part])
                maps = self._take("maps", used * n * n, torch.float64)
                maps.copy_(torch.from_numpy(host))
                psf, mtf = psf_device(maps.view(used, n, n), [pupil_params(p) for p in part],
                                      n, m)
                psf_h = psf.cpu().numpy()
                mtf_h = mtf.cpu().numpy()
                for t, p in enumerate(part):
                    r = out[first + t]
                    r.psf = psf_h[t].reshape(-1)
                    r.mtf_sagittal = mtf_h[t, 0].copy()
                    r.mtf_tangential = mtf_h[t, 1].copy()
                # the figures of every tuple on the host threads (the finish runs in the
                # library with the interpreter lock released; each tuple is independent)
                items = [(out[first + t], p) for t, p in enumerate(part)]
                workers = min(len(items), os.cpu_count() or 1)
                if workers > 1:
                    with ThreadPoolExecutor(max_workers=workers) as ex:
                        list(ex.map(lambda rp: finish_psf(*rp), items))
                else:
                    for r, p in items:
                        finish_psf(r, p)
                self.last_run.tranches += 1
        self.last_run.tranche = tranche
        self.last_run.work_bytes = int(_capi.lib().mkb_psf_workspace_bytes(tranche, n, m))
        self.last_run.device_bytes = self.device_bytes()
        self.last_run.budget_bytes = usable
        return out


def psf_from_eval_device(eval_out: dict, tuples: int, grid: int, samples: int, half: bool,
                         column: torch.Tensor, row: torch.Tensor, params, fft_size: int,
                         stream=None) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    """The device EVAL -> PSF chain: maps from EVAL's device OPD and status (mkb_psf_maps_device)
    and mkb_psf_device on them. Returns maps, psf, mtf (device tensors)."""
    lib = _capi.lib()
    opd, status = eval_out["opd"], eval_out["st"]
    maps = torch.empty((tuples, grid, grid), dtype=torch.float64, device=opd.device)
    _capi.check(lib.mkb_psf_maps_device(tuples, grid, samples, int(half),
                                        C.c_void_p(opd.data_ptr()), C.c_void_p(status.data_ptr()),
                                        C.c_void_p(column.data_ptr()), C.c_void_p(row.data_ptr()),
                                        C.c_void_p(maps.data_ptr()), _stream_handle(stream)),
                "psf maps")
    psf, mtf = psf_device(maps, params, grid, fft_size, stream)
    return maps, psf, mtf
