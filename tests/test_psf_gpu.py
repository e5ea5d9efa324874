"""Scalar PSF and MTF on the device (PsfEngine::compute): the library's own shared-memory FFT
against the reference's psf_cpu (radix-2 FFT on the CPU) within the reference's own CPU/GPU bar
(1e-13 in units of the unaberrated peak and of MTF(0) = 1, tests/tolerances.hpp:286), on EVAL
results of singlets (full and half pupils) and objectives with failed rays, on given pupils with
mirrored axes and holes, over the FFT sizes that select each column-tile width; the figures of
finish_psf; the device EVAL -> PSF chain; repeat runs bit for bit."""

import numpy as np
import pytest
import torch

from conftest import has_reference_build
from mikroptim_b200 import engine, psf, workloads
from mikroptim_b200.batch import ResidualLayout
import oracle.pyoracle as po

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_reference_build(), reason="reference build missing")]

BAR = 1e-13  # kPsfCpuGpu
FIGURES = po.Reference.PSF_METRICS
# figures that depend on the pupil map only (bit for bit), and on the PSF (within the bar)
EXACT = ("transmitted", "strehl_origin", "strehl", "reference_x", "reference_y", "dx", "dy",
         "airy_radius")
NEAR = ("energy", "strehl_fft", "peak")


def _compare(r: psf.PsfResult, want_psf, want_mtf, want_metrics):
    assert np.abs(r.psf - want_psf).max() <= BAR
    assert np.abs(r.mtf_sagittal - want_mtf[0]).max() <= BAR
    assert np.abs(r.mtf_tangential - want_mtf[1]).max() <= BAR
    m = dict(zip(FIGURES, want_metrics))
    for k in EXACT:
        got, exp = getattr(r, k), m[k]
        assert got == exp or (np.isnan(got) and np.isnan(exp)), k
    for k in NEAR:
        assert abs(getattr(r, k) - m[k]) <= BAR, k
    if (r.peak_x, r.peak_y) != (m["peak_x"], m["peak_y"]):  # a tie within the rounding
        M = r.fft_size
        i = int(round(m["peak_x"] / r.dx + M / 2))
        j = int(round(m["peak_y"] / r.dy + M / 2))
        assert abs(r.psf_at(i, j) - r.peak) <= BAR


@pytest.mark.parametrize("make,grid,half", [(lambda: workloads.singlet(2), 16, False),
                                            (lambda: workloads.singlet(2), 15, True),
                                            (lambda: workloads.singlet(1), 64, False),
                                            (lambda: workloads.objective(2, rings=4, spokes=8),
                                             20, False)])
def test_psf_of_eval_results_within_the_references_bar(make, grid, half):
    ref = po.reference()
    b, st, _, _ = make()
    lay = ResidualLayout(b.topology, st)
    res = engine.TraceEngine(0).evaluate(b, engine.EvalSettings(grid=grid, half_pupil=half))
    eng = psf.PsfEngine(0)
    for v in range(b.variants):
        got = eng.compute(b, res, v, psf.PsfSettings())
        want = ref.psf(b, lay, v, grid, half)
        assert len(got) == b.fields * b.wavelengths
        for t, r in enumerate(got):
            assert r.fft_size == want["fft_size"]
            _compare(r, want["psf"][t], want["mtf"][t], want["metrics"][t])
    assert eng.last_run.pupils == b.fields * b.wavelengths and eng.last_run.tranches == 1


def _aberrated_pupil(N, seed, holes=True):
    rng = np.random.default_rng(seed)
    a = (2 * np.arange(N) + 1 - N) / N
    x, y = np.meshgrid(a, a)
    r2 = x * x + y * y
    opd = (3e-4 * r2 + 2e-4 * r2 * r2 + 8e-5 * y * r2 + 4e-5 * x + 2e-5 *
           rng.standard_normal((N, N)))
    opd[r2 > 1.0] = np.nan
    if holes:
        opd[rng.integers(0, N, 5), rng.integers(0, N, 5)] = np.nan
    return opd.reshape(-1), int(np.count_nonzero(r2 <= 1.0))


@pytest.mark.parametrize("N,M", [(8, 16), (24, 64), (40, 128), (64, 512), (100, 1024),
                                 (256, 2048)])
def test_given_pupils_with_mirrored_axes_and_holes(N, M):
    ref = po.reference()
    pupils = []
    for k, (fx, fy) in enumerate(((0, 0), (1, 0), (0, 1), (1, 1))):
        opd, full = _aberrated_pupil(N, 11 + k)
        pupils.append(psf.PsfPupil(0, k, N, full, 486.1 + 50 * k, 0.15 + 0.05 * k, 0.2,
                                   bool(fx), bool(fy), opd))
    got = psf.PsfEngine(0).compute(pupils, M)
    for p, r in zip(pupils, got):
        want = ref.psf_pupil(N, M, p.opd, p.full_count, p.wavelength_nm, p.na_x, p.na_y,
                             p.flip_x, p.flip_y)
        _compare(r, want["psf"], want["mtf"], want["metrics"])


@pytest.mark.parametrize("N,M", [(32, 128), (1024, 8192)])
def test_unaberrated_pupil(N, M):
    a = (2 * np.arange(N) + 1 - N) / N
    x, y = np.meshgrid(a, a)
    inside = x * x + y * y <= 1.0
    opd = np.where(inside, 0.0, np.nan).reshape(-1)
    p = psf.PsfPupil(0, 0, N, int(inside.sum()), 550.0, 0.1, 0.1, False, False, opd)
    r = psf.PsfEngine(0).compute([p], M)[0]
    assert abs(r.strehl_fft - 1.0) <= 1e-12 and abs(r.peak - 1.0) <= 1e-12
    assert r.peak_x == 0.0 and r.peak_y == 0.0
    assert abs(r.energy - 1.0) <= 1e-12
    assert r.mtf_sagittal[0] == pytest.approx(1.0, abs=1e-14)
    assert r.mtf_sagittal[N] <= 1e-3 and r.mtf_tangential[N] <= 1e-3


def test_device_chain_equals_the_host_maps_and_repeats_bit_for_bit():
    b, st, _, _ = workloads.objective(2, rings=4, spokes=8)
    grid = 24
    settings = engine.EvalSettings(grid=grid)
    db = engine.DeviceSystemBatch(b)
    pts, _, _, out = engine.evaluate_device_tensors(db, b, settings)
    res = engine.evaluate_device(db, b, settings)
    col, row, full, half = psf.grid_cells(res)
    T = b.variants * b.fields * b.wavelengths
    pupils = [p for v in range(b.variants) for p in psf.make_psf_pupils(b, res, v)]
    params = [psf.pupil_params(p) for p in pupils]
    M = psf.psf_fft_size(grid, 4.0)
    dev = db.device
    maps, P, mtf = psf.psf_from_eval_device(out, T, grid, pts.shape[0], half,
                                            torch.from_numpy(col).to(dev),
                                            torch.from_numpy(row).to(dev), params, M)
    host_maps = np.stack([p.opd for p in pupils]).reshape(T, grid, grid)
    assert np.array_equal(maps.cpu().numpy(), host_maps, equal_nan=True)
    got = psf.PsfEngine(0).compute(pupils, M)
    P2, mtf2 = psf.psf_device(maps, params, grid, M)
    assert torch.equal(P, P2) and torch.equal(mtf, mtf2)
    for t, r in enumerate(got):
        assert np.array_equal(r.psf, P[t].cpu().numpy().reshape(-1))
        assert np.array_equal(r.mtf_sagittal, mtf[t, 0].cpu().numpy())


def test_tranches_equal_one_call():
    pupils = []
    for k in range(6):
        opd, full = _aberrated_pupil(16, 30 + k)
        pupils.append(psf.PsfPupil(0, k, 16, full, 550.0, 0.2, 0.2, False, bool(k & 1), opd))
    one = psf.PsfEngine(0).compute(pupils, 64)
    per = psf.PsfEngine.tranche_bytes(1, 16, 64)
    small = psf.PsfEngine(0, engine.EngineOptions(
        memory_limit_bytes=(300 << 20) + 2 * per,
        reserve=engine.MemoryReserve(min_bytes=300 << 20, fraction=0.0)))
    parts = small.compute(pupils, 64)
    assert small.last_run.tranches > 1
    for a, c in zip(one, parts):
        assert np.array_equal(a.psf, c.psf) and a.strehl_fft == c.strehl_fft
