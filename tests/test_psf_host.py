"""The host half of the scalar PSF, on the CPU: the FFT size rule (psf_fft_size), the pupil
maps from an EVAL result (eval_opd_map), the NA and mirror flags of the pupil imaging from the
field rays (make_psf_pupil) and the per-tuple figures (finish_psf) against the reference's own
functions on the reference's EVAL and PSF, bit for bit; and the device entry point's argument
checks, which run before anything is enqueued."""

import ctypes as C

import numpy as np
import pytest

from conftest import has_reference_build
from mikroptim_b200 import _capi, engine, psf, workloads
from mikroptim_b200.batch import ResidualLayout
import oracle.pyoracle as po

FIGURES = po.Reference.PSF_METRICS


@pytest.mark.parametrize("grid,padding,want", [(64, 4.0, 256), (100, 2.5, 256), (1, 2.0, 2),
                                               (33, 2.0, 128), (2048, 4.0, 8192),
                                               (3, 3.0, 16)])
def test_fft_size_rule(grid, padding, want):
    assert psf.psf_fft_size(grid, padding) == want


@pytest.mark.parametrize("grid,padding", [(0, 4.0), (2049, 4.0), (2048, 4.1), (64, 1.9),
                                          (64, float("inf"))])
def test_fft_size_rejects(grid, padding):
    with pytest.raises(ValueError):
        psf.psf_fft_size(grid, padding)


def _eval_result(ref, b, lay, grid, half, reference=0, delta=1e-3):
    want = ref.eval(b, lay, grid, half, reference, delta)
    return engine.EvalResult(b.variants, b.fields, b.wavelengths, engine.eval_grid(grid, half),
                             want["kappa"], want["exit_pupil"], want["opd"], want["spot_x"],
                             want["spot_y"], want["status"], want["field_rays"],
                             want["field_status"], grid, half, delta)


@pytest.mark.skipif(not has_reference_build(), reason="reference CPU build missing")
@pytest.mark.parametrize("make,grid,half", [(lambda: workloads.singlet(3), 16, False),
                                            (lambda: workloads.singlet(3), 15, True),
                                            (lambda: workloads.objective(2, rings=4, spokes=8),
                                             20, False)])
def test_pupils_and_figures_equal_the_reference(make, grid, half):
    ref = po.reference()
    b, st, _, _ = make()
    lay = ResidualLayout(b.topology, st)
    res = _eval_result(ref, b, lay, grid, half)
    for v in range(b.variants):
        want = ref.psf(b, lay, v, grid, half)
        pupils = psf.make_psf_pupils(b, res, v)
        M = want["fft_size"]
        assert M == psf.psf_fft_size(grid, 4.0)
        for t, p in enumerate(pupils):
            assert p.full_count == want["full_count"]
            assert np.array_equal(p.opd, want["maps"][t], equal_nan=True)
            assert (p.na_x, p.na_y) == tuple(want["na"][t])
            assert (int(p.flip_x), int(p.flip_y)) == tuple(want["flips"][t])
            # finish_psf on the reference's own PSF: every figure bit for bit
            r = psf.prepare_psf_result(p, M)
            r.psf = want["psf"][t]
            psf.finish_psf(r, p)
            got = np.array([getattr(r, k) for k in FIGURES], dtype=np.float64)
            assert np.array_equal(got, want["metrics"][t], equal_nan=True), (v, t)


@pytest.mark.skipif(not has_reference_build(), reason="reference CPU build missing")
def test_finish_with_flips_holes_and_a_given_na():
    ref = po.reference()
    N, M = 24, 64
    rng = np.random.default_rng(7)
    a = (2 * np.arange(N) + 1 - N) / N
    x, y = np.meshgrid(a, a)
    opd = 2e-4 * (x * x + y * y) + 5e-5 * y + 1e-5 * rng.standard_normal((N, N))
    opd[x * x + y * y > 1.0] = np.nan
    opd[3, 10] = np.nan  # a failed ray
    full = int(np.count_nonzero(x * x + y * y <= 1.0))
    for fx, fy in ((0, 0), (1, 0), (0, 1), (1, 1)):
        want = ref.psf_pupil(N, M, opd.reshape(-1), full, 546.1, 0.2, 0.25, fx, fy)
        p = psf.PsfPupil(0, 0, N, full, 546.1, 0.2, 0.25, bool(fx), bool(fy), opd.reshape(-1))
        r = psf.prepare_psf_result(p, M)
        r.psf = want["psf"]
        psf.finish_psf(r, p)
        got = np.array([getattr(r, k) for k in FIGURES], dtype=np.float64)
        assert np.array_equal(got, want["metrics"], equal_nan=True), (fx, fy)


def test_aperture_rejects_an_undetermined_na():
    lib = _capi.lib()
    rays = np.zeros(20)
    status = np.array([0, 0, 0, 1], dtype=np.uint8)  # the sagittal field ray failed
    na = [C.c_double(), C.c_double()]
    fl = [C.c_int32(), C.c_int32()]
    args = [rays.ctypes.data, status.ctypes.data, 1.0, 1e-3]
    rc = lib.mkb_psf_aperture_host(*args, 0.0, C.byref(na[0]), C.byref(na[1]), C.byref(fl[0]),
                                   C.byref(fl[1]))
    assert rc == _capi.MKB_ERR_ARGUMENT
    rc = lib.mkb_psf_aperture_host(*args, 0.3, C.byref(na[0]), C.byref(na[1]), C.byref(fl[0]),
                                   C.byref(fl[1]))
    assert rc == _capi.MKB_OK and na[0].value == na[1].value == 0.3


@pytest.mark.parametrize("tuples,grid,fft,null", [(1, 16, 48, False), (1, 16, 16, False),
                                                  (1, 0, 16, False), (1, 16, 16384, False),
                                                  (-1, 16, 64, False), (2, 16, 64, True)])
def test_device_entry_rejects_bad_arguments_before_launch(tuples, grid, fft, null):
    lib = _capi.lib()
    dummy = C.c_void_p(0 if null else 1 << 20)
    rc = lib.mkb_psf_device(tuples, grid, fft, dummy, dummy, dummy, dummy, dummy, 0, None)
    assert rc == _capi.MKB_ERR_ARGUMENT
    assert (lib.mkb_psf_workspace_bytes(tuples, grid, fft) > 0) == null


def test_workspace_holds_the_row_spectra():
    lib = _capi.lib()
    # twiddles (M/2 complex), the N x M row spectra and the projections of every tuple
    assert lib.mkb_psf_workspace_bytes(10, 64, 256) >= 10 * 64 * 256 * 16 + 128 * 16
