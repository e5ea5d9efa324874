"""An aperture stop inside the system (MKB_SURFACE_APERTURE_STOP) on the GPU.

The trace of an aimed batch is the reference's trace of the same systems with the stop as a
plane and surface 0 at the aimed entrance pupil: RESIDUALS and MERIT bit for bit. Applying
the variables on the device aims the records exactly as packing does. The aimed pupil moves
with the variables before the stop, and the adjoint folds that motion into every column
(d/da and d/dt0 of the start ray times the pupil's sensitivities): the materialised adjoint
Jacobian agrees with refined central differences of the aimed traces, and the fused normal equations
with the materialised ones. The LM optimises aimed objectives (configuration 2 with its stop
at surface 8).
"""

import ctypes as C

import numpy as np
import pytest
import torch

from conftest import has_reference_build
from mikroptim_b200 import _capi, engine, workloads
from mikroptim_b200.batch import (PRECISION_FP64, PRECISION_FP64_FMA, PRECISION_MIXED,
                                  ResidualLayout)
import oracle.pyoracle as po

pytestmark = pytest.mark.gpu


def aimed(make, stop, precision=PRECISION_FP64):
    b, st, vs, x0 = make()
    ab, st, avs, ax0 = workloads.with_aperture_stop(b, st, vs, stop)
    st.precision = precision
    return ab, st, avs, ax0, ResidualLayout(ab.topology, st)


CASES = [(lambda: workloads.singlet(24), 2),
         (lambda: workloads.objective(6, rings=6, spokes=8, na=0.3), 8),
         (lambda: workloads.objective(6, rings=6, spokes=8, na=0.3), 4)]


@pytest.mark.skipif(not has_reference_build(), reason="reference build missing")
@pytest.mark.parametrize("make,stop", CASES)
def test_trace_equals_the_reference_on_the_aimed_systems(make, stop):
    b, st, _, _, lay = aimed(make, stop)
    db = engine.DeviceSystemBatch(b)
    res = engine.residuals_device(db, lay, b)
    mer = engine.merit_device(db, lay, b)
    ref = po.reference()
    eq = po.port().aimed_equivalent(b)
    leq = ResidualLayout(eq.topology, st)
    r, opd, status = ref.residuals(eq, leq)
    m, failed, hard = ref.merit(eq, leq)
    torch.cuda.synchronize()
    assert np.array_equal(res.residuals.cpu().numpy(), r)
    assert np.array_equal(res.status.cpu().numpy(), status)
    assert np.array_equal(mer.merit.cpu().numpy(), m)
    assert np.array_equal(mer.failed.cpu().numpy(), failed)


def test_device_apply_aims_like_the_pack():
    b, st, vs, x0, lay = aimed(CASES[1][0], 8)
    lib = _capi.lib()
    db = engine.DeviceSystemBatch(b)
    xs = torch.from_numpy(np.ascontiguousarray(x0)).cuda()
    out = torch.empty_like(db.records)
    bs = db.c_struct()
    vars_ = vs.c_struct()
    rc = lib.mkb_apply_variables_device(C.byref(bs), C.byref(vars_), C.c_void_p(xs.data_ptr()),
                                        b.variants, C.c_void_p(out.data_ptr()), None)
    _capi.check(rc, "apply")
    torch.cuda.synchronize()
    assert torch.equal(out, db.records)
    # moving a curvature before the stop moves the entrance pupil the same way on both sides
    x1 = x0.copy()
    k = next(i for i, v in enumerate(vs.variables) if v.type == 0 and v.surface < 8)
    x1[:, k] *= 1.02
    b1 = b.subset(0, b.variants)
    for v in range(b.variants):
        vs.apply(b1, v, x1[v])
    d1 = engine.DeviceSystemBatch(b1)
    rc = lib.mkb_apply_variables_device(C.byref(bs), C.byref(vars_),
                                        C.c_void_p(torch.from_numpy(x1).cuda().data_ptr()),
                                        b.variants, C.c_void_p(out.data_ptr()), None)
    _capi.check(rc, "apply")
    torch.cuda.synchronize()
    assert torch.equal(out, d1.records)
    assert not torch.equal(out, db.records)


def _aimed_rows(port, one, st, vs, x):
    """Residuals and statuses of a one-variant aimed batch at x: the oracle's aiming and trace
    (the reference's arithmetic) on the equivalent batch."""
    bb = one.subset(0, 1)
    vs.apply(bb, 0, x)
    eq = port.aimed_equivalent(bb)
    r, _, status = port.residuals(eq, ResidualLayout(eq.topology, st))
    return r[0], status[0]


def _refined_column(port, one, st, vs, x, j, rel=1e-7):
    """dr/dx_j by Richardson-extrapolated central differences (steps h and h/2, h = rel
    max(|x_j|, typical)); rows whose statuses change inside the stencil are NaN."""
    h = rel * max(abs(x[j]), vs.variables[j].typical)
    d, same = [], None
    for step in (h, h / 2):
        xp, xm = x.copy(), x.copy()
        xp[j] += step
        xm[j] -= step
        (rp, sp), (rm, sm) = _aimed_rows(port, one, st, vs, xp), _aimed_rows(port, one, st, vs, xm)
        d.append((rp - rm) / (2 * step))
        eq = np.concatenate([sp == sm] * 2)  # ray rows, then the penalty rows
        same = eq if same is None else same & eq
    out = (4 * d[1] - d[0]) / 3
    out[~same] = np.nan
    return out


@pytest.mark.parametrize("make,stop", CASES)
def test_adjoint_jacobian_matches_refined_differences(make, stop):
    """The aiming fold: the pupil's radius and distance move with the variables before the
    stop, and the adjoint J carries that motion. Checked column by column against central
    differences of the aimed traces (the oracle's aiming and trace) refined by Richardson
    extrapolation: the device FD Jacobian's fixed step is too coarse on these aberrated rays
    (up to 5e-2 of a column), the refined differences agree with the adjoint to their own
    truncation. Without the fold the same columns are off by their whole size."""
    b, st, vs, x0, lay = aimed(make, stop)
    db = engine.DeviceSystemBatch(b)
    Ja, _, _ = engine.adjoint_jacobian_device(db, lay, b, vs, x0)
    eq = po.port().aimed_equivalent(b)
    Je, _, _ = engine.adjoint_jacobian_device(engine.DeviceSystemBatch(eq),
                                              ResidualLayout(eq.topology, st), eq, vs, x0)
    Ja, Je = Ja.cpu().numpy(), Je.cpu().numpy()
    port = po.port()
    before = [j for j, v in enumerate(vs.variables) if v.surface < stop]
    # step of the differences: the singlets' residuals are large against their derivatives
    # (rounding wants a wide step), the objectives' rays are strongly curved (truncation wants
    # a narrow one); at these steps two refinements agree to ~1e-7 (median)
    rel = 1e-5 if b.surfaces <= 4 else 1e-7
    errs, nofold = [], []
    for run in range(min(b.variants, 4)):
        one = b.subset(run, 1)
        for j in before:
            ref = _refined_column(port, one, st, vs, x0[run], j, rel)
            ok = ~np.isnan(ref)
            scale = np.linalg.norm(ref[ok]) + 1e-300
            errs.append(np.linalg.norm(Ja[run, j][ok] - ref[ok]) / scale)
            nofold.append(np.linalg.norm(Je[run, j][ok] - ref[ok]) / scale)
    errs, nofold = np.array(errs), np.array(nofold)
    assert np.median(errs) <= 1e-6 and errs.max() <= 1e-3, (np.median(errs), errs.max())
    assert np.median(nofold) >= 1e-2, np.median(nofold)


def test_device_fd_agrees_with_the_adjoint_on_singlets():
    """On singlets the device FD Jacobian's step is fine enough: every column of the aimed
    adjoint J within 2e-6 of the FD J (both FP64) relative to the column norm."""
    b, st, vs, x0, lay = aimed(CASES[0][0], CASES[0][1])
    db = engine.DeviceSystemBatch(b)
    Ja, ra, _ = engine.adjoint_jacobian_device(db, lay, b, vs, x0)
    Jf, rf, ch = engine.fd_jacobian_device(db, lay, b, vs, x0)
    Ja, Jf, ra, rf, ch = (t.cpu().numpy() for t in (Ja, Jf, ra, rf, ch))
    assert np.array_equal(ra, rf)
    for run in range(b.variants):
        for j in range(vs.size):
            if ch[run, j]:
                continue
            scale = max(np.linalg.norm(Jf[run, j]), 1e-300)
            assert np.linalg.norm(Ja[run, j] - Jf[run, j]) <= 2e-6 * scale, (run, j)


@pytest.mark.parametrize("precision,median_bar,max_bar", [(PRECISION_FP64_FMA, 1e-10, 1e-8),
                                                          (PRECISION_MIXED, 1e-5, 2e-3)])
def test_fused_normal_equations_with_an_interior_stop(precision, median_bar, max_bar):
    b, st, vs, x0, lay = aimed(CASES[1][0], 8)
    db = engine.DeviceSystemBatch(b)
    J, r0, _ = engine.adjoint_jacobian_device(db, lay, b, vs, x0)
    ref = engine.normal_equations_device(J, r0, True)
    b2, st2, vs2, x02, lay2 = aimed(CASES[1][0], 8, precision)
    fused = engine.adjoint_normal_equations_device(engine.DeviceSystemBatch(b2), lay2, b2, vs2,
                                                   x02)
    ref, fused = ref.cpu().numpy(), fused.cpu().numpy()
    d = np.abs(np.diagonal(ref, axis1=1, axis2=2))
    d = np.maximum(d, 1e-20 * d.max(axis=1, keepdims=True) + 1e-300)
    err = np.abs(fused - ref) / np.sqrt(d[:, :, None] * d[:, None, :])
    assert np.median(err) <= median_bar and err.max() <= max_bar, (np.median(err), err.max())


@pytest.mark.parametrize("method", [engine.JACOBIAN_ADJOINT, engine.JACOBIAN_FD])
def test_lm_optimises_objectives_with_the_stop_at_surface_8(method):
    b, st, vs, x0, lay = aimed(lambda: workloads.objective(8, rings=6, spokes=8, na=0.3), 8,
                               PRECISION_FP64_FMA)
    out = engine.optimize_lm_gpu(b, lay, vs, x0, engine.LmOptions(
        max_iterations=15, jacobian=method, fail_weight_factor=1.0))
    assert np.all(out["merit"] <= out["history"][:, 0])
    assert np.mean(out["merit"] < 0.9 * out["history"][:, 0]) >= 0.5
