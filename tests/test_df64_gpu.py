"""The reference's reduced-precision trace type on the B200: DF64 (double-float pairs on the
FP32 pipes, include/mikroptim/math/df64.hpp of the reference) in RESIDUALS and MERIT. Bar as the
reference's (docs/numerik.md, "df64"): per ray |OPD_df64 - OPD_FP64| <= max(1e-9 mm,
1e-10 |OPD|), the same statuses, merit within 1e-9 relative on variants without failed rays,
against the bit-exact FP64 trace.
"""

import dataclasses

import numpy as np
import pytest
import torch

from mikroptim_b200 import engine, workloads
from mikroptim_b200.batch import PRECISION_DF64, PRECISION_FP64, ResidualLayout

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("make", [lambda: workloads.singlet(64),
                                  lambda: workloads.objective(16, rings=6, spokes=12),
                                  lambda: workloads.ghost(16),
                                  lambda: workloads.tolerancing(8, elements=3, rings=6,
                                                                spokes=12)])
def test_df64_trace_within_the_references_bar(make):
    b, st, _, _ = make()
    db = engine.DeviceSystemBatch(b)
    out = {}
    for p in (PRECISION_FP64, PRECISION_DF64):
        lay = ResidualLayout(b.topology, dataclasses.replace(st, precision=p))
        r = engine.residuals_device(db, lay, b)
        m = engine.merit_device(db, lay, b)
        torch.cuda.synchronize()
        out[p] = (r.opd.cpu().numpy(), r.status.cpu().numpy(), m.merit.cpu().numpy())
    (o64, s64, m64), (od, sd, md) = out[PRECISION_FP64], out[PRECISION_DF64]
    assert np.mean(s64 == sd) >= 0.999
    same = (s64 == sd) & (s64 == 0)
    err = np.abs(od - o64)[same]
    bar = np.maximum(1e-9, 1e-10 * np.abs(o64[same]))
    assert np.all(err <= bar), float((err / bar).max())
    # merit on the variants whose every ray is Ok (a ray continued past a soft failure
    # amplifies rounding, in FP64 with contraction as much as here)
    clean = np.all((s64 == sd) & (s64 == 0), axis=1)
    if clean.any():
        rel = np.abs(md - m64)[clean] / np.maximum(m64[clean], 1e-300)
        assert rel.max() <= 1e-9, rel.max()


@pytest.mark.parametrize("make", [lambda: workloads.objective(8, rings=4, spokes=8),
                                  lambda: workloads.ghost(8),
                                  lambda: workloads.tolerancing(4, elements=3, rings=4,
                                                                spokes=8)])
def test_df64_extrema_within_the_bar(make):
    """Per-surface extrema in DF64 (the reference's merit kernel reduces them for df64 too):
    the largest heights within 1e-9 relative and the smallest cos I within 1e-9 of the FP64
    ones."""
    b, st, _, _ = make()
    eng = engine.TraceEngine(0)
    got = {}
    for p in (PRECISION_FP64, PRECISION_DF64):
        ts = engine.TraceSettings(dataclasses.replace(st, precision=p), extrema=True)
        got[p] = eng.run(b, engine.TraceMode.MERIT, ts).merit.extrema
    e, d = got[PRECISION_FP64], got[PRECISION_DF64]
    assert np.any(e[:, 1:, 0] > 0.0)
    h = np.abs(d[..., 0] - e[..., 0]) / np.maximum(np.abs(e[..., 0]), 1e-300)
    assert h.max() <= 1e-9, h.max()
    assert np.abs(d[..., 1] - e[..., 1]).max() <= 1e-9
