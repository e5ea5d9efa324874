"""The trace autotuner and the launch shapes it chooses between.

Every plan (pack_rays x variants_per_cta) must give bit-identical RESIDUALS and MERIT in every
precision mode -- the FP64 mode stays equal to the reference CPU -- on singlets, objectives,
uneven batches, ghost plates and decentered systems; the tuner must measure, cache and return
one of its candidates.
"""

import dataclasses
import json

import numpy as np
import pytest
import torch

from mikroptim_b200 import _capi, autotune, engine, workloads
from mikroptim_b200.batch import PRECISION_FP64, PRECISION_FP64_FMA, ResidualLayout
import oracle.pyoracle as po

pytestmark = pytest.mark.gpu

PLANS = [autotune.TracePlan(r, v) for r in (128, 384, 512, 1024) for v in (1, 2, 3, 8)]


def _cases():
    yield "singlet", *workloads.singlet(37)[:2]
    yield "objective", *workloads.objective(11, rings=5, spokes=8)[:2]
    yield "uneven", *workloads.uneven(13, rings=4, spokes=8)[:2]
    yield "ghost", *workloads.ghost(9)[:2]
    yield "decentered", *workloads.tolerancing(10, elements=3, rings=4, spokes=8)[:2]


@pytest.mark.parametrize("precision", [PRECISION_FP64, PRECISION_FP64_FMA])
def test_every_plan_gives_bit_identical_results(precision):
    for name, b, st in _cases():
        st = dataclasses.replace(st, precision=precision)
        lay = ResidualLayout(b.topology, st)
        db = engine.DeviceSystemBatch(b)
        r0 = engine.residuals_device(db, lay, b)
        m0 = engine.merit_device(db, lay, b)
        for tp in PLANS:
            r = engine.residuals_device(db, lay, b, pack_rays=tp.pack_rays,
                                        variants_per_cta=tp.variants_per_cta)
            m = engine.merit_device(db, lay, b, pack_rays=tp.pack_rays,
                                    variants_per_cta=tp.variants_per_cta)
            assert torch.equal(r.residuals, r0.residuals), (name, tp)
            assert torch.equal(r.opd, r0.opd) and torch.equal(r.status, r0.status), (name, tp)
            assert torch.equal(m.merit, m0.merit), (name, tp)
            assert torch.equal(m.failed, m0.failed) and torch.equal(m.hard_failed,
                                                                    m0.hard_failed)
        if precision == PRECISION_FP64 and name != "uneven":
            mo, fo, _ = po.port().merit(b, lay)
            assert np.array_equal(m0.merit.cpu().numpy(), mo), name
    assert _capi.lib().mkb_device_status() == _capi.MKB_OK


def test_autotuner_measures_caches_and_reuses(tmp_path):
    b, st, _, _ = workloads.singlet(2048)
    lay = ResidualLayout(b.topology, st)
    path = str(tmp_path / "plans.json")
    tuner = autotune.TraceAutotuner(cache_path=path, launches=2,
                                    candidates=[autotune.TracePlan(r, v)
                                                for r in (256, 512) for v in (1, 2, 4)])
    plan = tuner.plan(b, lay, "merit")
    assert plan in tuner.candidates
    entry = json.load(open(path))[autotune.shape_key(b, lay, "merit")]
    assert len(entry["timings"]) == 6 and entry["ms"] == min(t[2] for t in entry["timings"])
    again = autotune.TraceAutotuner(cache_path=path).plan(b, lay, "merit")
    assert again == plan  # from the file, no measurement
    m = engine.merit_device(engine.DeviceSystemBatch(b), lay, b, pack_rays=plan.pack_rays,
                            variants_per_cta=plan.variants_per_cta)
    assert np.array_equal(m.merit.cpu().numpy(), po.port().merit(b, lay)[0])


def test_plans_beyond_the_limits_are_refused():
    b, st, _, _ = workloads.objective(4, rings=16, spokes=32)
    lay = ResidualLayout(b.topology, st)
    db = engine.DeviceSystemBatch(b)
    with pytest.raises(ValueError):
        engine.merit_device(db, lay, b, variants_per_cta=9)
    with pytest.raises(ValueError):  # 8 x 4096-ray packs do not fit in shared memory
        engine.merit_device(db, lay, b, pack_rays=4096, variants_per_cta=8)
