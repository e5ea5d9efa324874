"""FP32 prefilter of multistart variants (TraceEngine::prefilter_variants, the reference's
prefilter_cpu in src/batch/batch_prefilter.cpp).

The kernel traces in float with the reference's order of operations (every operation
separately rounded, sums in ascending sample order), so its per-variant results -- the float
merit of the certainly valid rays, the optical length, and the counts of certainly failed,
uncertain valid and uncertain failed rays -- equal the reference CPU prefilter bit for bit on
multistart batches of every kind (singlets, seven-element objectives, ghost plates, decentered
and tilted systems; soft and hard FP64 truth). The decision on the host is checked against the
reference's decision, and against the FP64 truth: no variant is rejected for a reason its FP64
merit does not have, and merit_lower <= F_FP64 <= merit_upper for every variant.
"""

import dataclasses

import numpy as np
import pytest
import torch

from conftest import has_reference_build
from mikroptim_b200 import _capi, engine, workloads
from mikroptim_b200.batch import FAILURE_HARD, FAILURE_SOFT, PRECISION_FP64, ResidualLayout
import oracle.pyoracle as po

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_reference_build(), reason="reference CPU build missing")]

STATS = ("merit", "optical_length", "failed", "uncertain_ok", "uncertain_failed")


def _batches():
    b, st, _, _ = workloads.singlet(600)
    yield "singlet", workloads.multistart(b), st
    b, st, _, _ = workloads.objective(84, rings=4, spokes=8)
    yield "objective", workloads.multistart(b, seed=20261203 + 22), st
    b, st, _, _ = workloads.ghost(140)
    yield "ghost", workloads.multistart(b, seed=20261203 + 23), st
    b, st, _, _ = workloads.tolerancing(56, elements=3, rings=4, spokes=8, decenter_mm=0.5,
                                        tilt_rad=0.05)
    b.curvature[:] *= 3.0  # stronger elements and a wider pupil: rays fail
    b.pupil_radius[:] *= 4.0
    yield "decentered", workloads.multistart(b, seed=20261203 + 24), st


def _criteria(fp64_merit, failed, rays):
    """The reference acceptance test's kinds of criteria: failed-ray fractions, merits above
    quantiles of the FP64 values, merits above multiples of the best, and combinations."""
    q = np.quantile(fp64_merit, [0.25, 0.5, 0.9])
    fq = float(np.quantile(failed / rays, 0.9))
    inf = float("inf")
    out = [dict(max_failed_fraction=x) for x in (0.01, 0.1, 0.5, fq)]
    out += [dict(max_failed_fraction=1.0, max_merit=float(x)) for x in q]
    out += [dict(max_failed_fraction=1.0, max_merit_factor=x) for x in (2.0, 10.0, 100.0, 1e4)]
    out += [dict(max_failed_fraction=0.1, max_merit=float(q[2]), max_merit_factor=100.0)]
    return [engine.PrefilterOptions(**{**dict(max_merit=inf, max_merit_factor=inf), **c})
            for c in out]


@pytest.mark.parametrize("failure", [FAILURE_SOFT, FAILURE_HARD])
def test_prefilter_stats_bitwise_equal_to_the_reference(failure):
    ref = po.reference()
    for name, b, st in _batches():
        st = dataclasses.replace(st, failure=failure, precision=PRECISION_FP64)
        lay = ResidualLayout(b.topology, st)
        got = engine.prefilter_device(engine.DeviceSystemBatch(b), lay, b, 0.15)
        want = ref.prefilter(b, lay, engine.PrefilterOptions().c_struct())
        for k in STATS:
            assert np.array_equal(getattr(got, k), want[k]), (name, k)
        # the batches exercise every class
        assert got.failed.sum() > 0 and (got.uncertain_ok + got.uncertain_failed).sum() > 0, name
    assert _capi.lib().mkb_device_status() == _capi.MKB_OK


@pytest.mark.parametrize("boundary", [0.0, 0.05, 0.3])
def test_prefilter_stats_follow_the_boundary(boundary):
    ref = po.reference()
    b, st, _, _ = workloads.singlet(300)
    b = workloads.multistart(b)
    lay = ResidualLayout(b.topology, st)
    got = engine.prefilter_device(engine.DeviceSystemBatch(b), lay, b, boundary)
    want = ref.prefilter(b, lay, engine.PrefilterOptions(boundary=boundary).c_struct())
    for k in STATS:
        assert np.array_equal(getattr(got, k), want[k]), k


@pytest.mark.parametrize("failure", [FAILURE_SOFT, FAILURE_HARD])
def test_prefilter_decisions_equal_the_reference_and_never_reject_wrongly(failure):
    ref = po.reference()
    eng = engine.TraceEngine(0)
    for name, b, st in _batches():
        st = dataclasses.replace(st, failure=failure, precision=PRECISION_FP64)
        lay = ResidualLayout(b.topology, st)
        fp64 = eng.run(b, engine.TraceMode.MERIT, st).merit
        rng = np.random.default_rng(7)
        for extra in (None, rng.uniform(0.0, 2.0, b.variants)):
            for opt in _criteria(fp64.merit, fp64.failed, lay.rays_per_variant):
                res = eng.prefilter_variants(b, engine.PrefilterSettings(st, opt, extra))
                want = ref.prefilter(b, lay, opt.c_struct(), extra)
                assert np.array_equal(res.reject, want["reject"]), (name, opt)
                assert np.array_equal(res.merit_lower, want["merit_lower"]), name
                assert np.array_equal(res.merit_upper, want["merit_upper"]), name
                assert res.reference_merit == want["reference_merit"]
                assert res.reference_variant == want["reference_variant"]
                assert res.kept == want["kept"]
                truth = engine.prefilter_decide_exact(fp64.merit, fp64.failed,
                                                      lay.rays_per_variant, opt, extra)
                assert np.array_equal(truth, ref.prefilter_decide_exact(
                    opt.c_struct(), fp64.merit, fp64.failed, lay.rays_per_variant, extra))
                # a reason the FP64 truth does not have never occurs
                assert not np.any(res.reject & ~truth), (name, opt)
                total = fp64.merit + (extra if extra is not None else 0.0)
                assert np.all(res.merit_lower <= total), name
                assert np.all(total <= res.merit_upper), name
                # the failed-ray bracket of assumption (A)
                assert np.all(res.stats.failed <= fp64.failed), name
                assert np.all(fp64.failed <= res.stats.failed + res.stats.uncertain_ok +
                              res.stats.uncertain_failed), name


def test_prefilter_repeats_and_batch_positions_bit_identical():
    b, st, _, _ = workloads.objective(40, rings=4, spokes=8)
    b = workloads.multistart(b, seed=20261203 + 25)
    lay = ResidualLayout(b.topology, st)
    whole = engine.prefilter_device(engine.DeviceSystemBatch(b), lay, b)
    again = engine.prefilter_device(engine.DeviceSystemBatch(b), lay, b)
    part = b.subset(13, 20)
    sub = engine.prefilter_device(engine.DeviceSystemBatch(part), lay, part)
    for k in STATS:
        assert np.array_equal(getattr(whole, k), getattr(again, k))
        assert np.array_equal(getattr(whole, k)[13:33], getattr(sub, k))
