"""The host half of the FP32 prefilter, on the CPU: the conservative decision
(mkb_prefilter_decide_host) and the FP64 truth rule (mkb_prefilter_decide_exact_host) against
the reference's prefilter_decide / prefilter_decide_exact on the reference's own per-variant
results, bit for bit, and the argument checks."""

import ctypes as C

import numpy as np
import pytest

from conftest import has_reference_build
from mikroptim_b200 import _capi, engine, workloads
from mikroptim_b200.batch import FAILURE_HARD, ResidualLayout
import oracle.pyoracle as po

STATS = ("merit", "optical_length", "failed", "uncertain_ok", "uncertain_failed")


@pytest.mark.skipif(not has_reference_build(), reason="reference CPU build missing")
@pytest.mark.parametrize("failure", [0, FAILURE_HARD])
def test_decide_host_equals_the_reference(failure):
    ref = po.reference()
    b, st, _, _ = workloads.singlet(150)
    b = workloads.multistart(b)
    st.failure = failure
    lay = ResidualLayout(b.topology, st)
    m, f, _ = ref.merit(b, lay)
    extra = np.linspace(0.0, 1.0, b.variants)
    for opt in (engine.PrefilterOptions(),
                engine.PrefilterOptions(max_failed_fraction=0.05, max_merit_factor=10.0),
                engine.PrefilterOptions(max_merit=float(np.median(m)), merit_relative=0.1,
                                        opl_error_factor=100.0)):
        for ex in (None, extra):
            want = ref.prefilter(b, lay, opt.c_struct(), ex)
            stats = engine.PrefilterStats(b.variants, lay.rays_per_variant,
                                          *[want[k] for k in STATS])
            got = engine.prefilter_decide(stats, lay, b, opt, ex)
            assert np.array_equal(got.merit_lower, want["merit_lower"])
            assert np.array_equal(got.merit_upper, want["merit_upper"])
            assert np.array_equal(got.reject, want["reject"])
            assert got.reference_merit == want["reference_merit"]
            assert got.reference_variant == want["reference_variant"]
            assert got.kept == want["kept"]
            truth = engine.prefilter_decide_exact(m, f, lay.rays_per_variant, opt, ex)
            assert np.array_equal(truth, ref.prefilter_decide_exact(opt.c_struct(), m, f,
                                                                    lay.rays_per_variant, ex))
            assert not np.any(got.reject & ~truth)


def test_decide_rejects_bad_options():
    b, st, _, _ = workloads.singlet(2)
    lay = ResidualLayout(b.topology, st)
    stats = engine.PrefilterStats(2, lay.rays_per_variant, np.ones(2), np.ones(2),
                                  np.zeros(2, np.int64), np.zeros(2, np.int64),
                                  np.zeros(2, np.int64))
    for bad in (dict(merit_relative=1.0), dict(boundary=-0.1), dict(opl_error_factor=np.nan),
                dict(max_failed_fraction=-1.0), dict(max_merit_factor=np.nan)):
        with pytest.raises(ValueError):
            engine.prefilter_decide(stats, lay, b, engine.PrefilterOptions(**bad))
    with pytest.raises(ValueError):
        engine.prefilter_decide(stats, lay, b, engine.PrefilterOptions(), np.ones(3))


def test_default_options_are_the_references():
    o = _capi.PrefilterOptions()
    _capi.lib().mkb_prefilter_default_options(C.byref(o))
    d = engine.PrefilterOptions()
    for k in ("max_failed_fraction", "max_merit", "max_merit_factor", "boundary",
              "opl_error_factor", "merit_relative"):
        assert getattr(o, k) == getattr(d, k), k


def test_field_table_uses_the_float_sine_and_cosine():
    b, st, _, _ = workloads.objective(3, rings=2, spokes=4)
    view = b.view()
    out = np.zeros((3, b.fields, 2), np.float32)
    assert _capi.lib().mkb_prefilter_field_trig_host(C.byref(view), out.ctypes.data) == 0
    theta = np.asarray(b.field_angle, dtype=np.float32)
    lib = C.CDLL("libm.so.6")
    lib.sinf.restype = lib.cosf.restype = C.c_float
    lib.sinf.argtypes = lib.cosf.argtypes = [C.c_float]
    for v in range(3):
        for f in range(b.fields):
            assert out[v, f, 0] == np.float32(lib.sinf(float(theta[v, f])))
            assert out[v, f, 1] == np.float32(lib.cosf(float(theta[v, f])))
