"""TraceEngine (include/mikroptim/cuda/trace_engine.hpp): tranches sized against the device
memory, run_on_device, max_variants and the per-run settings (opd, status, extra_residuals,
extra_merit, pack_rays). Every variant's results are bit-identical whatever the split and the
pack size (the kernels do not depend on a variant's position in the batch), as the reference
requires of its engine (ADR-0007).
"""

import ctypes as C

import numpy as np
import pytest

from mikroptim_b200 import _capi, engine, workloads
from mikroptim_b200.batch import ResidualLayout
import oracle.pyoracle as po

pytestmark = pytest.mark.gpu


def singlets(n=1024):
    b, st, vs, x0 = workloads.singlet(n)
    return b, st, ResidualLayout(b.topology, st)


def per_variant_bytes(b, lay, merit, opd=1, extra=0):
    shape = engine.TraceEngine._shape(b.topology, False)
    per, fixed = C.c_size_t(0), C.c_size_t(0)
    _capi.check(_capi.lib().mkb_trace_run_bytes(C.byref(shape), C.byref(lay.plan(b)), merit,
                                                0, opd, extra, C.byref(per), C.byref(fixed)),
                "run bytes")
    return per.value, fixed.value


def small_engine(b, lay, merit, tranche, opd=1):
    per, fixed = per_variant_bytes(b, lay, merit, opd)
    opts = engine.EngineOptions(memory_limit_bytes=fixed + tranche * per,
                                reserve=engine.MemoryReserve(0, 0.0))
    return engine.TraceEngine(0, opts)


def test_tranches_bit_identical_to_one_run():
    b, st, lay = singlets(1024)
    ts = engine.TraceSettings(st, opd=True)
    whole = engine.TraceEngine(0).run(b, engine.TraceMode.RESIDUALS, ts)
    assert whole.info.tranches == 1
    eng = small_engine(b, lay, 0, 300)
    split = eng.run(b, engine.TraceMode.RESIDUALS, ts)
    assert split.info.tranches == 4 and split.info.tranche_variants == 300
    for k in ("residuals", "opd", "status"):
        assert np.array_equal(getattr(split.residuals, k), getattr(whole.residuals, k)), k
    ro, oo, so = po.port().residuals(b, lay, threads=8)
    assert np.array_equal(split.residuals.residuals, ro)
    m_whole = engine.TraceEngine(0).run(b, engine.TraceMode.MERIT, ts)
    m_split = small_engine(b, lay, 1, 250, opd=0).run(b, engine.TraceMode.MERIT, ts)
    assert m_split.info.tranches == 5
    for k in ("merit", "failed", "hard_failed"):
        assert np.array_equal(getattr(m_split.merit, k), getattr(m_whole.merit, k)), k


def test_pack_rays_changes_nothing():
    b, st, vs, x0 = workloads.objective(8, rings=4, spokes=8)
    lay = ResidualLayout(b.topology, st)
    eng = engine.TraceEngine(0)
    outs = [eng.run(b, engine.TraceMode.RESIDUALS,
                    engine.TraceSettings(st, opd=True, pack_rays=k)).residuals
            for k in (1, 37, 512, 100000)]
    merits = [eng.run(b, engine.TraceMode.MERIT, engine.TraceSettings(st, pack_rays=k)).merit
              for k in (1, 37, 512, 100000)]
    for o in outs[1:]:
        assert np.array_equal(o.residuals, outs[0].residuals)
        assert np.array_equal(o.opd, outs[0].opd) and np.array_equal(o.status, outs[0].status)
    for m in merits[1:]:
        assert np.array_equal(m.merit, merits[0].merit)


def test_extra_residuals_and_extra_merit():
    b, st, lay = singlets(64)
    eng = engine.TraceEngine(0)
    base = eng.run(b, engine.TraceMode.RESIDUALS, st).residuals
    more = eng.run(b, engine.TraceMode.RESIDUALS,
                   engine.TraceSettings(st, extra_residuals=5)).residuals
    assert more.stride == lay.trace_rows + 5 and base.stride == lay.trace_rows
    assert np.array_equal(more.residuals[:, :lay.trace_rows], base.residuals)
    assert np.all(more.residuals[:, lay.trace_rows:] == 0.0)
    assert base.opd.size == 0 and base.status.shape == (64, lay.rays_per_variant)
    quiet = eng.run(b, engine.TraceMode.RESIDUALS, engine.TraceSettings(st, status=False))
    assert quiet.residuals.status.size == 0 and quiet.merit.variants == 0
    extra = np.random.default_rng(5).uniform(0.0, 3.0, 64)
    m0 = eng.run(b, engine.TraceMode.MERIT, st).merit
    m1 = eng.run(b, engine.TraceMode.MERIT, engine.TraceSettings(st, extra_merit=extra)).merit
    assert np.array_equal(m1.merit, m0.merit + extra)  # one rounded add after the tuple sums
    with pytest.raises(ValueError):
        eng.run(b, engine.TraceMode.MERIT, engine.TraceSettings(st, extra_merit=extra[:3]))


def test_run_on_device_tranches_keep_groups_together():
    b, st, lay = singlets(200)
    want = engine.TraceEngine(0).run(b, engine.TraceMode.RESIDUALS,
                                     engine.TraceSettings(st, opd=True)).residuals
    eng = small_engine(b, lay, 0, 50)
    got = np.zeros_like(want.residuals)
    seen = []

    def consume(t):
        assert t.count % 7 == 0 or t.first + t.count == 200
        seen.append((t.first, t.count))
        got[t.first:t.first + t.count] = t.residuals.cpu().numpy()
        assert np.array_equal(t.status.cpu().numpy(), want.status[t.first:t.first + t.count])

    info = eng.run_on_device(b, engine.TraceSettings(st, opd=True), 7, consume)
    assert info.tranche_variants == 49 and info.tranches == 5
    assert seen[0] == (0, 49) and seen[-1] == (196, 4)
    assert np.array_equal(got, want.residuals)
    with pytest.raises(ValueError):
        eng.run_on_device(b, st, 0, consume)


def test_max_variants_and_out_of_memory():
    b, st, lay = singlets(64)
    big = engine.TraceEngine(0).max_variants(b.topology, engine.TraceMode.RESIDUALS, st)
    assert big > 100000
    eng = small_engine(b, lay, 0, 10)
    assert eng.max_variants(b.topology, engine.TraceMode.RESIDUALS,
                            engine.TraceSettings(st, opd=True)) == 10
    tiny = engine.TraceEngine(0, engine.EngineOptions(memory_limit_bytes=1 << 20,
                                                      reserve=engine.MemoryReserve(0, 0.0)))
    assert tiny.max_variants(b.topology, engine.TraceMode.MERIT, st) == 0
    with pytest.raises(RuntimeError):
        tiny.run(b, engine.TraceMode.MERIT, st)
    with pytest.raises(ValueError):
        engine.TraceEngine(0, engine.EngineOptions(reserve=engine.MemoryReserve(0, 2.0)))
    eng.release()
    assert eng.device_bytes() == 0


def test_reused_output_and_fresh_results():
    """A loop that passes its TraceOutput back gets its results in that object's (pinned)
    arrays; a call without one gets arrays of its own that later runs leave alone."""
    b1, st, lay = singlets(64)
    b2, _, _ = singlets(100)
    eng = engine.TraceEngine(0)
    ts = engine.TraceSettings(st, opd=True)
    fresh1 = eng.run(b1, engine.TraceMode.RESIDUALS, ts).residuals
    keep = fresh1.residuals.copy()
    out = engine.TraceOutput()
    for b in (b1, b2, b1):
        got = eng.run(b, engine.TraceMode.RESIDUALS, ts, out).residuals
        want = engine.TraceEngine(0).run(b, engine.TraceMode.RESIDUALS, ts).residuals
        assert np.array_equal(got.residuals, want.residuals)
        assert np.array_equal(got.opd, want.opd) and np.array_equal(got.status, want.status)
        m = eng.run(b, engine.TraceMode.MERIT, ts, out).merit
        assert np.array_equal(m.merit, engine.TraceEngine(0).run(
            b, engine.TraceMode.MERIT, ts).merit.merit)
    assert np.array_equal(fresh1.residuals, keep)
