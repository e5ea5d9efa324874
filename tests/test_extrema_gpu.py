"""Per-surface extrema of a trace (TraceSettings::extrema; SurfaceExtremaResult and
surface_extrema_cpu, include/mikroptim/batch/batch_extrema.hpp): per variant and table surface
the largest ray height and the smallest cos I over the rays with status Ok, in RESIDUALS and in
MERIT runs, coaxial and decentered (a tilted surface's values in its own frame). The maximum
and minimum do not depend on the order of the rays, so precision FP64 gives the reference's
values bit for bit; FP64_FMA agrees within 1e-12 relative."""

import numpy as np
import pytest

from conftest import has_reference_build
from mikroptim_b200 import engine, workloads
from mikroptim_b200.batch import PRECISION_FP64_FMA, ResidualLayout, make_non_coaxial
import oracle.pyoracle as po

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_reference_build(), reason="reference build missing")]

CASES = [lambda: workloads.singlet(64), lambda: workloads.objective(8, rings=4, spokes=8),
         lambda: workloads.ghost(8)]


@pytest.mark.parametrize("make", CASES)
@pytest.mark.parametrize("mode", [engine.TraceMode.RESIDUALS, engine.TraceMode.MERIT])
def test_extrema_bitwise_equal_reference(make, mode):
    b, st, vs, x0 = make()
    lay = ResidualLayout(b.topology, st)
    want = po.reference().surface_extrema(b, lay)
    out = engine.TraceEngine(0).run(b, mode, engine.TraceSettings(st, extrema=True))
    got = out.merit.extrema if mode == engine.TraceMode.MERIT else out.residuals.extrema
    assert got.shape == (b.variants, b.surfaces, 2)
    assert np.array_equal(got, want)
    assert np.any(got[:, 1:, 0] > 0.0)  # variants without a valid ray keep the neutral 0


def test_extrema_fma_and_tranches():
    b, st, vs, x0 = workloads.objective(8, rings=4, spokes=8)
    lay = ResidualLayout(b.topology, st)
    want = po.reference().surface_extrema(b, lay)
    st.precision = PRECISION_FP64_FMA
    got = engine.TraceEngine(0).run(b, engine.TraceMode.MERIT,
                                    engine.TraceSettings(st, extrema=True)).merit.extrema
    assert np.allclose(got, want, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("mode", [engine.TraceMode.RESIDUALS, engine.TraceMode.MERIT])
def test_extrema_of_decentered_batches_bitwise_equal_reference(mode):
    """Decentered and tilted surfaces: the height and incidence in each surface's own frame
    (the reference's observer takes the state back into the tilted frame)."""
    b, st, vs, x0 = workloads.tolerancing(6, elements=3, rings=4, spokes=8)
    assert b.non_coaxial and np.any(b.decenter_tilt != 0.0)
    lay = ResidualLayout(b.topology, st)
    want = po.reference().surface_extrema(b, lay)
    out = engine.TraceEngine(0).run(b, mode, engine.TraceSettings(st, extrema=True))
    got = out.merit.extrema if mode == engine.TraceMode.MERIT else out.residuals.extrema
    assert np.array_equal(got, want)
    # the same systems made non-coaxial with no motion give the coaxial values
    s1, st1, _, _ = workloads.singlet(8)
    nc = make_non_coaxial(s1)
    lay_nc = ResidualLayout(nc.topology, st1)
    got_nc = engine.TraceEngine(0).run(nc, mode, engine.TraceSettings(st1, extrema=True))
    got_nc = got_nc.merit.extrema if mode == engine.TraceMode.MERIT else got_nc.residuals.extrema
    assert np.array_equal(got_nc, po.reference().surface_extrema(nc, lay_nc))
