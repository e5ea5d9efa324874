"""Host-side LM argument checks (no GPU): start points outside the variable bounds are
rejected before any device work, as the reference's VariableSet validation does."""

import numpy as np
import pytest

from mikroptim_b200 import workloads
from mikroptim_b200.engine import check_start_points, pad_rows


def test_start_points_inside_bounds_pass():
    b, st, vs, x0 = workloads.singlet(4)
    check_start_points(vs, x0)


def test_start_point_below_a_bound_is_rejected():
    b, st, vs, x0 = workloads.singlet(4)
    x = x0.copy()
    x[2, 2] = vs.lower()[2] - 1e-9
    with pytest.raises(ValueError, match="run 2, variable 2"):
        check_start_points(vs, x)


def test_per_run_sets_and_padded_rows():
    b, st, vss, x0 = workloads.uneven(12, rings=2, spokes=4)
    rows = pad_rows(x0, 12, max(v.size for v in vss))
    check_start_points(vss, rows)
    assert rows.shape == (12, max(v.size for v in vss))
    assert all(np.array_equal(rows[i, :len(r)], r) for i, r in enumerate(x0))
    rows[5, 0] = vss[5].upper()[0] * 2
    with pytest.raises(ValueError, match="run 5"):
        check_start_points(vss, rows)
