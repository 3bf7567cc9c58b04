"""The reference's interleaved state layout Q[f::nvars, f::nvars, f::nvars]
(src/Classes.py:30-34, :253-259, :476-482) against the dense one (no GPU)."""
import numpy as np
import pytest

from pyspectral_b200.Classes import from_stride3, to_stride3


@pytest.mark.parametrize("nv", [3, 6, 12])
def test_stride_round_trip(nv):
    rng = np.random.default_rng(nv)
    Q = rng.standard_normal((nv, 4, 5, 3)) + 1j * rng.standard_normal((nv, 4, 5, 3))
    Q3 = to_stride3(Q)
    assert Q3.shape == (4 * nv, 5 * nv, 3 * nv)
    assert np.array_equal(Q3[2::nv, 2::nv, 2::nv], Q[2])
    assert np.array_equal(from_stride3(Q3, nv), Q)
    assert np.count_nonzero(Q3) == Q.size
