"""The bench's accuracy check (after the reference's tests/test_bench_validation.py:6-11): a shape
mismatch or a non-finite value raises instead of being reported, bins below the floor are
ignored, and the measure is the max relative error over the kept bins. CPU only."""

import numpy as np
import pytest

import bench


def test_rel_err_rejects_shape_error_and_nonfinite_values():
    ref = np.ones((2, 20), dtype=np.float64)
    with pytest.raises(RuntimeError, match="shape"):
        bench.rel_err_bins(ref[:, :-1], ref)
    with pytest.raises(RuntimeError, match="non-finite"):
        bench.rel_err_bins(np.full_like(ref, np.nan), ref)
    with pytest.raises(RuntimeError, match="non-finite"):
        bench.rel_err_bins(np.where(np.arange(20) == 3, np.inf, ref), ref)


def test_rel_err_measures_kept_bins_per_row():
    ref = np.array([[1.0, 0.5, 1e-9, 2.0], [4.0, 1e-12, 1.0, 2.0]])
    got = ref.copy()
    got[0, 1] *= 1 + 3e-6   # kept: 3e-6 relative
    got[0, 2] *= 2.0        # below 1e-6 of row 0's peak: ignored
    got[1, 1] = 1.0         # below 1e-6 of row 1's peak: ignored
    got[1, 2] *= 1 - 5e-6   # kept: the largest kept error
    assert bench.rel_err_bins(got, ref) == pytest.approx(5e-6, rel=1e-6)
    assert bench.rel_err_bins(ref, ref) == 0.0
    assert bench.rel_err_bins(np.zeros((2, 0)), np.zeros((2, 0))) == 0.0
    assert bench.ACCURACY_BAR == 1e-5
