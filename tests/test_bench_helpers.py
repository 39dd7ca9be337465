"""Host helpers of bench.py that need no GPU."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def test_solution_rel_error():
    import torch
    import bench
    ref = torch.tensor([3.0, 4.0], dtype=torch.float64)
    assert bench.solution_rel_error(ref.clone(), ref) == 0.0
    assert abs(bench.solution_rel_error(torch.tensor([3.0, 4.5], dtype=torch.float64), ref)
               - 0.1) < 1e-15
    assert bench.solution_rel_error(ref, torch.zeros(2, dtype=torch.float64)) is None
    assert bench.solution_rel_error(ref, "not a tensor") is None


def test_peaks_fallback_or_measured():
    import bench
    peak, kind = bench.peaks()
    assert peak > 1000 and kind in ("measured", "fallback")
    assert np.isfinite(peak)
