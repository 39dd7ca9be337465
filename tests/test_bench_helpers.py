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


def _small_net():
    from blood_network_b200.network import vascular_network
    return vascular_network(depth=6, n_nodes=3000, seed=1)


def test_reference_solve_wave_runs_forked_solves():
    import pytest
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "oracle"))
    import ref as R
    if not R.have_reference():
        pytest.skip("reference library not built")
    import bench
    import scipy.sparse as sp
    net = _small_net()
    S = R.RefSolver(net.n, net.indptr, net.indices, net.data, theta=0.5, min_size=100,
                    coarsening=2)
    x = bench.shared_vector(net.n)
    res = bench.ref_solve_wave(S, net.rhs, 1e-8, 3, 2, x_out=x)
    S.close()
    assert len(res) == 3 and all(it > 0 and t > 0 for it, t in res)
    A = sp.csr_matrix((net.data, net.indices, net.indptr), shape=(net.n, net.n))
    assert np.linalg.norm(net.rhs - A @ x) <= 1e-6 * np.linalg.norm(net.rhs)


def test_baseline_child_reports_the_reference_solve():
    import pytest
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "oracle"))
    import ref as R
    if not R.have_reference():
        pytest.skip("reference library not built")
    import bench
    net = _small_net()
    child = bench.start_baseline_child(net, {"theta": 0.5, "coarsening": "hmis"})
    out, x = bench.finish_baseline_child(child, limit_s=120)
    assert "error" not in out, out
    assert out["iterations"] > 0 and out["solve_s"] > 0 and out["setup_s"] > 0
    assert out["relres"] < 1e-6 and np.isfinite(np.asarray(x)).all()


def test_headline_config_is_shared_by_both_arms():
    import bench
    from blood_network_b200.network import CONFIGS
    c = bench.headline_config(10, 28, CONFIGS[bench.WORKLOAD])
    assert c == bench.headline_config(10, 28, CONFIGS[bench.WORKLOAD])
    assert c["workload"].startswith(bench.WORKLOAD) and "1e-8" in c["stop"]
    assert bench.host_cores() >= 1 and bench.host_mem_available() > 0
