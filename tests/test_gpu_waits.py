"""The give-up path of the sync-free sweeps' bounded waits.

The sweeps (IC(0) forward/backward, ordered Gauss-Seidel) poll their
dependencies' values; a wait that runs out raises the sweep's abort word so
that every other waiting row ends at once, and the host reports the wait
record as AMG_ERR_SPIN.  Here a chain whose first row is left out of the
schedule makes row 1 wait for a value that nothing publishes (a flag that
nothing sets), and every later row waits for its predecessor; the launch
must end in about one limit, report a row that gave up, and leave the
device usable.
"""
import ctypes as C

import numpy as np
import pytest

from blood_network_b200 import amg


@pytest.mark.gpu
@pytest.mark.parametrize("n,limit_ms", [(2, 5.0), (5000, 20.0), (200000, 50.0)])
def test_stalled_sweep_gives_up_within_one_limit(n, limit_ms):
    lib = amg.load_library()
    ms = C.c_double(-1.0)
    rc = lib.amg_debug_wait_timeout(n, limit_ms, C.byref(ms))
    msg = lib.amg_solver_last_error().decode()
    assert rc == amg.ERR_SPIN, (rc, msg)
    # every row of the chain waits from the start; the record names the one
    # whose wait ran out first, a row waiting for its predecessor
    import re
    m = re.search(r"row (\d+) waited [0-9.]+ ms for row (\d+)", msg)
    assert m, msg
    row, dep = int(m.group(1)), int(m.group(2))
    assert 1 <= row < n and dep == row - 1, msg
    # one limit for the whole launch, not one per waiting row
    assert limit_ms * 0.9 <= ms.value <= limit_ms + 250.0, (ms.value, msg)


@pytest.mark.gpu
def test_device_usable_after_a_stalled_sweep():
    lib = amg.load_library()
    assert lib.amg_debug_wait_timeout(1000, 10.0, None) == amg.ERR_SPIN
    # a solve on the same device afterwards: its own sweeps finish normally
    import scipy.sparse as sp
    n = 3000
    rng = np.random.default_rng(3)
    u = np.arange(n - 1)
    w = rng.uniform(0.5, 1.5, n - 1)
    W = sp.coo_matrix((np.r_[w, w], (np.r_[u, u + 1], np.r_[u + 1, u])), shape=(n, n)).tocsr()
    A = (sp.diags(np.asarray(W.sum(1)).ravel() + 1e-2) - W).tocsr()
    A.sort_indices()
    b = rng.standard_normal(n)
    s = amg.AMGSolver(n, A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data,
                      stop=amg.STOP_RELRES, min_size=100)
    x, it = s.solve(b, tol=1e-8, maxiter=100)
    s.close()
    assert it > 0
    assert np.linalg.norm(b - A @ x) <= 1e-8 * np.linalg.norm(b)


@pytest.mark.gpu
def test_wait_selftest_rejects_bad_arguments():
    lib = amg.load_library()
    assert lib.amg_debug_wait_timeout(1, 10.0, None) == amg.ERR_ARG
    assert lib.amg_debug_wait_timeout(100, 0.0, None) == amg.ERR_ARG
    assert lib.amg_debug_wait_timeout(100, 1e6, None) == amg.ERR_ARG
