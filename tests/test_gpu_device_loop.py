"""PCG iterations as one CUDA graph (a conditional WHILE node whose body is
one iteration; the stopping test runs on the device) against the
host-driven loop (BN_HOST_LOOP=1): the same kernels in the same order, so
the same iterates bit for bit, the same iteration count and status."""
import os

import numpy as np
import pytest

from blood_network_b200 import amg
from blood_network_b200.network import batch_networks, block_diagonal, make_config

pytestmark = pytest.mark.gpu


def _pair(make):
    os.environ.pop("BN_HOST_LOOP", None)
    dev = make()
    os.environ["BN_HOST_LOOP"] = "1"
    try:
        host = make()
    finally:
        os.environ.pop("BN_HOST_LOOP", None)
    return dev, host


@pytest.mark.parametrize("precision", [amg.PREC_FP64, amg.PREC_MIXED])
@pytest.mark.parametrize("stop", [amg.STOP_RELRES, amg.STOP_BNORM])
def test_device_loop_equals_host_loop(precision, stop):
    net = make_config("vascular_20k")
    dev, host = _pair(lambda: amg.AMGSolver(net.n, net.indptr, net.indices, net.data,
                                            precision=precision, stop=stop))
    x1, it1 = dev.solve(net.rhs, tol=1e-8)
    s1 = dev.stats()
    x2, it2 = host.solve(net.rhs, tol=1e-8)
    s2 = host.stats()
    assert s1.device_loop == 1 and s2.device_loop == 0
    assert it1 == it2 > 0
    assert x1.tobytes() == x2.tobytes()
    # a second solve on the same graph, and maxiter reached on the device
    x3, it3 = dev.solve(net.rhs, tol=1e-8)
    assert it3 == it1 and x3.tobytes() == x1.tobytes()
    x4, it4 = dev.solve(net.rhs, tol=1e-30, maxiter=3)
    assert it4 == -3 and dev.stats().converged == 0
    dev.close()
    host.close()


def test_segmented_device_loop_equals_host_loop():
    nets = batch_networks(6, lo=2000, hi=20000, seed=3)
    n, ia, ja, val, rhs, ptr = block_diagonal(nets)
    dev, host = _pair(lambda: amg.AMGSolver(n, ia, ja, val, precision=amg.PREC_MIXED,
                                            stop=amg.STOP_RELRES))
    x1, its1, rel1, rc1 = dev.solve_segmented(ptr, rhs, tol=1e-8)
    x2, its2, rel2, rc2 = host.solve_segmented(ptr, rhs, tol=1e-8)
    assert dev.stats().device_loop == 1 and host.stats().device_loop == 0
    assert rc1 == rc2 == 0
    assert np.array_equal(its1, its2)
    assert x1.tobytes() == x2.tobytes()
    assert rel1.max() <= 1e-8
    dev.close()
    host.close()
