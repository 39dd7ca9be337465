"""Gauss-Seidel in a given visiting order (the MATLAB gateway cf_gauss_seidel_mex's
computation, Matlab_amg/cf_gauss_seidel_mex.c:58-101) on the device, against the
sequential sweep written out in Python: bit for bit."""
import ctypes as C

import numpy as np
import pytest

from blood_network_b200 import amg
from blood_network_b200.network import make_config, vascular_network

pytestmark = pytest.mark.gpu


def sequential(ia, ja, val, b, x0, order, nu, backward):
    n = len(b)
    x = x0.copy()
    d = np.ones(n)
    for i in range(n):
        for k in range(ia[i], ia[i + 1]):
            if ja[k] == i:
                d[i] = val[k]
                break
    seq = order[::-1] if backward else order
    for _ in range(nu):
        for i in seq:
            s = b[i]
            for k in range(ia[i], ia[i + 1]):
                j = ja[k]
                if j != i:
                    s -= val[k] * x[j]
            x[i] = s / d[i]
    return x


def device(ia, ja, val, b, x0, order, nu, backward):
    lib = amg.load_library()
    x = np.array(x0, dtype=np.float64, copy=True)
    o = np.ascontiguousarray(order, dtype=np.int32)
    rc = lib.amg_gauss_seidel_ordered(len(b), int(ia[-1]), amg._p(ia), amg._p(ja), amg._p(val),
                                      amg._p(b), amg._p(x), amg._p(o), nu, backward)
    return rc, x


@pytest.mark.parametrize("backward,nu", [(0, 1), (1, 1), (0, 2)])
def test_cf_order_bit_exact(backward, nu):
    net = vascular_network(depth=8, n_nodes=3000, seed=4)
    ia, ja, val = net.indptr, net.indices, net.data
    rng = np.random.default_rng(1)
    b = rng.standard_normal(net.n)
    x0 = rng.standard_normal(net.n)
    cf = rng.random(net.n) < 0.3  # a C/F split: C points first, then F points
    order = np.concatenate([np.nonzero(cf)[0], np.nonzero(~cf)[0]]).astype(np.int32)
    want = sequential(ia, ja, val, b, x0, order, nu, backward)
    rc, got = device(ia, ja, val, b, x0, order, nu, backward)
    assert rc == 0
    assert got.tobytes() == want.tobytes()


def test_natural_order_on_20k():
    net = make_config("vascular_20k")
    ia, ja, val = net.indptr, net.indices, net.data
    b = np.ascontiguousarray(net.rhs)
    x0 = np.zeros(net.n)
    order = np.arange(net.n, dtype=np.int32)
    want = sequential(ia, ja, val, b, x0, order, 1, 0)
    rc, got = device(ia, ja, val, b, x0, order, 1, 0)
    assert rc == 0 and got.tobytes() == want.tobytes()


def test_rejects_a_non_permutation():
    net = vascular_network(depth=5, n_nodes=200, seed=2)
    order = np.zeros(net.n, dtype=np.int32)
    rc, _ = device(net.indptr, net.indices, net.data, np.ones(net.n), np.zeros(net.n), order, 1, 0)
    assert rc == -1
