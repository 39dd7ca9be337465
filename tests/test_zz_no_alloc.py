"""ichol_solve_noalloc against the allocating ichol_solve entry point.

The no-allocation IC(0) solve keeps its scratch in a fixed device array of
the library; two calls in a row must both reproduce ichol_solve's result
(bit-identical: the same operations in the same order), and sizes beyond
the array are rejected with AMG_ERR_ARG.
"""
import ctypes as C

import numpy as np
import pytest

from blood_network_b200 import amg, network

pytestmark = pytest.mark.gpu

MAX_ROWS = 131072


def _factor(lib, net):
    A = amg.DcsrMat(net.n, net.n, net.nnz,
                    net.indptr.ctypes.data_as(C.POINTER(C.c_int)),
                    net.indices.ctypes.data_as(C.POINTER(C.c_int)),
                    net.data.ctypes.data_as(C.POINTER(C.c_double)))
    f = amg.IcholFactor()
    lib.ichol_compute(C.byref(A), C.byref(f))
    assert lib.amg_solver_last_status() == 0, lib.amg_solver_last_error()
    ia = np.ctypeslib.as_array(f.ia, shape=(f.n + 1,)).copy()
    ja = np.ctypeslib.as_array(f.ja, shape=(f.nnz,)).copy()
    val = np.ctypeslib.as_array(f.val, shape=(f.nnz,)).copy()
    return f, ia, ja, val


@pytest.mark.parametrize("n_nodes,depth", [(5_000, 8), (100_000, 12)])
def test_noalloc_matches_ichol_solve(n_nodes, depth):
    import torch
    lib = amg.load_library()
    net = network.vascular_network(depth=depth, n_nodes=n_nodes, seed=3)
    assert net.n <= MAX_ROWS
    f, ia, ja, val = _factor(lib, net)
    dev = torch.device("cuda:0")
    d_ia = torch.from_numpy(ia).to(dev)
    d_ja = torch.from_numpy(ja).to(dev)
    d_val = torch.from_numpy(val).to(dev)
    stream = torch.cuda.current_stream(dev)
    rng = np.random.default_rng(11)
    try:
        for call in range(2):
            b = rng.standard_normal(net.n)
            want = np.zeros(net.n)
            lib.ichol_solve(C.byref(f), amg._p(b), amg._p(want))
            assert lib.amg_solver_last_status() == 0, lib.amg_solver_last_error()
            d_b = torch.from_numpy(b).to(dev)
            d_x = torch.full((net.n,), float("nan"), dtype=torch.float64, device=dev)
            torch.cuda.synchronize()
            rc = lib.ichol_solve_noalloc(net.n, C.c_void_p(d_ia.data_ptr()),
                                         C.c_void_p(d_ja.data_ptr()),
                                         C.c_void_p(d_val.data_ptr()),
                                         C.c_void_p(d_b.data_ptr()),
                                         C.c_void_p(d_x.data_ptr()),
                                         C.c_void_p(stream.cuda_stream))
            assert rc == 0, lib.amg_solver_last_error()
            torch.cuda.synchronize()
            got = d_x.cpu().numpy()
            # same arithmetic in the same order: tolerance 0 (bit-identical)
            assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), call
    finally:
        lib.ichol_free(C.byref(f))


def test_noalloc_rejects_oversize_and_empty():
    import torch
    lib = amg.load_library()
    dev = torch.device("cuda:0")
    one = torch.zeros(4, dtype=torch.float64, device=dev)
    p = C.c_void_p(one.data_ptr())
    rc = lib.ichol_solve_noalloc(MAX_ROWS + 1, p, p, p, p, p, None)
    assert rc == -1
    assert b"131072" in lib.amg_solver_last_error()
    assert lib.ichol_solve_noalloc(-1, p, p, p, p, p, None) == -1
    assert lib.ichol_solve_noalloc(0, None, None, None, None, None, None) == 0
    assert lib.ichol_solve_noalloc(3, None, p, p, p, p, None) == -1
