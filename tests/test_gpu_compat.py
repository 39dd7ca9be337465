"""The reference's internal hierarchy API (amg_build_hierarchy, amg_vcycle_precond,
amg_ichol_precond, amg_backslash/fwdslash, amg_pcg with a host callback) through
the C ABI, on the 20k-node network.

amg_build_hierarchy must fill the reference's amg_data with the same levels as
the reference (checked against the oracle bit for bit); the preconditioners,
driven through amg_pcg exactly as the reference's wrapper drives them, must
converge like the reference's solver does.
"""
import ctypes as C

import numpy as np
import pytest

from blood_network_b200 import amg
from blood_network_b200.network import make_config

from helpers import bits_equal, relres

pytestmark = pytest.mark.gpu


def _arr(ptr, n, dtype):
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


def _host_csr(m: amg.DcsrMat):
    return (_arr(m.ia, m.row + 1, np.int32), _arr(m.ja, m.nnz, np.int32),
            _arr(m.val, m.nnz, np.float64))


def _dcsr(ia, ja, val, n):
    return amg.DcsrMat(n, n, int(ia[-1]), ia.ctypes.data_as(C.POINTER(C.c_int)),
                       ja.ctypes.data_as(C.POINTER(C.c_int)),
                       val.ctypes.data_as(C.POINTER(C.c_double)))


@pytest.fixture(scope="module")
def built():
    lib = amg.load_library()
    net = make_config("vascular_20k")
    ia, ja, val = (np.ascontiguousarray(net.indptr), np.ascontiguousarray(net.indices),
                   np.ascontiguousarray(net.data))
    A = _dcsr(ia, ja, val, net.n)
    d = amg.AmgData()
    d.threshold, d.min_size, d.max_levels, d.nu = 0.25, 500, 20, 1
    d.smoother, d.omega_jacobi, d.coarsening = amg.SMOOTHER_CF_GS, 0.5, amg.COARSEN_PMIS
    lib.amg_build_hierarchy(C.byref(d), C.byref(A))
    assert lib.amg_solver_last_status() == 0, lib.amg_solver_last_error()
    yield lib, net, d, A, (ia, ja, val)
    lib.amg_free(C.byref(d))


def test_hierarchy_fields_match_reference(built, oracle):
    lib, net, d, _, _ = built
    ref = oracle.OracleSolver(net.n, net.indptr, net.indices, net.data, theta=0.25,
                              coarsening=1, smoother=2)
    try:
        assert d.num_levels == ref.num_levels
        for k in range(d.num_levels):
            L = d.levels[k]
            R = ref.level(k)
            assert L.n == R["n"]
            for a, b in zip(_host_csr(L.A), R["A"]):
                assert bits_equal(a, b), k
            l1 = _arr(L.l1_diag, L.n, np.float64)
            ia, _, va = R["A"]
            want = np.array([np.sum(np.abs(va[ia[i]:ia[i + 1]])) for i in range(min(L.n, 2000))])
            np.testing.assert_allclose(l1[:len(want)], want, rtol=1e-14, atol=0)
            if k < d.num_levels - 1:
                assert L.n_coarse == R["n_coarse"]
                for a, b in zip(_host_csr(L.P), R["P"]):
                    assert bits_equal(a, b), k
                for a, b in zip(_host_csr(L.A_filtered), R["S"]):
                    assert bits_equal(a, b), k
                mis = _arr(L.mis, L.n, np.int32)
                assert np.array_equal(mis, (R["cf"] == 1).astype(np.int32))
                order = _arr(L.cf_order, L.n, np.int32)
                c = np.nonzero(R["cf"] == 1)[0]
                f = np.nonzero(R["cf"] != 1)[0]
                assert np.array_equal(order, np.concatenate([c, f]))
                assert not _arr(L.isolated, L.n, np.int32).any()
        # coarsest level: its IC(0) factor, bit for bit
        last = d.levels[d.num_levels - 1]
        Lr = oracle.orc_ichol(last.n, *_host_csr(last.A))
        f = last.L_ichol
        got = (_arr(f.ia, f.n + 1, np.int32), _arr(f.ja, f.nnz, np.int32),
               _arr(f.val, f.nnz, np.float64))
        for a, b in zip(got, Lr):
            assert bits_equal(a, b)
    finally:
        ref.close()


def _pcg(lib, A, b, fn, tol=1e-8, maxiter=200):
    x = np.zeros(len(b))
    cb = amg.PRECOND_FN(fn)
    it = lib.amg_pcg(C.byref(A), amg._p(b), amg._p(x), cb, None, tol, maxiter, 0)
    return x, it


def test_pcg_with_host_callbacks(built, oracle):
    lib, net, d, A, (ia, ja, val) = built
    b = np.ascontiguousarray(net.rhs)
    n = net.n

    # plain CG (identity callback) on a well-conditioned tridiagonal system
    m = 200
    tia = np.arange(0, 3 * m - 1, 3, dtype=np.int32)
    rows = [np.array([j for j in (i - 1, i, i + 1) if 0 <= j < m], np.int32) for i in range(m)]
    tia = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int32)
    tja = np.concatenate(rows).astype(np.int32)
    tval = np.concatenate([np.where(r == i, 4.0, -1.0) for i, r in enumerate(rows)])
    T = _dcsr(tia, tja, tval, m)
    tb = np.random.default_rng(3).standard_normal(m)

    def identity(data, g, bg):
        C.memmove(bg, g, 8 * m)
    tx, it = _pcg(lib, T, tb, identity, tol=1e-10, maxiter=500)
    assert 0 < it < 100
    assert relres(tia, tja, tval, tx, tb) < 1e-8

    def vcycle(data, g, bg):
        lib.amg_vcycle_precond(C.byref(d), C.cast(g, C.c_void_p), C.cast(bg, C.c_void_p))
    x, it_v = _pcg(lib, A, b, vcycle, maxiter=1000)
    assert it_v > 0
    assert relres(ia, ja, val, x, b) < 1e-6

    # the reference wrapper's preconditioner: AMG + IC(0) of the fine matrix
    f = amg.IcholFactor()
    lib.ichol_compute(C.byref(A), C.byref(f))

    def amg_ichol(data, g, bg):
        lib.amg_ichol_precond(C.byref(d), C.byref(A), C.byref(f), C.cast(g, C.c_void_p),
                              C.cast(bg, C.c_void_p))
    try:
        x, it_i = _pcg(lib, A, b, amg_ichol)
        ref = oracle.OracleSolver(n, net.indptr, net.indices, net.data, theta=0.25,
                                  coarsening=1, smoother=2)
        _, it_ref = ref.solve(b, tol=1e-8)
        ref.close()
        assert 0 < it_i <= it_ref + 2, (it_i, it_ref)
        assert relres(ia, ja, val, x, b) < 1e-7
    finally:
        lib.ichol_free(C.byref(f))
    # the hierarchy's own level-0 matrix as A (no second copy on the device)
    f2 = amg.IcholFactor()

    def amg_ichol_own(data, g, bg):
        lib.amg_ichol_precond(C.byref(d), C.byref(d.levels[0].A), C.byref(f2),
                              C.cast(g, C.c_void_p), C.cast(bg, C.c_void_p))
    lib.ichol_compute(C.byref(d.levels[0].A), C.byref(f2))
    try:
        x, it_o = _pcg(lib, d.levels[0].A, b, amg_ichol_own)
        assert 0 < it_o <= it_ref + 2
    finally:
        lib.ichol_free(C.byref(f2))


def test_vcycle_is_backslash_then_fwdslash(built):
    lib, net, d, A, (ia, ja, val) = built
    import scipy.sparse as sp
    M = sp.csr_matrix((val, ja, ia), shape=(net.n, net.n))
    g = M @ np.random.default_rng(5).standard_normal(net.n)
    x = np.zeros(net.n)
    lib.amg_vcycle_precond(C.byref(d), amg._p(g), amg._p(x))
    u = np.zeros(net.n)
    lib.amg_backslash(C.byref(d), 0, amg._p(g), amg._p(u), 1)
    r = g - M @ u
    c = np.zeros(net.n)
    lib.amg_fwdslash(C.byref(d), 0, amg._p(r), amg._p(c), 1)
    assert np.linalg.norm(u + c - x) <= 1e-8 * np.linalg.norm(x)
    # level 1: the slashes accept an initial guess
    n1 = d.levels[1].n
    b1 = np.random.default_rng(6).standard_normal(n1)
    x1 = np.zeros(n1)
    lib.amg_backslash(C.byref(d), 1, amg._p(b1), amg._p(x1), 1)
    x2 = x1.copy()
    lib.amg_fwdslash(C.byref(d), 1, amg._p(b1), amg._p(x2), 1)
    A1 = sp.csr_matrix((_host_csr(d.levels[1].A)[2], _host_csr(d.levels[1].A)[1],
                        _host_csr(d.levels[1].A)[0]), shape=(n1, n1))
    assert np.linalg.norm(b1 - A1 @ x2) < np.linalg.norm(b1 - A1 @ x1)


def test_rebuild_and_free(built, oracle):
    """amg_rebuild_values with changed values (every segment's conductance
    scaled by U(0.8, 1.25)): every level's A and P bit-identical to the
    reference's amg_rebuild_values (build_hierarchy.c:170-242) on the same
    matrices; then the original values again restore the original levels."""
    if not oracle.have_reference():
        pytest.skip("reference library not built")
    from blood_network_b200.network import assemble
    lib, net, d, A, _ = built
    before = [_host_csr(d.levels[k].A)[2].copy() for k in range(d.num_levels)]
    rng = np.random.default_rng(7)
    g2 = net.conductance * rng.uniform(0.8, 1.25, net.conductance.shape[0])
    new = assemble(net.n_total, net.seg_u, net.seg_v, g2, net.boundary, net.p_boundary)
    ia2, ja2, val2 = (np.ascontiguousarray(new.indptr), np.ascontiguousarray(new.indices),
                      np.ascontiguousarray(new.data))
    A2 = _dcsr(ia2, ja2, val2, net.n)
    lib.amg_rebuild_values(C.byref(d), C.byref(A2))
    assert lib.amg_solver_last_status() == 0, lib.amg_solver_last_error()
    r = oracle.RefSolver(net.n, net.indptr, net.indices, net.data, theta=0.25, min_size=500,
                         coarsening=1)
    r.update(ia2, ja2, val2)
    try:
        assert d.num_levels == r.num_levels
        for k in range(d.num_levels):
            want = r.level(k)
            got = _host_csr(d.levels[k].A)
            for j in range(3):
                assert bits_equal(got[j], want["A"][j]), ("A", k, j)
            if k < d.num_levels - 1:
                gotp = _host_csr(d.levels[k].P)
                for j in range(3):
                    assert bits_equal(gotp[j], want["P"][j]), ("P", k, j)
    finally:
        r.close()
    changed = sum(not bits_equal(_host_csr(d.levels[k].A)[2], before[k])
                  for k in range(d.num_levels))
    assert changed == d.num_levels
    lib.amg_rebuild_values(C.byref(d), C.byref(A))
    for k in range(d.num_levels):
        assert bits_equal(_host_csr(d.levels[k].A)[2], before[k])
    tmp = amg.AmgData()
    tmp.threshold, tmp.min_size, tmp.max_levels, tmp.nu = 0.25, 500, 20, 1
    tmp.smoother, tmp.coarsening = amg.SMOOTHER_CF_GS, amg.COARSEN_PMIS
    lib.amg_build_hierarchy(C.byref(tmp), C.byref(A))
    assert tmp.num_levels == d.num_levels
    lib.amg_free(C.byref(tmp))
    assert tmp.num_levels == 0
    lib.amg_free(C.byref(tmp))  # a second free is harmless
