"""Batched solves: many right-hand sides on one hierarchy
(amg_solver_solve_batch), and many independent networks packed
block-diagonally, each with its own PCG (amg_solver_solve_segmented).
The segmented PCG's per-segment result is checked against a separate solve of
that network on its own and against scipy residuals."""
import numpy as np
import pytest

from helpers import relres
from blood_network_b200 import amg
from blood_network_b200.network import block_diagonal, make_config, vascular_network


def _nets():
    sizes = [(6, 900), (7, 2500), (8, 6000), (6, 1500), (9, 12000)]
    return [vascular_network(depth=d, n_nodes=m, seed=10 + k) for k, (d, m) in enumerate(sizes)]


def test_block_diagonal_layout():
    nets = _nets()
    n, ia, ja, val, rhs, ptr = block_diagonal(nets)
    assert n == sum(nt.n for nt in nets) and ptr[-1] == n and len(ptr) == len(nets) + 1
    for k, nt in enumerate(nets):
        r0, r1 = ptr[k], ptr[k + 1]
        blk = ja[ia[r0]:ia[r1]]
        assert blk.min() >= r0 and blk.max() < r1
        assert np.array_equal(val[ia[r0]:ia[r1]], nt.data)
        assert np.array_equal(rhs[r0:r1], nt.rhs)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [amg.PREC_FP64, amg.PREC_MIXED])
def test_batch_columns_equal_single_solves(precision):
    net = make_config("vascular_20k")
    rng = np.random.default_rng(3)
    k = 5
    B = rng.uniform(0.5, 1.5, (net.n, k)) * net.rhs[:, None]
    S = amg.AMGSolver(net.n, net.indptr, net.indices, net.data, precision=precision)
    X, its = S.solve_batch(B, tol=1e-8, maxiter=100)
    assert X.shape == (net.n, k)
    for j in range(k):
        x, it = S.solve(B[:, j].copy(), tol=1e-8, maxiter=100)
        assert it == its[j] and it > 0
        assert X[:, j].tobytes() == x.tobytes()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [amg.PREC_FP64, amg.PREC_MIXED])
def test_segmented_solves_each_network(precision):
    nets = _nets()
    n, ia, ja, val, rhs, ptr = block_diagonal(nets)
    S = amg.AMGSolver(n, ia, ja, val, precision=precision, stop=amg.STOP_RELRES)
    tol = 1e-8
    x, its, rel, rc = S.solve_segmented(ptr, rhs, tol=tol, maxiter=200)
    assert rc == 0 and S.stats().solve_seconds > 0
    for k, nt in enumerate(nets):
        r0, r1 = ptr[k], ptr[k + 1]
        xs = x[r0:r1]
        got = relres(nt.indptr, nt.indices, nt.data, xs, nt.rhs)
        assert got < tol and abs(got - rel[k]) <= 1e-3 * tol + 1e-6 * got
        # the same network solved on its own: same tolerance, similar work
        Sk = amg.AMGSolver(nt.n, nt.indptr, nt.indices, nt.data, precision=precision,
                           stop=amg.STOP_RELRES)
        xk, itk = Sk.solve(nt.rhs, tol=tol, maxiter=200)
        assert itk > 0 and abs(int(its[k]) - itk) <= max(3, itk // 3)
        # two solutions of residual < tol differ by up to cond(A) * tol
        assert np.linalg.norm(xs - xk) <= 1e-4 * np.linalg.norm(xk)


@pytest.mark.gpu
def test_segmented_single_segment_matches_plain_solve():
    net = make_config("vascular_20k")
    S = amg.AMGSolver(net.n, net.indptr, net.indices, net.data)
    x1, it1 = S.solve(net.rhs, tol=1e-8, maxiter=100)
    x2, its, rel, rc = S.solve_segmented([0, net.n], net.rhs, tol=1e-8, maxiter=100)
    assert rc == 0 and its[0] == it1
    assert np.linalg.norm(x2 - x1) <= 1e-9 * np.linalg.norm(x1)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [amg.PREC_FP64, amg.PREC_MIXED])
def test_segments_do_not_interact(precision):
    nets = _nets()[:3]
    n, ia, ja, val, rhs, ptr = block_diagonal(nets)
    rhs = rhs.copy()
    rhs[ptr[1]:ptr[2]] = 0.0  # network 1: b = 0, x0 = 0 -> already solved
    S = amg.AMGSolver(n, ia, ja, val, precision=precision)
    x, its, rel, rc = S.solve_segmented(ptr, rhs, tol=1e-8, maxiter=200)
    assert rc == 0 and its[1] == 0 and not np.any(x[ptr[1]:ptr[2]])
    assert its[0] > 0 and its[2] > 0
    # other right-hand sides in networks 1 and 2 (so they iterate and stop
    # differently) leave network 0's iterates bit for bit as they were
    rhs2 = rhs.copy()
    rng = np.random.default_rng(5)
    rhs2[ptr[1]:] = nets[1].rhs.tolist() + (rng.uniform(0.5, 1.5, ptr[3] - ptr[2])
                                            * rhs[ptr[2]:]).tolist()
    x2, its2, _, rc2 = S.solve_segmented(ptr, rhs2, tol=1e-8, maxiter=200)
    assert rc2 == 0 and its2[1] > 0
    assert its2[0] == its[0] and x2[:ptr[1]].tobytes() == x[:ptr[1]].tobytes()
    # and a repeat is deterministic
    x3, its3, _, _ = S.solve_segmented(ptr, rhs, tol=1e-8, maxiter=200)
    assert x3.tobytes() == x.tobytes() and np.array_equal(its, its3)


@pytest.mark.gpu
def test_segmented_errors():
    nets = _nets()[:2]
    n, ia, ja, val, rhs, ptr = block_diagonal(nets)
    S = amg.AMGSolver(n, ia, ja, val)
    with pytest.raises(amg.AMGError):  # splits a connected network
        S.solve_segmented([0, ptr[1] // 2, n], rhs)
    with pytest.raises(amg.AMGError):  # offsets do not end at n
        S.solve_segmented([0, ptr[1]], rhs)
    with pytest.raises(amg.AMGError):  # decreasing offsets
        S.solve_segmented([0, ptr[1], ptr[1] - 1, n], rhs)
    x, its, rel, rc = S.solve_segmented(ptr, rhs, tol=1e-12, maxiter=2)
    assert rc == -4 and np.all(its == -2)


# ------------------------------------------------------------ block PCG
def _scenarios(net, k, seed=0):
    """k boundary-pressure scenarios: inlet ~ U(10, 16) kPa, outlet ~ U(1, 3) kPa."""
    from blood_network_b200.network import assemble
    rng = np.random.default_rng(seed)
    B = np.zeros((net.n, k), order="F")
    for j in range(k):
        pb = np.array([rng.uniform(10e3, 16e3), rng.uniform(1e3, 3e3)])
        sysj = assemble(net.n_total, net.seg_u, net.seg_v, net.conductance, net.boundary, pb)
        B[:, j] = sysj.rhs
    return B


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [amg.PREC_FP64, amg.PREC_MIXED])
@pytest.mark.parametrize("stop", [amg.STOP_BNORM, amg.STOP_RELRES])
def test_block_pcg_columns(precision, stop):
    net = make_config("vascular_20k")
    k = 6  # padded to 8 inside
    B = _scenarios(net, k)
    S = amg.AMGSolver(net.n, net.indptr, net.indices, net.data, precision=precision, stop=stop)
    X, its, rel, rc = S.solve_block(B, tol=1e-8, maxiter=100)
    assert rc == 0 and X.shape == (net.n, k)
    for j in range(k):
        got = relres(net.indptr, net.indices, net.data, X[:, j], B[:, j])
        assert abs(got - rel[j]) <= 1e-3 * got + 1e-14
        if stop == amg.STOP_RELRES:
            assert got < 1e-8
        else:
            assert got < 1e-7
        x1, it1 = S.solve(B[:, j].copy(), tol=1e-8, maxiter=100)
        assert abs(int(its[j]) - it1) <= 1
        assert np.linalg.norm(X[:, j] - x1) <= 1e-5 * np.linalg.norm(x1)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [amg.PREC_FP64, amg.PREC_MIXED])
def test_block_columns_do_not_interact(precision):
    net = make_config("vascular_20k")
    B = _scenarios(net, 8, seed=3)
    S = amg.AMGSolver(net.n, net.indptr, net.indices, net.data, precision=precision)
    X1, its1, _, _ = S.solve_block(B, tol=1e-8)
    B2 = B.copy()
    B2[:, 5] *= 1.7
    B2[:, 6] = 0.0  # a zero column: converged at the start, x stays 0
    X2, its2, _, _ = S.solve_block(B2, tol=1e-8)
    for j in (0, 1, 2, 3, 4, 7):
        assert its1[j] == its2[j] and X1[:, j].tobytes() == X2[:, j].tobytes()
    assert its2[6] == 0 and not np.any(X2[:, 6])
    X3, its3, _, _ = S.solve_block(B, tol=1e-8)  # deterministic
    assert X3.tobytes() == X1.tobytes() and np.array_equal(its1, its3)


@pytest.mark.gpu
def test_block_pcg_hub_rows_and_errors():
    from test_gpu_hubs import hub_matrix
    import scipy.sparse as sp
    n, ia, ja, val = hub_matrix()
    rng = np.random.default_rng(2)
    B = rng.standard_normal((n, 3))
    S = amg.AMGSolver(n, ia, ja, val, threshold=0.5, coarsening=amg.COARSEN_HMIS, min_size=100,
                      stop=amg.STOP_RELRES)
    X, its, rel, rc = S.solve_block(B, tol=1e-8, maxiter=100)
    A = sp.csr_matrix((val, ja, ia), shape=(n, n))
    assert rc == 0
    for j in range(3):
        assert np.linalg.norm(B[:, j] - A @ X[:, j]) <= 1e-8 * np.linalg.norm(B[:, j])
    with pytest.raises(amg.AMGError):
        S.solve_block(np.zeros((n, 65)))
    X, its, rel, rc = S.solve_block(B, tol=1e-14, maxiter=2)
    assert rc == -4 and np.all(its == -2)


@pytest.mark.gpu
def test_block_ic_sweep_forms_agree():
    """The block PCG's many-column IC(0) sweeps, sync-free (default), by level
    launches (BN_BLOCK_IC_LEVELS=1) or tiled (BN_BLOCK_IC_TILES=1), compute
    every column of every row in the same operation order: the block solves
    agree bit for bit, in both precisions."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r)\n"
        "from blood_network_b200 import amg\n"
        "from blood_network_b200.network import make_config\n"
        "net = make_config('vascular_20k')\n"
        "rng = np.random.default_rng(3)\n"
        "B = np.asfortranarray(net.rhs[:, None] * rng.uniform(0.5, 1.5, (1, 40)))\n"
        "out = []\n"
        "for prec in (amg.PREC_FP64, amg.PREC_MIXED):\n"
        "    s = amg.AMGSolver(net.n, net.indptr, net.indices, net.data, precision=prec)\n"
        "    X, its, rel, rc = s.solve_block(B, tol=1e-8)\n"
        "    assert rc == 0 and rel.max() <= 1e-8\n"
        "    out.append(X)\n"
        "    s.close()\n"
        "np.save(sys.argv[1], np.stack(out))\n" % root)
    res = []
    for k, extra in enumerate([{}, {"BN_BLOCK_IC_LEVELS": "1"}, {"BN_BLOCK_IC_TILES": "1"}]):
        path = os.path.join(os.environ.get("TMPDIR", "/tmp"), f"blkic_{k}_{os.getpid()}.npy")
        env = dict(os.environ)
        env.pop("BN_BLOCK_IC_LEVELS", None)
        env.pop("BN_BLOCK_IC_TILES", None)
        env.update(extra)
        subprocess.run([sys.executable, "-c", code, path], check=True, timeout=600, env=env)
        res.append(np.load(path))
        os.remove(path)
    for r in res[1:]:
        assert r.tobytes() == res[0].tobytes()
