"""Parity of the CUDA library (through its C ABI) with the oracle.

Setup (symmetrisation, strength, PMIS, interpolation, RAP, IC(0)) must be
bit-identical to the reference; the solve phase replaces the sequential
CF Gauss-Seidel with a multicolour one, so solutions are checked by their
true relative residual (<= 1e-8, the tolerance the metric is stated at) and
by the PCG iteration count next to the reference's.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import bits_equal, digest, level_from_golden, relres

pytestmark = pytest.mark.gpu

from blood_network_b200 import amg  # noqa: E402
from blood_network_b200.network import make_config, vascular_network  # noqa: E402


def _solver(n, ia, ja, val, **kw):
    return amg.AMGSolver(n, ia, ja, val, **kw)


@pytest.fixture(scope="module")
def net20k():
    return make_config("vascular_20k")


# ------------------------------------------------------------------ hierarchy
def test_small_golden_hierarchy_bit_exact(golden_small):
    g = golden_small
    s = _solver(int(g["n"]), g["indptr"], g["indices"], g["data"], threshold=0.25, min_size=50)
    assert s.num_levels == int(g["levels"])
    for k in range(s.num_levels):
        got, want = s.level(k), level_from_golden(g, k)
        for nm in ("A", "S", "P"):
            if want[nm] is None:
                continue
            for j in range(3):
                assert bits_equal(got[nm][j], want[nm][j]), (k, nm, j)
        if want["cf"] is not None:
            assert np.array_equal(got["cf"], want["cf"]), k
    x, it = s.solve(g["rhs"], tol=1e-8)
    assert abs(it - int(g["solve_iters"])) <= 2
    assert relres(g["indptr"], g["indices"], g["data"], x, g["rhs"]) <= 1e-8


@pytest.mark.parametrize("key,cfg", [("pmis", "vascular_20k"), ("pmis_2m", "vascular_2m")])
def test_full_hierarchy_digests(golden_digests, key, cfg):
    net = make_config(cfg)
    ref = golden_digests[key]
    s = _solver(net.n, net.indptr, net.indices, net.data, threshold=ref["theta"])
    assert s.num_levels == len(ref["levels"])
    for k, want in enumerate(ref["levels"]):
        L = s.level(k)
        assert digest(*L["A"]) == want["A"], (key, k)
        if "S" in want:
            assert digest(*L["S"]) == want["S"], (key, k)
            assert digest(*L["P"]) == want["P"], (key, k)
            assert digest(L["cf"]) == want["cf"], (key, k)
    # solve to the metric's tolerance, both precision forms
    for prec in (amg.PREC_FP64, amg.PREC_MIXED):
        s.set_precision(prec)
        s.set_stop(amg.STOP_BNORM)
        x, it = s.solve(net.rhs, tol=1e-8)
        assert 0 < it <= ref["iterations"] + 2, (prec, it, ref["iterations"])
        assert relres(net.indptr, net.indices, net.data, x, net.rhs) <= 1e-8
        s.set_stop(amg.STOP_RELRES)
        x, it = s.solve(net.rhs, tol=1e-8)
        assert it > 0 and s.stats().relres <= 1e-8
        assert relres(net.indptr, net.indices, net.data, x, net.rhs) <= 1e-8
    s.close()


# ------------------------------------------------------------------ kernels
def _dcsr(n, m, ia, ja, val):
    ia = np.ascontiguousarray(ia, np.int32)
    ja = np.ascontiguousarray(ja, np.int32)
    val = np.ascontiguousarray(val, np.float64)
    d = amg.DcsrMat(n, m, int(ia[-1]), ia.ctypes.data_as(C.POINTER(C.c_int)),
                    ja.ctypes.data_as(C.POINTER(C.c_int)),
                    val.ctypes.data_as(C.POINTER(C.c_double)))
    d._keep = (ia, ja, val)
    return d


def _out(d):
    n, nnz = d.row, d.nnz
    ia = np.ctypeslib.as_array(d.ia, shape=(n + 1,)).copy()
    ja = np.ctypeslib.as_array(d.ja, shape=(max(nnz, 1),))[:nnz].copy()
    val = np.ctypeslib.as_array(d.val, shape=(max(nnz, 1),))[:nnz].copy()
    return ia, ja, val


def test_kernel_dropins_bit_exact(oracle, net20k):
    lib = amg.load_library()
    n = net20k.n
    A = (net20k.indptr, net20k.indices, net20k.data)
    # strength
    S_ref, ml_ref = oracle.orc_strength(n, *A, 0.25)
    dS = amg.DcsrMat()
    ml = C.c_int()
    lib.rs_strength(C.byref(_dcsr(n, n, *A)), 0.25, C.byref(dS), C.byref(ml))
    assert lib.amg_solver_last_status() == 0
    S = _out(dS)
    assert ml.value == ml_ref
    for j in range(3):
        assert bits_equal(S[j], S_ref[j])
    # PMIS (glibc rand weights) and the parallel RS first pass
    cf_ref, nc_ref = oracle.orc_split(n, *S_ref, "pmis")
    cf = np.zeros(n, np.int32)
    nc = C.c_int()
    lib.pmis_coarsening(C.byref(_dcsr(n, n, *S)), amg._p(cf), C.byref(nc))
    assert nc.value == nc_ref and np.array_equal(cf, cf_ref)
    # interpolation
    P_ref = oracle.orc_interp(n, A, S_ref, cf_ref)
    dP = amg.DcsrMat()
    lib.rs_standard_interpolation(C.byref(_dcsr(n, n, *A)), C.byref(_dcsr(n, n, *S)),
                                  amg._p(cf), C.byref(dP))
    P = _out(dP)
    for j in range(3):
        assert bits_equal(P[j], P_ref[j])
    # RAP with R = P^T
    R_ref = oracle.orc_transpose(n, nc_ref, *P_ref)
    Ac_ref = oracle.orc_rap(nc_ref, n, R_ref, A, P_ref)
    dAc = amg.DcsrMat()
    lib.dcsr_rap(C.byref(_dcsr(nc_ref, n, *R_ref)), C.byref(_dcsr(n, n, *A)),
                 C.byref(_dcsr(n, nc_ref, *P_ref)), C.byref(dAc))
    Ac = _out(dAc)
    for j in range(3):
        assert bits_equal(Ac[j], Ac_ref[j])
    # IC(0) factor and solve
    L_ref = oracle.orc_ichol(n, *A)
    f = amg.IcholFactor()
    lib.ichol_compute(C.byref(_dcsr(n, n, *A)), C.byref(f))
    L = (np.ctypeslib.as_array(f.ia, shape=(n + 1,)).copy(),
         np.ctypeslib.as_array(f.ja, shape=(f.nnz,)).copy(),
         np.ctypeslib.as_array(f.val, shape=(f.nnz,)).copy())
    for j in range(3):
        assert bits_equal(L[j], L_ref[j])
    b = np.sin(np.arange(n) * 0.1)
    x = np.zeros(n)
    lib.ichol_solve(C.byref(f), amg._p(b), amg._p(x))
    assert bits_equal(x, oracle.orc_ichol_solve(n, L_ref, b))
    lib.ichol_free(C.byref(f))
    # SpMV family (row-sequential sums, the reference's order)
    xv = np.cos(np.arange(n) * 0.3)
    y = np.zeros(n)
    lib.abyvg(amg._p(A[0]), amg._p(A[1]), amg._p(A[2]), amg._p(xv), n, amg._p(y))
    assert bits_equal(y, oracle.orc_spmv(n, n, A, xv))
    z = np.zeros(n)
    lib.abyvam(amg._p(b), amg._p(A[0]), amg._p(A[1]), amg._p(A[2]), amg._p(xv), n, amg._p(z))
    assert bits_equal(z, oracle.orc_spmv(n, n, A, xv, "res", b=b))
    y2 = b.copy()
    lib.abyvcs(amg._p(A[0]), amg._p(A[1]), amg._p(A[2]), amg._p(xv), n, amg._p(y2))
    assert bits_equal(y2, oracle.orc_spmv(n, n, A, xv, "add", y0=b))
    yt = np.zeros(nc_ref)
    lib.vbya(amg._p(P_ref[0]), amg._p(P_ref[1]), amg._p(P_ref[2]), amg._p(xv), n, nc_ref,
             amg._p(yt))
    assert bits_equal(yt, oracle.orc_spmv(n, nc_ref, P_ref, xv, "t"))


# ------------------------------------------------------------------ solver paths
@pytest.mark.parametrize("coarsen,theta", [(amg.COARSEN_HMIS, 0.5), (amg.COARSEN_RS, 0.25)])
def test_parallel_first_pass_splits(oracle, net20k, coarsen, theta):
    """HMIS/RS run a parallel RS-style first pass on the device: the split is
    a valid C/F splitting and the solver converges like the reference's."""
    n = net20k.n
    s = _solver(n, net20k.indptr, net20k.indices, net20k.data, threshold=theta,
                coarsening=coarsen)
    for k in range(s.num_levels - 1):
        L = s.level(k)
        Sia, Sja, _ = L["S"]
        cf = L["cf"]
        assert set(np.unique(cf)) <= {1, -1}
        for i in np.nonzero(cf == -1)[0][::7]:
            assert np.any(cf[Sja[Sia[i]:Sia[i + 1]]] == 1), "F point without a strong C point"
    ref_it = oracle.OracleSolver(n, net20k.indptr, net20k.indices, net20k.data, theta, 500, 20,
                                 1, 2 if coarsen == amg.COARSEN_HMIS else 0).solve(
        net20k.rhs, tol=1e-8)[1]
    x, it = s.solve(net20k.rhs, tol=1e-8)
    assert relres(net20k.indptr, net20k.indices, net20k.data, x, net20k.rhs) <= 1e-8
    assert it <= ref_it + 3


def test_update_refreshes_values(net20k):
    """amg_solver_update keeps S, C/F and P's pattern and recomputes values
    (build_hierarchy.c:170-242): updating with the same matrix reproduces the
    hierarchy bit for bit; a perturbed matrix keeps the pattern and solves."""
    n = net20k.n
    s = _solver(n, net20k.indptr, net20k.indices, net20k.data)
    before = [s.level(k) for k in range(s.num_levels)]
    s.update(net20k.indptr, net20k.indices, net20k.data)
    for k in range(s.num_levels):
        after = s.level(k)
        for j in range(3):
            assert bits_equal(after["A"][j], before[k]["A"][j]), k
        if before[k]["P"] is not None:
            for j in range(3):
                assert bits_equal(after["P"][j], before[k]["P"][j]), k
    rows = np.repeat(np.arange(n), np.diff(net20k.indptr))
    a2 = net20k.data + 0.05 * np.where(net20k.indices == rows, net20k.data, 0.0)
    s.update(net20k.indptr, net20k.indices, a2)
    for k in range(s.num_levels):
        after = s.level(k)
        assert bits_equal(after["A"][0], before[k]["A"][0])   # same pattern
        if before[k]["P"] is not None:
            assert bits_equal(after["P"][1], before[k]["P"][1])
    x, it = s.solve(net20k.rhs, tol=1e-8)
    assert it > 0
    assert relres(net20k.indptr, net20k.indices, a2, x, net20k.rhs) <= 1e-8


def test_update_matches_the_reference_update(net20k, oracle):
    """amg_solver_update with changed values (every segment's conductance
    scaled by U(0.8, 1.25)) against the reference's own amg_solver_update
    (amg_wrapper.c:114-149 -> amg_rebuild_values, build_hierarchy.c:170-242)
    run on the same matrices: every level's A and P bit-identical, and the
    same iteration count after the update."""
    if not oracle.have_reference():
        pytest.skip("reference library not built")
    from blood_network_b200.network import assemble
    n = net20k.n
    rng = np.random.default_rng(5)
    g2 = net20k.conductance * rng.uniform(0.8, 1.25, net20k.conductance.shape[0])
    new = assemble(net20k.n_total, net20k.seg_u, net20k.seg_v, g2, net20k.boundary,
                   net20k.p_boundary)
    assert np.array_equal(new.indptr, net20k.indptr)
    assert np.array_equal(new.indices, net20k.indices)
    assert not np.array_equal(new.data, net20k.data)
    s = _solver(n, net20k.indptr, net20k.indices, net20k.data)
    r = oracle.RefSolver(n, net20k.indptr, net20k.indices, net20k.data, theta=0.25,
                         min_size=500, coarsening=1)
    s.update(new.indptr, new.indices, new.data)
    r.update(new.indptr, new.indices, new.data)
    assert s.num_levels == r.num_levels
    for k in range(s.num_levels):
        a, b = s.level(k), r.level(k)
        for j in range(3):
            assert bits_equal(a["A"][j], b["A"][j]), ("A", k, j)
        if b["P"] is not None:
            for j in range(3):
                assert bits_equal(a["P"][j], b["P"][j]), ("P", k, j)
    x, it = s.solve(new.rhs, tol=1e-8)
    xr, itr = r.solve(new.rhs, tol=1e-8)
    r.close()
    assert it > 0 and abs(it - itr) <= 2, (it, itr)


def test_two_matrix_mode(net20k, oracle):
    """amg_solver_set_matrix: hierarchy from Ap, IC(0) and PCG on A.  The
    three-stage preconditioner is only symmetric when both matrices agree, so
    the reference converges for nearby matrices (0.1% on the diagonal: 19
    iterations at tol 1e-10) and stalls near 1e-3 for a 5% change; the same
    holds here."""
    n = net20k.n
    s = _solver(n, net20k.indptr, net20k.indices, net20k.data)
    rows = np.repeat(np.arange(n), np.diff(net20k.indptr))
    a2 = net20k.data + 1e-3 * np.where(net20k.indices == rows, net20k.data, 0.0)
    s.set_matrix(net20k.indptr, net20k.indices, a2)
    x, it = s.solve(net20k.rhs, tol=1e-10, maxiter=300)
    assert 0 < it <= 19 + 3
    import scipy.sparse as sp
    A2 = sp.csr_matrix((a2, net20k.indices, net20k.indptr), shape=(n, n))
    A2 = 0.5 * (A2 + A2.T)
    r = np.linalg.norm(net20k.rhs - A2 @ x) / np.linalg.norm(net20k.rhs)
    assert r <= 1e-8


@pytest.mark.parametrize("smoother", [amg.SMOOTHER_L1, amg.SMOOTHER_GS, amg.SMOOTHER_JACOBI])
def test_other_smoothers_converge(net20k, smoother):
    s = _solver(net20k.n, net20k.indptr, net20k.indices, net20k.data)
    s.set_smoother(smoother, 0.5)
    x, it = s.solve(net20k.rhs, tol=1e-9, maxiter=400)
    assert it > 0
    assert relres(net20k.indptr, net20k.indices, net20k.data, x, net20k.rhs) <= 1e-8


def test_invalid_inputs_are_reported():
    lib = amg.load_library()
    ia = np.array([0, 2, 3], np.int32)
    ja = np.array([0, 0, 1], np.int32)            # duplicate column in row 0
    v = np.array([2.0, -1.0, 2.0])
    h = lib.amg_solver_create(2, 3, amg._p(ia), amg._p(ja), amg._p(v), 0.25, 1, 20, 1)
    assert not h and lib.amg_solver_last_status() == -9
    ja2 = np.array([0, 5, 1], np.int32)           # column out of range
    h = lib.amg_solver_create(2, 3, amg._p(ia), amg._p(ja2), amg._p(v), 0.25, 1, 20, 1)
    assert not h and lib.amg_solver_last_status() == -1
    ia3 = np.array([0, 3, 2], np.int32)           # decreasing row pointers
    h = lib.amg_solver_create(2, 3, amg._p(ia3), amg._p(ja), amg._p(v), 0.25, 1, 20, 1)
    assert not h and lib.amg_solver_last_status() == -1


def test_tiny_systems():
    # n below min_size: the single level is solved by the dense coarse solve
    net = vascular_network(depth=3, n_nodes=30, seed=2)
    s = _solver(net.n, net.indptr, net.indices, net.data)
    assert s.num_levels == 1
    x, it = s.solve(net.rhs, tol=1e-12)
    assert it >= 1
    assert relres(net.indptr, net.indices, net.data, x, net.rhs) <= 1e-10
    # non-converging run reports -maxiter and keeps the handle usable
    net2 = make_config("vascular_20k")
    s2 = _solver(net2.n, net2.indptr, net2.indices, net2.data)
    x2, it2 = s2.solve(net2.rhs, tol=1e-30, maxiter=2)
    assert it2 == -2
    x3, it3 = s2.solve(net2.rhs, tol=1e-8)
    assert it3 > 0


def test_bench_kernel_timings(net20k):
    s = _solver(net20k.n, net20k.indptr, net20k.indices, net20k.data)
    for which in range(4):
        for prec in (0, 1):
            assert s.bench_kernel(which, prec, reps=3) > 0.0


@pytest.mark.parametrize("precision", [amg.PREC_FP64, amg.PREC_MIXED])
def test_autotuner_choices(net20k, precision):
    """amg_solver_autotune keeps, per level operator, the fastest candidate
    (SpMV row tiles 0-3, staged tiles 5, lanes per row 4/8/16/32; GS staged
    tiles 0 or lanes 1/2/4/8/16/32), for A, R, P and the split residual
    operator; the solve still converges with the same work."""
    s = _solver(net20k.n, net20k.indptr, net20k.indices, net20k.data, precision=precision)
    x0, it0 = s.solve(net20k.rhs, tol=1e-8)
    rep = s.autotune(3)
    assert rep.shape[0] >= 3
    for lvl, op, choice, ms in rep:
        assert 0 <= lvl < s.num_levels - 1 and ms > 0
        if op == 3:
            assert choice in (0, 1, 2, 4, 8, 16, 32)  # Gauss-Seidel: staged tiles, lanes per row
        else:
            assert choice in (0, 1, 2, 3, 4, 5, 8, 16, 32)  # SpMV forms (5: staged tiles)
    x1, it1 = s.solve(net20k.rhs, tol=1e-8)
    assert abs(it1 - it0) <= 1
    assert relres(net20k.indptr, net20k.indices, net20k.data, x1, net20k.rhs) <= 1e-8
    s.close()


def test_row_tile_variants():
    """The row-tile SpMV with 256, 128, 64 or 32 rows per tile (pinned with
    BN_SPMV_GROUP) forms every row sum over the row's entries in storage
    order; only the order of the fused dot product's partial sums differs
    (the rows a thread holds), so whole solves agree to the tolerance, with
    the same iteration count, in both precisions."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r)\n"
        "from blood_network_b200 import amg\n"
        "from blood_network_b200.network import make_config\n"
        "net = make_config('vascular_20k')\n"
        "out, its = [], []\n"
        "for prec in (amg.PREC_FP64, amg.PREC_MIXED):\n"
        "    s = amg.AMGSolver(net.n, net.indptr, net.indices, net.data, precision=prec,\n"
        "                      stop=amg.STOP_RELRES)\n"
        "    x, it = s.solve(net.rhs, tol=1e-8)\n"
        "    out.append(x); its.append(it)\n"
        "np.save(sys.argv[1], np.stack(out)); np.save(sys.argv[1] + '.its.npy', np.array(its))\n"
        % root)
    res, its = [], []
    for g in ("0", "1", "2", "3", "5"):
        path = os.path.join(os.environ.get("TMPDIR", "/tmp"), f"tiles_{g}_{os.getpid()}.npy")
        subprocess.run([sys.executable, "-c", code, path], check=True, timeout=600,
                       env=dict(os.environ, BN_SPMV_GROUP=g))
        res.append(np.load(path))
        its.append(np.load(path + ".its.npy"))
        os.remove(path)
        os.remove(path + ".its.npy")
    net = make_config("vascular_20k")
    # the staged tiles (5) are the 256-row tiles (0) with bulk-copied
    # operands: same products, same sums, same dot partials, same solves
    assert res[4].tobytes() == res[0].tobytes()
    assert np.array_equal(its[4], its[0])
    for r, it in zip(res, its):
        assert np.all(np.abs(it - its[0]) <= 1)
        for x, x0 in zip(r, res[0]):
            assert relres(net.indptr, net.indices, net.data, x, net.rhs) <= 1e-8
            # two solutions of residual < 1e-8 differ by up to cond(A) * 1e-8
            assert np.linalg.norm(x - x0) <= 1e-4 * np.linalg.norm(x0)


def test_staged_gauss_seidel_equals_thread_per_row():
    """The Gauss-Seidel classes on the staged row tiles (BN_GS_LANES=0) form
    every row's sum as the thread-per-row kernel (BN_GS_LANES=1) does: the
    same preconditioner application bit for bit, in both precisions (the
    split first sweep included)."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r)\n"
        "from blood_network_b200 import amg\n"
        "from blood_network_b200.network import make_config\n"
        "net = make_config('vascular_20k')\n"
        "out = []\n"
        "for prec in (amg.PREC_FP64, amg.PREC_MIXED):\n"
        "    s = amg.AMGSolver(net.n, net.indptr, net.indices, net.data, precision=prec)\n"
        "    out.append(s.precond(net.rhs))\n"
        "    s.close()\n"
        "np.save(sys.argv[1], np.stack(out))\n" % root)
    res = []
    for g in ("1", "0"):
        path = os.path.join(os.environ.get("TMPDIR", "/tmp"), f"gs_{g}_{os.getpid()}.npy")
        subprocess.run([sys.executable, "-c", code, path], check=True, timeout=600,
                       env=dict(os.environ, BN_GS_LANES=g))
        res.append(np.load(path))
        os.remove(path)
    assert res[0].tobytes() == res[1].tobytes()


def test_ic_sweep_forms_agree():
    """Every form of the IC(0) triangular sweeps (level launches, one
    cooperative launch, chunked sync-free, tiled; BN_IC_MODE) computes each
    row in the reference's operation order, so the
    preconditioner application is bit-identical across them, in both
    precisions."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r)\n"
        "from blood_network_b200 import amg\n"
        "from blood_network_b200.network import make_config\n"
        "net = make_config('vascular_20k')\n"
        "out = []\n"
        "for prec in (amg.PREC_FP64, amg.PREC_MIXED):\n"
        "    s = amg.AMGSolver(net.n, net.indptr, net.indices, net.data, precision=prec)\n"
        "    out.append(s.precond(net.rhs))\n"
        "    s.close()\n"
        "np.save(sys.argv[1], np.stack(out))\n" % root)
    res = []
    for mode in ("flags", "levels", "coop", "tiles", "slab", "slabw"):
        path = os.path.join(os.environ.get("TMPDIR", "/tmp"), f"ic_{mode}_{os.getpid()}.npy")
        subprocess.run([sys.executable, "-c", code, path], check=True, timeout=600,
                       env=dict(os.environ, BN_IC_MODE=mode))
        res.append(np.load(path))
        os.remove(path)
    for r in res[1:]:
        assert r.tobytes() == res[0].tobytes()


def test_ic_slab_form_on_a_large_network():
    """On the 2M-node network (a slab per SM holds about one capillary-lattice
    plane; the tree generations are dealt to the slabs by rank) the slab
    form and its chunked variant are the ones that run when asked for, at
    both precisions (the staging rings fit), the sync-free form is the
    default, and both slab forms' preconditioner applications are
    bit-identical to the sync-free form's; so are the PCG iterates of a full
    solve."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r)\n"
        "from blood_network_b200 import amg\n"
        "from blood_network_b200.network import make_config\n"
        "net = make_config('vascular_2m')\n"
        "out, forms = [], []\n"
        "for prec in (amg.PREC_FP64, amg.PREC_MIXED):\n"
        "    s = amg.AMGSolver(net.n, net.indptr, net.indices, net.data, precision=prec)\n"
        "    out.append(s.precond(net.rhs))\n"
        "    out.append(s.solve(net.rhs, tol=1e-8)[0])\n"
        "    forms.append(s.stats().ichol_form)\n"
        "    s.close()\n"
        "np.save(sys.argv[1], np.stack(out))\n"
        "np.save(sys.argv[1] + '.forms.npy', np.array(forms))\n" % root)
    res, forms = [], []
    for mode in (None, "slab", "slabw"):
        path = os.path.join(os.environ.get("TMPDIR", "/tmp"), f"ic2m_{mode}_{os.getpid()}.npy")
        env = dict(os.environ)
        env.pop("BN_IC_MODE", None)
        if mode:
            env["BN_IC_MODE"] = mode
        subprocess.run([sys.executable, "-c", code, path], check=True, timeout=900, env=env)
        res.append(np.load(path))
        forms.append(np.load(path + ".forms.npy").tolist())
        os.remove(path)
        os.remove(path + ".forms.npy")
    assert forms == [[2, 2], [4, 4], [5, 5]]
    for r in res[1:]:
        assert r.tobytes() == res[0].tobytes()


def test_lanes_per_row_variants_converge():
    """Every lanes-per-row variant of the coloured Gauss-Seidel (BN_GS_LANES
    1/2/4/8/16/32) and of the group SpMV (BN_SPMV_GROUP 4/8/16/32) sums a
    row's products over its lanes with a fixed shuffle tree, so a variant
    changes only the rounding of the smoother and the coarse operators'
    products: whole solves reach the tolerance with the iteration count
    within one of the default's, in both precisions."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r)\n"
        "from blood_network_b200 import amg\n"
        "from blood_network_b200.network import make_config\n"
        "net = make_config('vascular_20k')\n"
        "its = []\n"
        "for prec in (amg.PREC_FP64, amg.PREC_MIXED):\n"
        "    s = amg.AMGSolver(net.n, net.indptr, net.indices, net.data, precision=prec,\n"
        "                      stop=amg.STOP_RELRES)\n"
        "    x, it = s.solve(net.rhs, tol=1e-8)\n"
        "    its.append(it)\n"
        "    np.save(sys.argv[1] + '.%%d.npy' %% prec, x)\n"
        "np.save(sys.argv[1], np.array(its))\n" % root)
    net = make_config("vascular_20k")
    runs = [{}] + [{"BN_GS_LANES": g} for g in ("1", "2", "4", "8", "16", "32")] + \
        [{"BN_SPMV_GROUP": g} for g in ("4", "8", "16", "32")]
    its = []
    for k, extra in enumerate(runs):
        path = os.path.join(os.environ.get("TMPDIR", "/tmp"), f"lanes_{k}_{os.getpid()}.npy")
        env = dict(os.environ)
        env.pop("BN_GS_LANES", None)
        env.pop("BN_SPMV_GROUP", None)
        env.update(extra)
        subprocess.run([sys.executable, "-c", code, path], check=True, timeout=600, env=env)
        its.append(np.load(path))
        os.remove(path)
        for prec in (0, 1):
            x = np.load(path + ".%d.npy" % prec)
            os.remove(path + ".%d.npy" % prec)
            assert relres(net.indptr, net.indices, net.data, x, net.rhs) <= 1e-8
    for it in its[1:]:
        assert np.all(np.abs(it - its[0]) <= 1)
