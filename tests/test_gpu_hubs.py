"""Graphs with hub points (rows of 10^3 entries and more, like the coarse
levels of the vessel trees): the C/F splits are decided by a block per hub
point and must equal the thread-per-point rules exactly.  PMIS against the
oracle (bit-exact with the reference); the parallel RS/HMIS first pass and
the reference's ordered second pass against a NumPy restatement below."""
import ctypes as C

import numpy as np
import pytest

from blood_network_b200 import amg


def hub_matrix(side=110, hubs=(900, 1500, 2500, 4000, 300, 700), weak_hubs=(700, 1200, 3000),
               seed=0):
    """Weighted graph Laplacian of a side x side grid plus hub nodes joined to
    many random grid nodes (diagonal = row sum + 1e-3).  The weak hubs hold
    mostly weak entries (weight 0.01) and a few strong ones (8 grid nodes and
    the next weak hub), so their rows are long but their strong sets short."""
    rng = np.random.default_rng(seed)
    m = side * side
    idx = np.arange(m).reshape(side, side)
    u = np.r_[idx[:, :-1].ravel(), idx[:-1, :].ravel()]
    v = np.r_[idx[:, 1:].ravel(), idx[1:, :].ravel()]
    for h, deg in enumerate(hubs):
        nb = rng.choice(m, deg, replace=False)
        u = np.r_[u, np.full(deg, m + h)]
        v = np.r_[v, nb]
    g = rng.uniform(0.5, 1.5, u.shape[0])
    w0 = m + len(hubs)
    for h, deg in enumerate(weak_hubs):
        nb = rng.choice(m, deg, replace=False)
        strong = np.zeros(deg)
        strong[:8] = 1.0
        u = np.r_[u, np.full(deg, w0 + h)]
        v = np.r_[v, nb]
        g = np.r_[g, np.where(strong > 0, 1.0, 0.01)]
        if h + 1 < len(weak_hubs):
            u, v, g = np.r_[u, w0 + h], np.r_[v, w0 + h + 1], np.r_[g, 1.0]
    n = w0 + len(weak_hubs)
    import scipy.sparse as sp
    W = sp.coo_matrix((np.r_[g, g], (np.r_[u, v], np.r_[v, u])), shape=(n, n)).tocsr()
    A = (sp.diags(np.asarray(W.sum(1)).ravel() + 1e-3) - W).tocsr()
    A.sort_indices()
    return n, A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data


def _tie_frac(i):
    x = (np.asarray(i, np.uint64) * np.uint64(0x9E3779B9)) & np.uint64(0xFFFFFFFF)
    x ^= x >> np.uint64(16)
    x = (x * np.uint64(0x7feb352d)) & np.uint64(0xFFFFFFFF)
    x ^= x >> np.uint64(15)
    x = (x * np.uint64(0x846ca68b)) & np.uint64(0xFFFFFFFF)
    x ^= x >> np.uint64(16)
    return (x >> np.uint64(1)).astype(np.float64) * (1.0 / 2147483648.0)


def reference_draws(n):
    """rand() after srand(12345): the C library's own generator (the
    sequence the reference's HMIS weights use, rs_classical.c:542-551)."""
    libc = C.CDLL(None)
    libc.srand(12345)
    return np.array([libc.rand() for _ in range(n)], np.float64)


RAND_MAX = 2147483647.0


def rs_first_pass(n, Sia, Sja, rs_quirk, hmis=False):
    """The device's parallel RS first pass, restated: rounds select undecided
    local maxima of lambda + tie over G = S u S^T; undecided points with a
    strong C become F; each new F adds 1 to its undecided strong dependencies.
    The tie is the reference HMIS's rand()/RAND_MAX for HMIS, a hash of the
    index for RS."""
    rows = np.repeat(np.arange(n), np.diff(Sia))
    lam = np.bincount(Sja, minlength=n).astype(np.int64)
    if rs_quirk:
        lam[0] = 0
    if hmis:
        w = lam.astype(np.float64) + reference_draws(n) / RAND_MAX
    else:
        w = lam.astype(np.float64) + _tie_frac(np.arange(n))
    gi = np.r_[rows, Sja]   # G edges (i, j): S rows and S^T rows
    gj = np.r_[Sja, rows]
    cf = np.zeros(n, np.int32)
    while (cf == 0).any():
        und = cf == 0
        beaten = np.zeros(n, bool)
        e = und[gj] & (w[gj] > w[gi])
        beaten[gi[e]] = True
        newc = und & ~beaten
        if not newc.any():
            cf[und] = 1
            break
        cf[newc] = 1
        hit = np.zeros(n, bool)
        hit[rows[cf[Sja] == 1]] = True
        newf = (cf == 0) & hit
        cf[newf] = -1
        sel = newf[rows] & (cf[Sja] == 0)
        np.add.at(w, Sja[sel], 1.0)
    # second pass (rs_classical.c:357-364): in order, an F point with no
    # strong C becomes C
    for i in range(n):
        if cf[i] == -1 and not (cf[Sja[Sia[i]:Sia[i + 1]]] == 1).any():
            cf[i] = 1
    return cf


def _dcsr(n, ia, ja, val):
    ia, ja, val = (np.ascontiguousarray(ia, np.int32), np.ascontiguousarray(ja, np.int32),
                   np.ascontiguousarray(val, np.float64))
    m = amg.DcsrMat(n, n, int(ia[-1]), ia.ctypes.data_as(C.POINTER(C.c_int)),
                    ja.ctypes.data_as(C.POINTER(C.c_int)),
                    val.ctypes.data_as(C.POINTER(C.c_double)))
    m._keep = (ia, ja, val)
    return m


def _strength(lib, n, A, theta):
    dS = amg.DcsrMat()
    ml = C.c_int()
    lib.rs_strength(C.byref(_dcsr(n, *A)), theta, C.byref(dS), C.byref(ml))
    nnz = dS.nnz
    S = (np.ctypeslib.as_array(dS.ia, shape=(n + 1,)).copy(),
         np.ctypeslib.as_array(dS.ja, shape=(nnz,)).copy(),
         np.ctypeslib.as_array(dS.val, shape=(nnz,)).copy())
    return S, ml.value


def test_restated_first_pass_is_a_split():
    n, ia, ja, val = hub_matrix(side=30, hubs=(200, 400), weak_hubs=(100, 300))
    # strength by hand: -a_ij >= theta * max_k(-a_ik)
    rows = np.repeat(np.arange(n), np.diff(ia))
    off = rows != ja
    neg = np.where(off, -val, 0.0)
    rmax = np.zeros(n)
    np.maximum.at(rmax, rows, neg)
    keep = off & (neg >= 0.25 * rmax[rows]) & (rmax[rows] > 0)
    Sja = ja[keep]
    Sia = np.r_[0, np.cumsum(np.bincount(rows[keep], minlength=n))].astype(np.int32)
    cf = rs_first_pass(n, Sia, Sja, False)
    assert set(np.unique(cf)) <= {1, -1}
    for i in np.nonzero(cf == -1)[0]:
        assert (cf[Sja[Sia[i]:Sia[i + 1]]] == 1).any()


@pytest.mark.gpu
@pytest.mark.parametrize("theta", [0.25, 0.5])
def test_hub_splits(oracle, theta):
    lib = amg.load_library()
    n, ia, ja, val = hub_matrix()
    A = (ia, ja, val)
    S, ml = _strength(lib, n, A, theta)
    lens = np.diff(S[0]) + np.bincount(S[1], minlength=n)
    assert lens.max() > 1000  # the hub path is exercised
    la, ls = np.diff(ia), np.diff(S[0])
    assert ((la > 32) & (ls <= 32)).sum() >= 3  # rows for the warp-per-row interpolation
    # PMIS: bit-exact with the reference's
    cf_ref, nc_ref = oracle.orc_split(n, *S, "pmis")
    cf = np.zeros(n, np.int32)
    nc = C.c_int()
    lib.pmis_coarsening(C.byref(_dcsr(n, *S)), amg._p(cf), C.byref(nc))
    assert nc.value == nc_ref and np.array_equal(cf, cf_ref)
    # interpolation (hub rows of A take the warp-per-row kernel): bit-exact
    P_ref = oracle.orc_interp(n, A, S, cf_ref)
    dP = amg.DcsrMat()
    lib.rs_standard_interpolation(C.byref(_dcsr(n, *A)), C.byref(_dcsr(n, *S)), amg._p(cf),
                                  C.byref(dP))
    P = (np.ctypeslib.as_array(dP.ia, shape=(n + 1,)).copy(),
         np.ctypeslib.as_array(dP.ja, shape=(dP.nnz,)).copy(),
         np.ctypeslib.as_array(dP.val, shape=(dP.nnz,)).copy())
    for a, b in zip(P, P_ref):
        assert a.tobytes() == b.tobytes()
    # HMIS and RS first passes
    for name, quirk in (("hmis", False), ("rs", True)):
        want = rs_first_pass(n, S[0], S[1], quirk, hmis=(name == "hmis"))
        cf = np.zeros(n, np.int32)
        nc = C.c_int()
        if name == "hmis":
            lib.hmis_coarsening(C.byref(_dcsr(n, *S)), amg._p(cf), C.byref(nc))
        else:
            lib.rs_coarsening(C.byref(_dcsr(n, *S)), ml, amg._p(cf), C.byref(nc))
        assert np.array_equal(cf, want), name
        assert nc.value == int((want == 1).sum())


@pytest.mark.gpu
def test_hmis_leaves_the_callers_rand_state():
    """The reference's HMIS first pass never reseeds the C library's
    generator; the device HMIS draws its weights from a private copy."""
    lib = amg.load_library()
    n, ia, ja, val = hub_matrix(side=30, hubs=(200,), weak_hubs=())
    S, ml = _strength(lib, n, (ia, ja, val), 0.5)
    libc = C.CDLL(None)
    libc.srand(777)
    want = [libc.rand() for _ in range(3)]
    libc.srand(777)
    cf = np.zeros(n, np.int32)
    nc = C.c_int()
    lib.hmis_coarsening(C.byref(_dcsr(n, *S)), amg._p(cf), C.byref(nc))
    assert nc.value > 0
    assert [libc.rand() for _ in range(3)] == want


@pytest.mark.gpu
def test_hub_solver_converges():
    n, ia, ja, val = hub_matrix()
    rng = np.random.default_rng(1)
    b = rng.standard_normal(n)
    for coarsen in (amg.COARSEN_PMIS, amg.COARSEN_HMIS):
        s = amg.AMGSolver(n, ia, ja, val, threshold=0.5, coarsening=coarsen, min_size=100)
        x, it = s.solve(b, tol=1e-8, maxiter=100)
        import scipy.sparse as sp
        A = sp.csr_matrix((val, ja, ia), shape=(n, n))
        assert it > 0 and np.linalg.norm(b - A @ x) <= 1e-7 * np.linalg.norm(b)
        s.close()


def reference_symmetrize(n, ia, ja, val):
    """(A + A^T)/2 in the reference's entry order (amg_wrapper.c:59-76 with
    dcsr_mat_add, agg_lib.h:186-243): each row holds A's entries in A's order,
    then A^T's entries absent from A in A^T's order (increasing row of A)."""
    rows = np.repeat(np.arange(n), np.diff(ia))
    order = np.argsort(ja, kind="stable")
    t_ia = np.r_[0, np.cumsum(np.bincount(ja, minlength=n))]
    t_ja, t_val = rows[order], val[order]
    oia, oja, oval = [0], [], []
    for i in range(n):
        ca, va = ja[ia[i]:ia[i + 1]], val[ia[i]:ia[i + 1]]
        ct, vt = t_ja[t_ia[i]:t_ia[i + 1]], t_val[t_ia[i]:t_ia[i + 1]]
        pos = {c: k for k, c in enumerate(ca)}
        acc = va.copy()
        extra_c, extra_v = [], []
        for c, v in zip(ct, vt):
            if c in pos:
                acc[pos[c]] = acc[pos[c]] + v
            else:
                extra_c.append(c)
                extra_v.append(v * 0.5)
        oja += list(ca) + extra_c
        oval += list(acc * 0.5) + extra_v
        oia.append(len(oja))
    return np.array(oia, np.int32), np.array(oja, np.int32), np.array(oval)


@pytest.mark.gpu
def test_symmetrize_huge_rows():
    """A row of 20,000 entries (and a transpose row adding 9,000 more) goes
    through the block-per-row merge; the result equals the reference's
    order and values bit for bit."""
    rng = np.random.default_rng(7)
    n = 30000
    ia, ja, val = [0], [], []
    for i in range(n):
        if i == 0:
            cols = np.r_[0, rng.permutation(np.arange(1, 20001))]
        elif i > 21000:
            cols = np.r_[i, 0]
        else:
            cols = np.r_[i, rng.choice(n, 2, replace=False)]
            cols = np.unique(cols)
            cols = np.r_[i, cols[cols != i]]
        v = -rng.uniform(0.5, 1.5, cols.shape[0])
        v[0] = 50.0 + 50000.0 * (i == 0)
        ja += list(cols)
        val += list(v)
        ia.append(len(ja))
    ia, ja, val = np.array(ia, np.int32), np.array(ja, np.int32), np.array(val)
    want = reference_symmetrize(n, ia, ja, val)
    assert want[0][1] - want[0][0] > 8192 + 9000
    s = amg.AMGSolver(n, ia, ja, val, threshold=0.25)
    got = s.level(0)["A"]
    for a, b in zip(got, want):
        assert np.asarray(a).tobytes() == np.asarray(b, dtype=np.asarray(a).dtype).tobytes()
    s.close()


@pytest.mark.gpu
def test_symmetrize_symmetric_pattern_with_a_hub_row():
    """A structurally symmetric matrix with unequal a_ij and a_ji keeps its
    pattern and entry order, each value (a_ij + a_ji) * 0.5 (binary search in
    the transpose's row; a block for the 3,000-entry hub row): equal to the
    reference's merge-add bit for bit."""
    rng = np.random.default_rng(11)
    n = 12000
    rows = [dict() for _ in range(n)]
    for i in range(n):
        rows[i][i] = 40.0 + rng.uniform(0.0, 1.0)
    def link(i, j):
        rows[i][j] = -rng.uniform(0.5, 1.5)
        rows[j][i] = -rng.uniform(0.5, 1.5)  # same pattern, another value
    for i in range(n - 1):
        link(i, i + 1)
    for j in rng.choice(np.arange(2, n), 3000, replace=False):
        link(0, int(j))
    rows[0][0] = 4000.0  # diagonally dominant hub row
    ia, ja, val = [0], [], []
    for i in range(n):
        cols = list(rows[i].keys())
        rng.shuffle(cols)  # rows in no particular column order
        ja += cols
        val += [rows[i][c] for c in cols]
        ia.append(len(ja))
    ia, ja, val = np.array(ia, np.int32), np.array(ja, np.int32), np.array(val)
    want = reference_symmetrize(n, ia, ja, val)
    assert np.array_equal(want[1], ja)  # the merge-add appends nothing
    s = amg.AMGSolver(n, ia, ja, val, threshold=0.25)
    got = s.level(0)["A"]
    for a, b in zip(got, want):
        assert np.asarray(a).tobytes() == np.asarray(b, dtype=np.asarray(a).dtype).tobytes()
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("long_len", [1100, 2500])
def test_spmv_dropins_with_a_long_row_among_short_rows(oracle, long_len):
    """The reference's abyvg / abyvam / abyvcs (sparse_ops.c:19-56) with a row
    over 1024 entries among short rows: bit-identical to the oracle's
    sequential row sums (the drop-ins sum every row in storage order, also
    when the row's tile overflows the shared product buffer)."""
    rng = np.random.default_rng(11)
    n = 3000
    rows, cols = [], []
    for i in range(n):
        c = rng.choice(n, long_len if i == 100 else 3, replace=False)
        rows += [i] * len(c)
        cols += list(c)
    import scipy.sparse as sp
    A = sp.csr_matrix((rng.standard_normal(len(rows)), (rows, cols)), shape=(n, n))
    A.sum_duplicates()
    A.sort_indices()
    ia, ja, val = (A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data)
    M = (ia, ja, val)
    lib = amg.load_library()
    x = rng.standard_normal(n)
    y0 = rng.standard_normal(n)
    y = np.zeros(n)
    lib.abyvg(amg._p(ia), amg._p(ja), amg._p(val), amg._p(x), n, amg._p(y))
    assert y.tobytes() == oracle.orc_spmv(n, n, M, x, "y").tobytes()
    r = np.zeros(n)
    lib.abyvam(amg._p(y0), amg._p(ia), amg._p(ja), amg._p(val), amg._p(x), n, amg._p(r))
    assert r.tobytes() == oracle.orc_spmv(n, n, M, x, "res", b=y0).tobytes()
    y2 = y0.copy()
    lib.abyvcs(amg._p(ia), amg._p(ja), amg._p(val), amg._p(x), n, amg._p(y2))
    assert y2.tobytes() == oracle.orc_spmv(n, n, M, x, "add", y0=y0).tobytes()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [amg.PREC_FP64, amg.PREC_MIXED])
def test_solve_with_a_long_row_in_a_short_tile(precision):
    """A ring with one node joined to 1,029 others: its row (1,032 entries)
    shares a 256-row tile of the SpMV with short rows (under the tile's 2,048
    entries), and the long-row kernel owns it."""
    import scipy.sparse as sp
    rng = np.random.default_rng(12)
    n = 20000
    u = np.arange(n)
    v = (u + 1) % n
    hub = 100
    nb = rng.choice(np.setdiff1d(np.arange(n), [hub - 1, hub, hub + 1]), 1029, replace=False)
    uu, vv = np.r_[u, np.full(nb.shape, hub)], np.r_[v, nb]
    w = rng.uniform(0.5, 1.5, uu.shape[0])
    W = sp.coo_matrix((np.r_[w, w], (np.r_[uu, vv], np.r_[vv, uu])), shape=(n, n)).tocsr()
    A = (sp.diags(np.asarray(W.sum(1)).ravel() + 1e-2) - W).tocsr()
    A.sort_indices()
    ia, ja, val = A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data
    assert ia[hub + 1] - ia[hub] == 1032  # diagonal, two ring neighbours, 1,029 others
    t0 = (hub // 256) * 256
    assert ia[min(t0 + 256, n)] - ia[t0] <= 2048
    b = rng.standard_normal(n)
    s = amg.AMGSolver(n, ia, ja, val, precision=precision, stop=amg.STOP_RELRES, min_size=100)
    x, it = s.solve(b, tol=1e-8, maxiter=100)
    assert 0 < it <= 40
    assert np.linalg.norm(b - A @ x) <= 1e-8 * np.linalg.norm(b)
    s.close()
