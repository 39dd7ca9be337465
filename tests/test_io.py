"""File formats: the COO text reader against the reference's own reader
(C_amg1/src/io.c:71-124, compiled from its sources under oracle/_ref) on
random files, right-hand-side files, labelled solutions, and network cases
(.fMx/.pMx/.dia/.BC) formed into the Dirichlet-reduced system."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

from blood_network_b200 import amg, io


def _write_coo(path, m, n, rows, cols, vals, fmt="%.17g"):
    with open(path, "w") as f:
        f.write(f"{m} {n} {len(rows)}\n")
        for r, c, v in zip(rows, cols, vals):
            f.write(f"{r} {c} {fmt % v}\n")


def _random_coo(rng, m, n, nnz, base):
    rows = rng.integers(0, m, nnz) + base
    cols = rng.integers(0, n, nnz) + base
    if base == 1 and nnz:
        rows[rng.integers(nnz)] = 1  # the smallest index is exactly 1
    vals = rng.standard_normal(nnz) * 10.0 ** rng.integers(-5, 6, nnz)
    return rows, cols, vals


def test_coo_known_answer(tmp_path):
    p = str(tmp_path / "a.txt")
    # 1-based; row 2 twice with the same column (kept, not summed); rows out of order
    _write_coo(p, 3, 3, [3, 1, 2, 2, 1], [1, 1, 3, 3, 2], [5.0, 1.0, 2.5, -1.0, 0.25])
    m, n, ia, ja, val = io.read_coo(p)
    assert (m, n) == (3, 3)
    assert ia.tolist() == [0, 2, 4, 5]
    assert ja.tolist() == [0, 1, 2, 2, 0]
    assert val.tolist() == [1.0, 0.25, 2.5, -1.0, 5.0]
    # 0-based file: no shift; a file whose smallest index is 2 is not shifted either
    _write_coo(p, 2, 2, [0, 1], [1, 0], [1.0, 2.0])
    assert io.read_coo(p)[3].tolist() == [1, 0]


@pytest.mark.parametrize("base", [0, 1])
@pytest.mark.parametrize("seed", range(4))
def test_coo_matches_reference_reader(tmp_path, oracle, base, seed):
    if not oracle.have_reference():
        pytest.skip("the reference library was not built here")
    rng = np.random.default_rng(seed)
    m, n = int(rng.integers(1, 300)), int(rng.integers(1, 300))
    rows, cols, vals = _random_coo(rng, m, n, int(rng.integers(1, 2000)), base)
    p = str(tmp_path / f"r{seed}.txt")
    _write_coo(p, m, n, rows, cols, vals, fmt=["%.17g", "%.6e", "%g", "%.3f"][seed])
    got = io.read_coo(p)
    want = oracle.ref_read_coo(p)
    assert got[0] == want[0] and got[1] == want[1]
    for a, b in zip(got[2:], want[2:]):
        assert a.tobytes() == b.tobytes()


def test_coo_errors(tmp_path):
    with pytest.raises(amg.AMGError):
        io.read_coo(str(tmp_path / "missing.txt"))
    p = str(tmp_path / "bad.txt")
    open(p, "w").write("3 3\n")
    with pytest.raises(amg.AMGError):
        io.read_coo(p)
    _write_coo(p, 2, 2, [0, 5], [0, 1], [1.0, 1.0])  # row 5 of 2
    with pytest.raises(amg.AMGError):
        io.read_coo(p)
    open(p, "w").write("2 2 3\n0 0 1.0\n1 1 x\n")
    with pytest.raises(amg.AMGError):
        io.read_coo(p)


def test_rhs_file_and_labeled_solution(tmp_path):
    rng = np.random.default_rng(2)
    b = rng.standard_normal(57)
    p = str(tmp_path / "rhs.txt")
    with open(p, "w") as f:
        f.write("57\n" + "\n".join("%.17g" % v for v in b) + "\n")
    assert io.read_vector(p, 57).tobytes() == b.tobytes()
    with pytest.raises(amg.AMGError):
        io.read_vector(p, 58)
    q = str(tmp_path / "sol.txt")
    nodes = np.array([2, 3, 7], np.int32)
    io.write_labeled_solution(q, nodes, np.array([1.5, -2.0, 1e-300]))
    assert open(q).read() == ("2 1.5000000000000000e+00\n3 -2.0000000000000000e+00\n"
                              "7 1.0000000000000000e-300\n")


def _cartesian_case(prefix, nx, ny, nz, hx=2.0, hy=3.0, hz=5.0):
    """A Cartesian lattice case: faces along +x, +y, +z, two Dirichlet nodes."""
    idx = np.arange(nx * ny * nz).reshape(nz, ny, nx)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    coords = np.stack([i.ravel() * hx, j.ravel() * hy, k.ravel() * hz], 1)
    faces = []
    for a, b in ((idx[:, :, :-1], idx[:, :, 1:]), (idx[:, :-1, :], idx[:, 1:, :]),
                 (idx[:-1, :, :], idx[1:, :, :])):
        faces.append(np.stack([a.ravel(), b.ravel()], 1))
    faces = np.concatenate(faces)
    nf = faces.shape[0]
    np.savetxt(prefix + ".fMx", np.column_stack([np.arange(1, nf + 1), faces + 1]), fmt="%d")
    np.savetxt(prefix + ".pMx", coords, fmt="%.6f")
    np.savetxt(prefix + ".dia", np.full(nf, 1e-3), fmt="%.6e")
    npt = nx * ny * nz
    np.savetxt(prefix + ".BC", np.array([[1, 1, 13300.0], [npt, 1, 2000.0]]), fmt="%.6f")
    return coords, faces, (hx, hy, hz)


def _expected_system(npt, faces, g, bnodes, pb):
    nf = faces.shape[0]
    C1 = sp.csr_matrix((np.r_[np.ones(nf), -np.ones(nf)],
                        (np.r_[np.arange(nf), np.arange(nf)], np.r_[faces[:, 0], faces[:, 1]])),
                       shape=(nf, npt))
    interior = np.setdiff1d(np.arange(npt), bnodes)
    W = sp.diags(g)
    CI, CB = C1[:, interior], C1[:, bnodes]
    return (CI.T @ W @ CI).tocsr(), -(CI.T @ W @ CB @ pb)


def test_case_reader_and_system(tmp_path):
    prefix = str(tmp_path / "nwk_Cartesian_4x3x2")
    coords, faces, (hx, hy, hz) = _cartesian_case(prefix, 4, 3, 2)
    c = io.read_case(prefix)
    assert (c.np_, c.nf) == (24, faces.shape[0]) and c.nt == c.np_ + c.nf
    g = io.diffusive_conductance(c.faces, c.coords)
    nx_f = 3 * 3 * 2
    ny_f = 4 * 2 * 2
    assert np.allclose(g[:nx_f], hy * hz / hx) and np.allclose(g[nx_f:nx_f + ny_f], hx * hz / hy)
    assert np.allclose(g[nx_f + ny_f:], hx * hy / hz)
    net = io.case_network(prefix)
    L, rhs = _expected_system(24, faces, g, np.array([0, 23]), np.array([13300.0, 2000.0]))
    A = sp.csr_matrix((net.data, net.indices, net.indptr), shape=(net.n, net.n))
    assert net.n == 22 and abs(A - L).max() <= 1e-12 * abs(L).max()
    assert np.allclose(net.rhs, rhs, rtol=1e-14, atol=0)
    # a face pointing the other way gets NaN (no positive component)
    f2 = c.faces.copy()
    f2[0, 1], f2[0, 2] = f2[0, 2], f2[0, 1]
    assert np.isnan(io.diffusive_conductance(f2, c.coords)[0])


@pytest.mark.gpu
def test_case_solved_and_written(tmp_path):
    prefix = str(tmp_path / "nwk_Cartesian_30x20x10")
    _cartesian_case(prefix, 30, 20, 10)
    net = io.case_network(prefix)
    S = amg.AMGSolver(net.n, net.indptr, net.indices, net.data)
    x, it = S.solve(net.rhs, tol=1e-10, maxiter=100)
    A = sp.csr_matrix((net.data, net.indices, net.indptr), shape=(net.n, net.n))
    assert it > 0 and np.linalg.norm(net.rhs - A @ x) <= 1e-8 * np.linalg.norm(net.rhs)
    interior = np.nonzero(net.interior_of >= 0)[0] + 1
    out = str(tmp_path / "p_interior_30x20x10_labeled.txt")
    io.write_labeled_solution(out, interior, x)
    back = np.loadtxt(out)
    assert np.array_equal(back[:, 0], interior) and np.allclose(back[:, 1], x, rtol=1e-15)


def test_large_coo_parsed_in_parallel_matches_reference(tmp_path, oracle):
    """Files over 1 MB are parsed by several threads (pieces cut at
    whitespace, tokens placed by their global position): same CSR as the
    reference's reader, with entries split across lines in odd places."""
    if not oracle.have_reference():
        pytest.skip("the reference library was not built here")
    rng = np.random.default_rng(7)
    m = n = 5000
    rows, cols, vals = _random_coo(rng, m, n, 120_000, 1)
    p = str(tmp_path / "big.txt")
    with open(p, "w") as f:
        f.write(f"{m} {n} {len(rows)}\n")
        for k, (r, c, v) in enumerate(zip(rows, cols, vals)):
            sep = "\n" if k % 7 == 0 else " "  # some entries span two lines
            f.write(f"{r}{sep}{c} {v:.17g}\n")
        f.write("1 2 3 trailing tokens past nnz are ignored\n")
    assert os.path.getsize(p) > 1 << 20
    got = io.read_coo(p)
    want = oracle.ref_read_coo(p)
    assert got[0] == want[0] and got[1] == want[1]
    for a, b in zip(got[2:], want[2:]):
        assert a.tobytes() == b.tobytes()
    # a malformed entry deep in the file is reported by its index
    bad = str(tmp_path / "bad_big.txt")
    with open(bad, "w") as f:
        f.write(f"{m} {n} 100000\n")
        for k in range(100_000):
            f.write(f"{rows[k]} {cols[k]} {'oops' if k == 87_654 else format(vals[k], '.17g')}\n")
    with pytest.raises(amg.AMGError, match="entry 87654"):
        io.read_coo(bad)
