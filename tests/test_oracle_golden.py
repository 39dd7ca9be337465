"""The CPU restatement (oracle/amg_oracle.c) against fixtures generated from
the reference solver itself (tests/golden/make_golden.py)."""
import numpy as np
import pytest

from helpers import bits_equal, digest, level_from_golden


def test_small_network_every_level_bit_exact(oracle, golden_small):
    g = golden_small
    o = oracle.OracleSolver(int(g["n"]), g["indptr"], g["indices"], g["data"], 0.25, 50, 20, 1, 1)
    assert o.num_levels == int(g["levels"])
    for k in range(o.num_levels):
        got, want = o.level(k), level_from_golden(g, k)
        for nm in ("A", "S", "P"):
            if want[nm] is None:
                continue
            for j in range(3):
                assert bits_equal(got[nm][j], want[nm][j]), (k, nm, j)
        if want["cf"] is not None:
            assert np.array_equal(got["cf"], want["cf"]), k
    ia, ja, val = o.ichol()
    assert bits_equal(ia, g["ichol_ia"]) and bits_equal(ja, g["ichol_ja"])
    assert bits_equal(val, g["ichol_val"])
    assert bits_equal(o.precond(g["precond_g"]), g["precond_z"])
    x, it = o.solve(g["rhs"], tol=1e-8)
    assert it == int(g["solve_iters"])
    assert bits_equal(x, g["solve_x"])


def test_edge_case_symmetrisation_strength_split(oracle, golden_edge):
    e = golden_edge
    o = oracle.OracleSolver(int(e["n"]), e["indptr"], e["indices"], e["data"], 0.25, 10, 20, 1, 1)
    L0 = o.level(0)
    assert bits_equal(L0["A"][0], e["A_ia"]) and bits_equal(L0["A"][1], e["A_ja"])
    assert bits_equal(L0["A"][2], e["A_val"])
    if "S_ia" in e:
        assert bits_equal(L0["S"][1], e["S_ja"]) and bits_equal(L0["S"][2], e["S_val"])
        assert np.array_equal(L0["cf"], e["cf"])


@pytest.mark.parametrize("name,coarsen", [("pmis", 1), ("hmis", 2), ("rs", 0)])
def test_20k_network_digests(oracle, golden_digests, name, coarsen):
    from blood_network_b200.network import make_config
    net = make_config("vascular_20k")
    assert digest(net.indptr, net.indices, net.data) == golden_digests["input"]
    ref = golden_digests[name]
    o = oracle.OracleSolver(net.n, net.indptr, net.indices, net.data, ref["theta"], 500, 20, 1,
                            coarsen)
    assert o.num_levels == len(ref["levels"])
    for k, want in enumerate(ref["levels"]):
        L = o.level(k)
        assert digest(*L["A"]) == want["A"], (name, k)
        if "S" in want:
            assert digest(*L["S"]) == want["S"], (name, k)
            assert digest(*L["P"]) == want["P"], (name, k)
            assert digest(L["cf"]) == want["cf"], (name, k)
    assert digest(*o.ichol()) == ref["ichol"]
    x, it = o.solve(net.rhs, tol=1e-8)
    assert it == ref["iterations"]
    assert digest(x) == ref["x"]


def test_oracle_matches_live_reference(oracle):
    """When the compiled reference is present, compare it live on a fresh seed."""
    if not oracle.have_reference():
        pytest.skip("compiled reference not built here")
    from blood_network_b200.network import vascular_network
    net = vascular_network(depth=8, n_nodes=4000, seed=11, diffusive_fraction=0.3)
    for coarsen, theta in ((1, 0.25), (2, 0.5)):
        r = oracle.RefSolver(net.n, net.indptr, net.indices, net.data, theta, 100, 20, 1, coarsen)
        o = oracle.OracleSolver(net.n, net.indptr, net.indices, net.data, theta, 100, 20, 1,
                                coarsen)
        assert r.num_levels == o.num_levels
        for k in range(r.num_levels):
            a, b = r.level(k), o.level(k)
            for j in range(3):
                assert bits_equal(a["A"][j], b["A"][j])
        xr, itr = r.solve(net.rhs)
        xo, ito = o.solve(net.rhs)
        assert itr == ito and bits_equal(xr, xo)
