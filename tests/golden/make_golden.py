"""Generates the golden fixtures in this directory from the REFERENCE solver.

Run from the repository root after `make -C oracle` has compiled the
reference C sources into oracle/_ref/ (needs the reference tree, so it runs
where that tree is mounted; the fixtures it writes are committed):

    python tests/golden/make_golden.py

Fixtures:
  small_pmis.npz   -- a 1.5k-node vascular network: every level's A, S, C/F
                      and P, the fine IC(0) factor, one preconditioner
                      application and the PCG solution (tol 1e-8), PMIS.
  edge_cases.npz   -- unsymmetric-pattern / unsorted-column inputs and the
                      reference's symmetrised matrix, strength and C/F.
  digests.json     -- SHA-256 digests of every level of the 20k-node network
                      (PMIS/HMIS/RS) and of the 2M-node network (PMIS), plus
                      iteration counts and solution digests, for bit-exact
                      checks without storing the arrays.
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import ref as R  # noqa: E402
from blood_network_b200.network import vascular_network, make_config  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def small_network():
    return vascular_network(depth=7, n_nodes=1500, seed=3)


def edge_matrices():
    """Inputs the reference's symmetrisation handles specially: an unsymmetric
    pattern with unsorted columns, and a matrix with a missing diagonal entry
    in the pattern of A^T only."""
    rng = np.random.default_rng(7)
    n = 40
    rows, cols, vals = [], [], []
    for i in range(n):
        rows.append(i); cols.append(i); vals.append(4.0 + rng.random())
        nb = rng.choice(n, size=3, replace=False)
        for j in nb:
            if j != i:
                rows.append(i); cols.append(int(j)); vals.append(-rng.random())
    ia = np.zeros(n + 1, np.int64)
    order = np.argsort(np.array(rows), kind="stable")
    rows = np.array(rows)[order]; cols = np.array(cols)[order]; vals = np.array(vals)[order]
    for r in rows:
        ia[r + 1] += 1
    ia = np.cumsum(ia)
    # shuffle columns inside each row (unsorted input)
    for i in range(n):
        s, e = ia[i], ia[i + 1]
        p = rng.permutation(e - s)
        cols[s:e] = cols[s:e][p]; vals[s:e] = vals[s:e][p]
    return n, ia.astype(np.int32), cols.astype(np.int32), vals


def main():
    # ---- small network, full arrays
    net = small_network()
    r = R.RefSolver(net.n, net.indptr, net.indices, net.data, 0.25, 50, 20, 1, 1)
    d = {"n": net.n, "indptr": net.indptr, "indices": net.indices, "data": net.data,
         "rhs": net.rhs, "levels": r.num_levels}
    for k in range(r.num_levels):
        L = r.level(k)
        for nm in ("A", "S", "P"):
            if L[nm] is not None:
                for j, part in enumerate(("ia", "ja", "val")):
                    d[f"L{k}_{nm}_{part}"] = L[nm][j]
        if L["cf"] is not None:
            d[f"L{k}_cf"] = L["cf"]
    lia, lja, lval = r.ichol()
    d["ichol_ia"], d["ichol_ja"], d["ichol_val"] = lia, lja, lval
    g = np.cos(0.37 * np.arange(net.n))
    d["precond_g"] = g
    d["precond_z"] = r.precond(g)
    x, it = r.solve(net.rhs, tol=1e-8)
    d["solve_x"], d["solve_iters"] = x, it
    np.savez_compressed(os.path.join(OUT, "small_pmis.npz"), **d)

    # ---- edge cases: symmetrisation of unsorted unsymmetric input, strength, C/F
    n, ia, ja, va = edge_matrices()
    r2 = R.RefSolver(n, ia, ja, va, 0.25, 10, 20, 1, 1)
    L0 = r2.level(0)
    e = {"n": n, "indptr": ia, "indices": ja, "data": va, "A_ia": L0["A"][0],
         "A_ja": L0["A"][1], "A_val": L0["A"][2]}
    if L0["S"] is not None:
        e.update(S_ia=L0["S"][0], S_ja=L0["S"][1], S_val=L0["S"][2], cf=L0["cf"])
    np.savez_compressed(os.path.join(OUT, "edge_cases.npz"), **e)

    # ---- 20k network digests, three coarsenings
    big = make_config("vascular_20k")
    dig = {"n": big.n, "nnz": big.nnz, "input": digest(big.indptr, big.indices, big.data),
           "rhs": digest(big.rhs)}
    for name, coarsen, theta in (("pmis", 1, 0.25), ("hmis", 2, 0.5), ("rs", 0, 0.25)):
        rr = R.RefSolver(big.n, big.indptr, big.indices, big.data, theta, 500, 20, 1, coarsen)
        levels = []
        for k in range(rr.num_levels):
            L = rr.level(k)
            ent = {"n": L["n"], "A": digest(*L["A"])}
            if L["S"] is not None:
                ent.update(S=digest(*L["S"]), P=digest(*L["P"]), cf=digest(L["cf"]),
                           n_coarse=L["n_coarse"])
            levels.append(ent)
        x, it = rr.solve(big.rhs, tol=1e-8)
        dig[name] = {"theta": theta, "levels": levels, "ichol": digest(*rr.ichol()),
                     "iterations": it, "x": digest(x)}
    # 2M-node network (full size of the 2M configuration), PMIS
    big2 = make_config("vascular_2m")
    rr = R.RefSolver(big2.n, big2.indptr, big2.indices, big2.data, 0.25, 500, 20, 1, 1)
    levels = []
    for k in range(rr.num_levels):
        L = rr.level(k)
        ent = {"n": L["n"], "A": digest(*L["A"])}
        if L["S"] is not None:
            ent.update(S=digest(*L["S"]), P=digest(*L["P"]), cf=digest(L["cf"]),
                       n_coarse=L["n_coarse"])
        levels.append(ent)
    x, it = rr.solve(big2.rhs, tol=1e-8)
    dig["pmis_2m"] = {"theta": 0.25, "n": big2.n, "nnz": big2.nnz,
                      "input": digest(big2.indptr, big2.indices, big2.data), "levels": levels,
                      "ichol": digest(*rr.ichol()), "iterations": it, "x": digest(x)}
    with open(os.path.join(OUT, "digests.json"), "w") as f:
        json.dump(dig, f, indent=1)
    print("fixtures written to", OUT)


if __name__ == "__main__":
    main()
