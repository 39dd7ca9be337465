import hashlib

import numpy as np


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def bits_equal(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.shape == b.shape and a.dtype == b.dtype and a.tobytes() == b.tobytes()


def level_from_golden(g, k):
    out = {}
    for nm in ("A", "S", "P"):
        key = f"L{k}_{nm}_ia"
        out[nm] = (g[key], g[f"L{k}_{nm}_ja"], g[f"L{k}_{nm}_val"]) if key in g else None
    out["cf"] = g.get(f"L{k}_cf")
    return out


def relres(indptr, indices, data, x, b):
    import scipy.sparse as sp
    n = len(indptr) - 1
    A = sp.csr_matrix((data, indices, indptr), shape=(n, n))
    return float(np.linalg.norm(b - A @ x) / np.linalg.norm(b))
