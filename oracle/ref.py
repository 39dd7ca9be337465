"""Test infrastructure: ctypes access to the CPU checkers in this directory.

* ``_ref/libamg_refdrv.so`` -- the reference C_amg1 solver compiled from its
  own sources (see Makefile) plus ref_driver.c, which drives it like
  amg_solver_create/solve with a selectable coarsening.
* ``liboracle_amg.so`` -- the CPU restatement in amg_oracle.c.

Only tests/, the smoke check and bench.py's CPU-baseline leg use this module.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DRV = os.path.join(HERE, "_ref", "libamg_refdrv.so")
ORACLE = os.path.join(HERE, "liboracle_amg.so")

_P = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731


def have_reference() -> bool:
    return os.path.exists(REF_DRV)


_ref = None


def ref_lib():
    global _ref
    if _ref is None:
        lib = C.CDLL(REF_DRV)
        vp, i, d = C.c_void_p, C.c_int, C.c_double
        lib.refdrv_create.restype = vp
        lib.refdrv_create.argtypes = [i, i, vp, vp, vp, d, i, i, i, i]
        lib.refdrv_solve.argtypes = [vp, vp, vp, d, i]
        lib.refdrv_num_levels.argtypes = [vp]
        lib.refdrv_level_sizes.argtypes = [vp, i, vp]
        lib.refdrv_level_copy.argtypes = [vp, i] + [vp] * 10
        lib.refdrv_ichol_nnz.argtypes = [vp]
        lib.refdrv_ichol_copy.argtypes = [vp, vp, vp, vp]
        lib.refdrv_precond_apply.argtypes = [vp, vp, vp]
        lib.refdrv_timed.argtypes = [i, i] + [vp] * 5 + [d, i, i, i, d, i, vp, vp]
        lib.refdrv_free.argtypes = [vp]
        _ref = lib
    return _ref


class RefSolver:
    """The reference C solver (CPU), built with the given coarsening."""

    def __init__(self, n, indptr, indices, data, theta=0.25, min_size=500, max_levels=20, nu=1,
                 coarsening=1):
        self.lib = ref_lib()
        self._a = (np.ascontiguousarray(indptr, np.int32), np.ascontiguousarray(indices, np.int32),
                   np.ascontiguousarray(data, np.float64))
        self.n = n
        self.h = self.lib.refdrv_create(n, int(self._a[0][-1]), _P(self._a[0]), _P(self._a[1]),
                                        _P(self._a[2]), theta, min_size, max_levels, nu,
                                        coarsening)

    @property
    def num_levels(self):
        return self.lib.refdrv_num_levels(self.h)

    def solve(self, b, x0=None, tol=1e-8, maxiter=200):
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(self.n) if x0 is None else np.array(x0, np.float64)
        it = self.lib.refdrv_solve(self.h, _P(b), _P(x), tol, maxiter)
        return x, it

    def precond(self, g):
        g = np.ascontiguousarray(g, np.float64)
        x = np.zeros(self.n)
        self.lib.refdrv_precond_apply(self.h, _P(g), _P(x))
        return x

    def level(self, k):
        sz = np.zeros(5, np.int32)
        self.lib.refdrv_level_sizes(self.h, k, _P(sz))
        n, annz, snnz, pnnz, nc = [int(v) for v in sz]
        A = (np.zeros(n + 1, np.int32), np.zeros(annz, np.int32), np.zeros(annz))
        S = (np.zeros(n + 1, np.int32), np.zeros(max(snnz, 1), np.int32), np.zeros(max(snnz, 1)))
        P = (np.zeros(n + 1, np.int32), np.zeros(max(pnnz, 1), np.int32), np.zeros(max(pnnz, 1)))
        mis = np.zeros(n, np.int32)
        self.lib.refdrv_level_copy(self.h, k, _P(A[0]), _P(A[1]), _P(A[2]), _P(S[0]), _P(S[1]),
                                   _P(S[2]), _P(P[0]), _P(P[1]), _P(P[2]), _P(mis))
        last = k == self.num_levels - 1
        if last:
            return dict(n=n, n_coarse=0, A=A, S=None, P=None, cf=None)
        S = (S[0], S[1][:snnz], S[2][:snnz])
        P = (P[0], P[1][:pnnz], P[2][:pnnz])
        cf = np.where(mis == 1, 1, -1).astype(np.int32)
        return dict(n=n, n_coarse=nc, A=A, S=S, P=P, cf=cf)

    def ichol(self):
        nnz = self.lib.refdrv_ichol_nnz(self.h)
        ia, ja, val = np.zeros(self.n + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz)
        self.lib.refdrv_ichol_copy(self.h, _P(ia), _P(ja), _P(val))
        return ia, ja, val

    def close(self):
        if self.h:
            self.lib.refdrv_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ref_timed(n, indptr, indices, data, b, theta, min_size, nu, coarsening, tol, maxiter):
    """Timed create+solve of the reference (CLOCK_MONOTONIC).  Returns
    (iterations, setup_s, solve_s, x)."""
    lib = ref_lib()
    a0, a1, a2 = (np.ascontiguousarray(indptr, np.int32), np.ascontiguousarray(indices, np.int32),
                  np.ascontiguousarray(data, np.float64))
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros(n)
    ts, tv = C.c_double(), C.c_double()
    it = lib.refdrv_timed(n, int(a0[-1]), _P(a0), _P(a1), _P(a2), _P(b), _P(x), theta, min_size,
                          nu, coarsening, tol, maxiter, C.byref(ts), C.byref(tv))
    return it, ts.value, tv.value, x
