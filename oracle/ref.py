"""Test infrastructure: ctypes access to the CPU oracles in this directory.

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
        lib.refdrv_update.argtypes = [vp, i, i, vp, vp, vp]
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

    def update(self, indptr, indices, data):
        """amg_solver_update: new values on the same pattern."""
        a = (np.ascontiguousarray(indptr, np.int32), np.ascontiguousarray(indices, np.int32),
             np.ascontiguousarray(data, np.float64))
        self.lib.refdrv_update(self.h, self.n, int(a[0][-1]), _P(a[0]), _P(a[1]), _P(a[2]))

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


# ------------------------------------------------------------------ restatement
_orc = None


def have_oracle() -> bool:
    return os.path.exists(ORACLE)


def orc_lib():
    global _orc
    if _orc is None:
        lib = C.CDLL(ORACLE)
        vp, i, d = C.c_void_p, C.c_int, C.c_double
        lib.orc_create.restype = vp
        lib.orc_create.argtypes = [i, i, vp, vp, vp, d, i, i, i, i, i, d]
        lib.orc_solve.argtypes = [vp, vp, vp, d, i]
        lib.orc_precond.argtypes = [vp, vp, vp]
        lib.orc_num_levels.argtypes = [vp]
        lib.orc_level_sizes.argtypes = [vp, i, vp]
        lib.orc_level_copy.argtypes = [vp, i] + [vp] * 10
        lib.orc_ichol_nnz.argtypes = [vp]
        lib.orc_ichol_copy.argtypes = [vp, vp, vp, vp]
        lib.orc_free.argtypes = [vp]
        P_ = C.POINTER
        lib.orc_csr_free.argtypes = [vp]
        for nm in ("orc_strength",):
            getattr(lib, nm).argtypes = [vp, d, vp, vp]
        for nm in ("orc_pmis", "orc_hmis"):
            getattr(lib, nm).argtypes = [vp, vp, vp]
        lib.orc_rs.argtypes = [vp, i, vp, vp]
        lib.orc_interp.argtypes = [vp, vp, vp, vp]
        lib.orc_transpose.argtypes = [vp, vp]
        lib.orc_rap.argtypes = [vp, vp, vp, vp]
        lib.orc_ichol.argtypes = [vp, vp]
        lib.orc_ichol_solve.argtypes = [vp, vp, vp]
        lib.orc_spmv.argtypes = [vp, vp, vp]
        lib.orc_residual.argtypes = [vp, vp, vp, vp]
        lib.orc_spmv_add.argtypes = [vp, vp, vp]
        lib.orc_spmv_t.argtypes = [vp, vp, i, vp]
        del P_
        _orc = lib
    return _orc


class OracleSolver(RefSolver):
    """The CPU restatement (amg_oracle.c), same interface as RefSolver."""

    def __init__(self, n, indptr, indices, data, theta=0.25, min_size=500, max_levels=20, nu=1,
                 coarsening=1, smoother=2, omega=0.5):
        self.lib = orc_lib()
        self._a = (np.ascontiguousarray(indptr, np.int32), np.ascontiguousarray(indices, np.int32),
                   np.ascontiguousarray(data, np.float64))
        self.n = n
        self.h = self.lib.orc_create(n, int(self._a[0][-1]), _P(self._a[0]), _P(self._a[1]),
                                     _P(self._a[2]), theta, min_size, max_levels, nu, coarsening,
                                     smoother, omega)

    @property
    def num_levels(self):
        return self.lib.orc_num_levels(self.h)

    def solve(self, b, x0=None, tol=1e-8, maxiter=200):
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(self.n) if x0 is None else np.array(x0, np.float64)
        it = self.lib.orc_solve(self.h, _P(b), _P(x), tol, maxiter)
        return x, it

    def precond(self, g):
        g = np.ascontiguousarray(g, np.float64)
        x = np.zeros(self.n)
        self.lib.orc_precond(self.h, _P(g), _P(x))
        return x

    def level(self, k):
        sz = np.zeros(5, np.int32)
        self.lib.orc_level_sizes(self.h, k, _P(sz))
        n, annz, snnz, pnnz, nc = [int(v) for v in sz]
        A = (np.zeros(n + 1, np.int32), np.zeros(annz, np.int32), np.zeros(annz))
        S = (np.zeros(n + 1, np.int32), np.zeros(max(snnz, 1), np.int32), np.zeros(max(snnz, 1)))
        P = (np.zeros(n + 1, np.int32), np.zeros(max(pnnz, 1), np.int32), np.zeros(max(pnnz, 1)))
        cf = np.zeros(max(n, 1), np.int32)
        self.lib.orc_level_copy(self.h, k, _P(A[0]), _P(A[1]), _P(A[2]), _P(S[0]), _P(S[1]),
                                _P(S[2]), _P(P[0]), _P(P[1]), _P(P[2]), _P(cf))
        if k == self.num_levels - 1:
            return dict(n=n, n_coarse=0, A=A, S=None, P=None, cf=None)
        return dict(n=n, n_coarse=nc, A=A, S=(S[0], S[1][:snnz], S[2][:snnz]),
                    P=(P[0], P[1][:pnnz], P[2][:pnnz]), cf=cf[:n])

    def ichol(self):
        nnz = self.lib.orc_ichol_nnz(self.h)
        ia, ja, val = np.zeros(self.n + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz)
        self.lib.orc_ichol_copy(self.h, _P(ia), _P(ja), _P(val))
        return ia, ja, val

    def close(self):
        if self.h:
            self.lib.orc_free(self.h)
            self.h = None


# ------------------------------------------------------------------ kernel-level oracle
class OrcCsr(C.Structure):
    _fields_ = [("n", C.c_int), ("m", C.c_int), ("nnz", C.c_int), ("ia", C.POINTER(C.c_int)),
                ("ja", C.POINTER(C.c_int)), ("val", C.POINTER(C.c_double))]


def _orc_in(n, m, ia, ja, val):
    ia = np.ascontiguousarray(ia, np.int32)
    ja = np.ascontiguousarray(ja, np.int32)
    val = np.ascontiguousarray(val, np.float64)
    s = OrcCsr(n, m, int(ia[-1]), ia.ctypes.data_as(C.POINTER(C.c_int)),
               ja.ctypes.data_as(C.POINTER(C.c_int)), val.ctypes.data_as(C.POINTER(C.c_double)))
    s._keep = (ia, ja, val)
    return s


def _orc_out(s):
    n, nnz = s.n, s.nnz
    ia = np.ctypeslib.as_array(s.ia, shape=(n + 1,)).copy()
    ja = np.ctypeslib.as_array(s.ja, shape=(max(nnz, 1),))[:nnz].copy()
    val = np.ctypeslib.as_array(s.val, shape=(max(nnz, 1),))[:nnz].copy()
    orc_lib().orc_csr_free(C.byref(s))
    return ia, ja, val


def orc_strength(n, ia, ja, val, theta):
    lib = orc_lib()
    a = _orc_in(n, n, ia, ja, val)
    s = OrcCsr()
    ml = C.c_int()
    lib.orc_strength(C.byref(a), C.c_double(theta), C.byref(s), C.byref(ml))
    return _orc_out(s), ml.value


def orc_split(n, sia, sja, sval, method, max_lam=1):
    lib = orc_lib()
    s = _orc_in(n, n, sia, sja, sval)
    cf = np.zeros(n, np.int32)
    nc = C.c_int()
    if method == "pmis":
        lib.orc_pmis(C.byref(s), _P(cf), C.byref(nc))
    elif method == "hmis":
        lib.orc_hmis(C.byref(s), _P(cf), C.byref(nc))
    else:
        lib.orc_rs(C.byref(s), max_lam, _P(cf), C.byref(nc))
    return cf, nc.value


def orc_interp(n, A, S, cf):
    lib = orc_lib()
    a = _orc_in(n, n, *A)
    s = _orc_in(n, n, *S)
    p = OrcCsr()
    cf = np.ascontiguousarray(cf, np.int32)
    lib.orc_interp(C.byref(a), C.byref(s), _P(cf), C.byref(p))
    return _orc_out(p)


def orc_transpose(n, m, ia, ja, val):
    lib = orc_lib()
    a = _orc_in(n, m, ia, ja, val)
    t = OrcCsr()
    lib.orc_transpose(C.byref(a), C.byref(t))
    return _orc_out(t)


def orc_rap(nc, nf, R, A, P):
    lib = orc_lib()
    r = _orc_in(nc, nf, *R)
    a = _orc_in(nf, nf, *A)
    p = _orc_in(nf, nc, *P)
    out = OrcCsr()
    lib.orc_rap(C.byref(r), C.byref(a), C.byref(p), C.byref(out))
    return _orc_out(out)


def orc_ichol(n, ia, ja, val):
    lib = orc_lib()
    a = _orc_in(n, n, ia, ja, val)
    L = OrcCsr()
    lib.orc_ichol(C.byref(a), C.byref(L))
    return _orc_out(L)


def orc_ichol_solve(n, L, b):
    lib = orc_lib()
    l = _orc_in(n, n, *L)
    x = np.zeros(n)
    b = np.ascontiguousarray(b, np.float64)
    lib.orc_ichol_solve(C.byref(l), _P(b), _P(x))
    return x


def orc_spmv(n, m, A, x, mode="y", b=None, y0=None):
    lib = orc_lib()
    a = _orc_in(n, m, *A)
    x = np.ascontiguousarray(x, np.float64)
    if mode == "y":
        y = np.zeros(n)
        lib.orc_spmv(C.byref(a), _P(x), _P(y))
    elif mode == "res":
        y = np.zeros(n)
        b = np.ascontiguousarray(b, np.float64)
        lib.orc_residual(C.byref(a), _P(b), _P(x), _P(y))
    elif mode == "add":
        y = np.array(y0, np.float64)
        lib.orc_spmv_add(C.byref(a), _P(x), _P(y))
    else:  # transpose
        y = np.zeros(m)
        lib.orc_spmv_t(C.byref(a), _P(x), m, _P(y))
    return y


def ref_read_coo(path):
    """The reference's COO text reader (C_amg1/src/io.c:71-124, compiled from
    its sources): returns (nrow, ncol, indptr, indices, data) or None when it
    reports an error."""
    from blood_network_b200.amg import DcsrMat
    lib = ref_lib()
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    libc.free.argtypes = [C.c_void_p]
    lib.dcsr_mat_dcoo.argtypes = [C.c_void_p, C.POINTER(DcsrMat)]
    lib.dcsr_mat_dcoo.restype = C.c_int
    fp = libc.fopen(path.encode(), b"r")
    out = DcsrMat()
    rc = lib.dcsr_mat_dcoo(fp, C.byref(out))
    libc.fclose(fp)
    if rc != 0:
        return None
    m, nnz = out.row, out.nnz
    ia = np.ctypeslib.as_array(out.ia, shape=(m + 1,)).copy()
    ja = np.ctypeslib.as_array(out.ja, shape=(nnz,)).copy() if nnz else np.zeros(0, np.int32)
    val = np.ctypeslib.as_array(out.val, shape=(nnz,)).copy() if nnz else np.zeros(0)
    for p in (out.ia, out.ja, out.val):
        libc.free(C.cast(p, C.c_void_p))
    return m, out.col, ia, ja, val
