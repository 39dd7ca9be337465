"""Python binding of the B200 AMG-PCG C ABI (``include/amg_b200.h``).

This mirrors how the reference's library is driven from Python ctypes (the
reference documents Julia ``ccall`` and ctypes use of ``amg_solver_*``,
``C_amg1/README.md:17,79-160``): an opaque handle from ``amg_solver_create``,
``amg_solver_solve`` with host arrays, ``amg_solver_free``.  Every call goes
through ``lib/libamg_b200.so``; there is no CPU fallback -- if the library or
a CUDA device is missing the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libamg_b200.so")

SMOOTHER_L1, SMOOTHER_GS, SMOOTHER_CF_GS, SMOOTHER_JACOBI = 0, 1, 2, 3
COARSEN_RS, COARSEN_PMIS, COARSEN_HMIS = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1
STOP_BNORM, STOP_RELRES = 0, 1

STATUS = {0: "OK", -1: "ERR_ARG", -2: "ERR_CUDA", -3: "ERR_OOM", -4: "ERR_NOT_CONVERGED",
          -5: "ERR_NAN", -6: "ERR_SPIN", -7: "ERR_COARSE", -8: "ERR_NO_DEVICE", -9: "ERR_DUP"}
ERR_ARG, ERR_CUDA, ERR_OOM, ERR_NOT_CONVERGED, ERR_NAN, ERR_SPIN, ERR_COARSE = -1, -2, -3, -4, -5, -6, -7


class AMGError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class Options(C.Structure):
    _fields_ = [("threshold", C.c_double), ("min_size", C.c_int), ("max_levels", C.c_int),
                ("nu", C.c_int), ("coarsening", C.c_int), ("smoother", C.c_int),
                ("omega", C.c_double), ("precision", C.c_int), ("stop", C.c_int),
                ("device", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("relres", C.c_double),
                ("bnorm_rel", C.c_double), ("setup_seconds", C.c_double),
                ("solve_seconds", C.c_double), ("num_levels", C.c_int),
                ("nnz_total", C.c_longlong), ("ichol_levels", C.c_int),
                ("device_loop", C.c_int), ("ichol_form", C.c_int)]


class DcsrMat(C.Structure):
    """The reference's dcsr_mat (C_amg1/include/agg_lib.h:37-44)."""
    _fields_ = [("row", C.c_int), ("col", C.c_int), ("nnz", C.c_int),
                ("ia", C.POINTER(C.c_int)), ("ja", C.POINTER(C.c_int)),
                ("val", C.POINTER(C.c_double))]


class IcholFactor(C.Structure):
    """The reference's ichol_factor (C_amg1/include/amg.h:344-351)."""
    _fields_ = [("n", C.c_int), ("ia", C.POINTER(C.c_int)), ("ja", C.POINTER(C.c_int)),
                ("val", C.POINTER(C.c_double)), ("nnz", C.c_int)]


class AmgLevel(C.Structure):
    """The reference's amg_level (C_amg1/include/amg.h:42-54)."""
    _fields_ = [("A", DcsrMat), ("P", DcsrMat), ("A_filtered", DcsrMat),
                ("mis", C.POINTER(C.c_int)), ("isolated", C.POINTER(C.c_int)),
                ("cf_order", C.POINTER(C.c_int)), ("n", C.c_int), ("n_coarse", C.c_int),
                ("L_ichol", IcholFactor), ("l1_diag", C.POINTER(C.c_double))]


class AmgData(C.Structure):
    """The reference's amg_data (C_amg1/include/amg.h:57-71)."""
    _fields_ = [("levels", AmgLevel * 20), ("num_levels", C.c_int), ("threshold", C.c_double),
                ("min_size", C.c_int), ("max_levels", C.c_int), ("maxit_prol", C.c_int),
                ("lump", C.c_int), ("nu", C.c_int), ("smoother", C.c_int),
                ("omega_jacobi", C.c_double), ("coarsening", C.c_int)]


class NetworkSystem(C.Structure):
    """amg_network_system: device CSR + rhs of a vessel network's pressure system."""
    _fields_ = [("n", C.c_int), ("nnz", C.c_int), ("n_nodes", C.c_int),
                ("ia", C.c_void_p), ("ja", C.c_void_p), ("val", C.c_void_p),
                ("rhs", C.c_void_p), ("interior_of", C.c_void_p), ("owner", C.c_void_p)]


# void (*precond)(const void* data, const double* g, double* Bg)
PRECOND_FN = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double))

_lib = None


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Load ``libamg_b200.so`` (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with blood_network_b200.build.build()")
    lib = C.CDLL(path)
    vp, ip, dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)
    i, d = C.c_int, C.c_double
    sig = {
        "amg_solver_create": (vp, [i, i, vp, vp, vp, d, i, i, i]),
        "amg_solver_create_ex": (vp, [i, i, vp, vp, vp, C.POINTER(Options)]),
        "amg_solver_create_device": (vp, [i, i, vp, vp, vp, C.POINTER(Options)]),
        "amg_solver_update": (i, [vp, i, i, vp, vp, vp]),
        "amg_solver_set_matrix": (i, [vp, i, i, vp, vp, vp]),
        "amg_solver_set_smoother": (None, [vp, i, d]),
        "amg_solver_set_precision": (i, [vp, i]),
        "amg_solver_set_stop": (i, [vp, i]),
        "amg_solver_solve": (i, [vp, vp, vp, d, i, i]),
        "amg_solver_solve_device": (i, [vp, vp, vp, d, i, i]),
        "amg_solver_solve_batch": (i, [vp, i, vp, vp, d, i, vp]),
        "amg_solver_solve_segmented": (i, [vp, i, vp, vp, vp, d, i, vp, vp]),
        "amg_solver_solve_block": (i, [vp, i, vp, vp, d, i, vp, vp]),
        "amg_solver_autotune": (i, [vp, i, vp, i]),
        "amg_solver_solve_block_device": (i, [vp, i, vp, vp, d, i, vp, vp]),
        "amg_solver_solve_segmented_device": (i, [vp, i, vp, vp, vp, d, i, vp, vp]),
        "amg_solver_precond": (i, [vp, vp, vp]),
        "amg_solver_size": (i, [vp]),
        "amg_solver_num_levels": (i, [vp]),
        "amg_solver_free": (None, [vp]),
        "amg_solver_stats": (i, [vp, C.POINTER(Stats)]),
        "amg_solver_level_info": (i, [vp, i, ip]),
        "amg_solver_level_copy": (i, [vp, i] + [vp] * 10),
        "amg_solver_bench_kernel": (i, [vp, i, i, i, C.POINTER(C.c_double)]),
        "amg_solver_last_error": (C.c_char_p, []),
        "amg_solver_last_status": (i, []),
        "amg_b200_launch_count": (C.c_ulonglong, []),
        "amg_b200_default_options": (None, [C.POINTER(Options)]),
        "rs_strength": (None, [C.POINTER(DcsrMat), d, C.POINTER(DcsrMat), ip]),
        "pmis_coarsening": (None, [C.POINTER(DcsrMat), vp, ip]),
        "hmis_coarsening": (None, [C.POINTER(DcsrMat), vp, ip]),
        "rs_coarsening": (None, [C.POINTER(DcsrMat), i, vp, ip]),
        "rs_standard_interpolation": (None, [C.POINTER(DcsrMat)] * 2 + [vp, C.POINTER(DcsrMat)]),
        "rs_standard_interpolation_sparsity": (None, [C.POINTER(DcsrMat), vp, C.POINTER(DcsrMat)]),
        "rs_standard_interpolation_values": (None, [C.POINTER(DcsrMat)] * 2 + [vp, C.POINTER(DcsrMat)]),
        "dcsr_rap": (None, [C.POINTER(DcsrMat)] * 4),
        "abyvg": (None, [vp, vp, vp, vp, i, vp]),
        "abyvcs": (None, [vp, vp, vp, vp, i, vp]),
        "abyvam": (None, [vp, vp, vp, vp, vp, i, vp]),
        "vbya": (None, [vp, vp, vp, vp, i, i, vp]),
        "ichol_compute": (None, [C.POINTER(DcsrMat), C.POINTER(IcholFactor)]),
        "ichol_solve": (None, [C.POINTER(IcholFactor), vp, vp]),
        "ichol_free": (None, [C.POINTER(IcholFactor)]),
        "ichol_solve_noalloc": (i, [i, vp, vp, vp, vp, vp, vp]),
        "amg_debug_wait_timeout": (i, [i, d, C.POINTER(C.c_double)]),
        "amg_build_hierarchy": (None, [C.POINTER(AmgData), C.POINTER(DcsrMat)]),
        "amg_rebuild_values": (None, [C.POINTER(AmgData), C.POINTER(DcsrMat)]),
        "amg_free": (None, [C.POINTER(AmgData)]),
        "amg_backslash": (None, [C.POINTER(AmgData), i, vp, vp, i]),
        "amg_fwdslash": (None, [C.POINTER(AmgData), i, vp, vp, i]),
        "amg_vcycle_precond": (None, [C.POINTER(AmgData), vp, vp]),
        "amg_ichol_precond": (None, [C.POINTER(AmgData), C.POINTER(DcsrMat),
                                     C.POINTER(IcholFactor), vp, vp]),
        "amg_pcg": (i, [C.POINTER(DcsrMat), vp, vp, PRECOND_FN, vp, d, i, i]),
        "amg_gauss_seidel_ordered": (i, [i, i, vp, vp, vp, vp, vp, vp, i, i]),
        "amg_network_assemble_device": (i, [i, i, vp, vp, vp, i, vp, vp,
                                            C.POINTER(NetworkSystem)]),
        "amg_network_system_free": (None, [C.POINTER(NetworkSystem)]),
        "amg_network_flows_device": (i, [C.POINTER(NetworkSystem), i, vp, vp, vp, vp, vp]),
        "amg_network_adjoint_device": (i, [vp, C.POINTER(NetworkSystem), i, vp, vp, vp, vp, d,
                                           i, vp, vp, ip]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def exported_symbols():
    """Names declared in include/amg_b200.h that the library must export."""
    import re
    hdr = os.path.join(os.path.dirname(_HERE), "include", "amg_b200.h")
    text = open(hdr).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b([a-z_][a-z0-9_]*)\s*\(", text)
    skip = {"if", "for", "while", "return", "sizeof", "defined", "void"}  # void (*fn)(...)
    return sorted({n for n in names if n not in skip})


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _check(lib, what):
    st = lib.amg_solver_last_status()
    if st != 0:
        raise AMGError(st, f"{what}: {lib.amg_solver_last_error().decode()}")


def default_options(**kw) -> Options:
    lib = load_library()
    o = Options()
    lib.amg_b200_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


@dataclass
class CSRArrays:
    n: int
    indptr: np.ndarray
    indices: np.ndarray
    data: np.ndarray


def as_csr(n, indptr, indices, data) -> CSRArrays:
    return CSRArrays(int(n), np.ascontiguousarray(indptr, dtype=np.int32),
                     np.ascontiguousarray(indices, dtype=np.int32),
                     np.ascontiguousarray(data, dtype=np.float64))


class AMGSolver:
    """Handle over ``amg_solver_*``: setup on construction, ``solve`` per RHS."""

    def __init__(self, n, indptr, indices, data, threshold=0.25, min_size=500, max_levels=20,
                 nu=1, coarsening=COARSEN_PMIS, smoother=SMOOTHER_CF_GS, precision=PREC_FP64,
                 stop=STOP_BNORM, device=0):
        self.lib = load_library()
        a = as_csr(n, indptr, indices, data)
        self._keep = a
        o = default_options(threshold=threshold, min_size=min_size, max_levels=max_levels, nu=nu,
                            coarsening=coarsening, smoother=smoother, precision=precision,
                            stop=stop, device=device)
        self.h = self.lib.amg_solver_create_ex(a.n, int(a.indptr[-1]), _p(a.indptr),
                                               _p(a.indices), _p(a.data), C.byref(o))
        if not self.h:
            raise AMGError(self.lib.amg_solver_last_status(),
                           "amg_solver_create: " + self.lib.amg_solver_last_error().decode())
        self.n = a.n

    def solve(self, b, x0=None, tol=1e-8, maxiter=200, print_level=0):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        it = self.lib.amg_solver_solve(self.h, _p(b), _p(x), tol, maxiter, print_level)
        st = self.lib.amg_solver_last_status()
        if st not in (0, -4, -5):
            raise AMGError(st, self.lib.amg_solver_last_error().decode())
        return x, it

    def solve_batch(self, B, X0=None, tol=1e-8, maxiter=200):
        """Columns of the n x k array B, each solved as ``solve`` would;
        returns (X, iterations per column)."""
        B = np.asfortranarray(B, dtype=np.float64).reshape(self.n, -1, order="F")
        k = B.shape[1]
        X = (np.zeros((self.n, k), order="F") if X0 is None
             else np.array(X0, dtype=np.float64, order="F", copy=True).reshape(self.n, k, order="F"))
        its = np.zeros(k, np.int32)
        rc = self.lib.amg_solver_solve_batch(self.h, k, _p(B), _p(X), tol, maxiter, _p(its))
        if rc not in (0, -4):
            raise AMGError(rc, self.lib.amg_solver_last_error().decode())
        return X, its

    def autotune(self, what=3):
        """Pick the fastest solve-phase kernel variant per level operator;
        returns records (level, operator 0 A / 1 R / 2 P / 3 GS, choice, ms)."""
        rep = np.zeros(4 * 4 * 64)
        m = self.lib.amg_solver_autotune(self.h, what, _p(rep), rep.shape[0])
        if m < 0:
            raise AMGError(m, self.lib.amg_solver_last_error().decode())
        return rep[:4 * m].reshape(m, 4)

    def solve_block(self, B, X0=None, tol=1e-8, maxiter=200):
        """The columns of the n x k array B (k <= 64) solved together, each
        with its own PCG; returns (X, iterations, relres, status)."""
        B = np.asfortranarray(B, dtype=np.float64).reshape(self.n, -1, order="F")
        k = B.shape[1]
        X = (np.zeros((self.n, k), order="F") if X0 is None
             else np.array(X0, dtype=np.float64, order="F", copy=True).reshape(self.n, k, order="F"))
        its, rel = np.zeros(k, np.int32), np.zeros(k)
        rc = self.lib.amg_solver_solve_block(self.h, k, _p(B), _p(X), tol, maxiter, _p(its),
                                             _p(rel))
        if rc not in (0, -4, -5):
            raise AMGError(rc, self.lib.amg_solver_last_error().decode())
        return X, its, rel, rc

    def solve_segmented(self, seg_ptr, b, x0=None, tol=1e-8, maxiter=200):
        """Block-diagonal independent systems (segment k: rows seg_ptr[k] ..
        seg_ptr[k+1]-1), each with its own PCG; returns (x, iterations,
        relres, status) with per-segment iterations and true relative
        residuals."""
        ptr = np.ascontiguousarray(seg_ptr, np.int32)
        nseg = len(ptr) - 1
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        its, rel = np.zeros(nseg, np.int32), np.zeros(nseg)
        rc = self.lib.amg_solver_solve_segmented(self.h, nseg, _p(ptr), _p(b), _p(x), tol,
                                                 maxiter, _p(its), _p(rel))
        if rc not in (0, -4, -5):
            raise AMGError(rc, self.lib.amg_solver_last_error().decode())
        return x, its, rel, rc

    def precond(self, g):
        g = np.ascontiguousarray(g, dtype=np.float64)
        x = np.zeros(self.n)
        rc = self.lib.amg_solver_precond(self.h, _p(g), _p(x))
        if rc != 0:
            raise AMGError(rc, self.lib.amg_solver_last_error().decode())
        return x

    def set_precision(self, p):
        rc = self.lib.amg_solver_set_precision(self.h, p)
        if rc != 0:
            raise AMGError(rc, self.lib.amg_solver_last_error().decode())

    def set_stop(self, s):
        self.lib.amg_solver_set_stop(self.h, s)

    def set_smoother(self, sm, omega=0.5):
        self.lib.amg_solver_set_smoother(self.h, sm, omega)
        _check(self.lib, "set_smoother")

    def update(self, indptr, indices, data):
        a = as_csr(self.n, indptr, indices, data)
        rc = self.lib.amg_solver_update(self.h, a.n, int(a.indptr[-1]), _p(a.indptr),
                                        _p(a.indices), _p(a.data))
        if rc != 0:
            raise AMGError(rc, self.lib.amg_solver_last_error().decode())

    def set_matrix(self, indptr, indices, data):
        a = as_csr(self.n, indptr, indices, data)
        rc = self.lib.amg_solver_set_matrix(self.h, a.n, int(a.indptr[-1]), _p(a.indptr),
                                            _p(a.indices), _p(a.data))
        if rc != 0:
            raise AMGError(rc, self.lib.amg_solver_last_error().decode())

    def bench_kernel(self, which, precision=0, reps=20):
        ms = C.c_double()
        rc = self.lib.amg_solver_bench_kernel(self.h, which, precision, reps, C.byref(ms))
        if rc != 0:
            raise AMGError(rc, self.lib.amg_solver_last_error().decode())
        return ms.value

    def solve_device(self, d_b, d_x, tol=1e-8, maxiter=200, print_level=0):
        """Solve with device pointers (ints), e.g. torch tensors' data_ptr()."""
        it = self.lib.amg_solver_solve_device(self.h, C.c_void_p(d_b), C.c_void_p(d_x), tol,
                                              maxiter, print_level)
        st = self.lib.amg_solver_last_status()
        if st not in (0, -4, -5):
            raise AMGError(st, self.lib.amg_solver_last_error().decode())
        return it

    @property
    def num_levels(self):
        return self.lib.amg_solver_num_levels(self.h)

    def stats(self) -> Stats:
        s = Stats()
        self.lib.amg_solver_stats(self.h, C.byref(s))
        return s

    def level(self, k):
        """Level k's A, S, P (as (indptr, indices, data)) and C/F marks."""
        info = (C.c_int * 5)()
        if self.lib.amg_solver_level_info(self.h, k, info) != 0:
            raise IndexError(k)
        n, annz, snnz, pnnz, nc = list(info)
        A = (np.zeros(n + 1, np.int32), np.zeros(annz, np.int32), np.zeros(annz))
        last = k == self.num_levels - 1
        if last:
            S = P = cf = None
            self.lib.amg_solver_level_copy(self.h, k, _p(A[0]), _p(A[1]), _p(A[2]),
                                           *([None] * 7))
        else:
            S = (np.zeros(n + 1, np.int32), np.zeros(snnz, np.int32), np.zeros(snnz))
            P = (np.zeros(n + 1, np.int32), np.zeros(pnnz, np.int32), np.zeros(pnnz))
            cf = np.zeros(n, np.int32)
            self.lib.amg_solver_level_copy(self.h, k, _p(A[0]), _p(A[1]), _p(A[2]), _p(S[0]),
                                           _p(S[1]), _p(S[2]), _p(P[0]), _p(P[1]), _p(P[2]),
                                           _p(cf))
        return dict(n=n, n_coarse=nc, A=A, S=S, P=P, cf=cf)

    def close(self):
        if getattr(self, "h", None):
            self.lib.amg_solver_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
