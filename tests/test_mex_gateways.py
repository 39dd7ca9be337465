"""The MATLAB gateways (blood_network_b200/mex): compiled against the local mex.h
and run through a stand-in MATLAB runtime (tests/mex/mxfake.c), since no MATLAB
is installed.  Argument checks and error ids on the CPU; outputs, classes and
values against the library's C entry points (or the sequential sweep) on the GPU.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from blood_network_b200 import amg
from blood_network_b200.network import vascular_network

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MEX = os.path.join(ROOT, "blood_network_b200", "mex")
LIBDIR = os.path.join(ROOT, "blood_network_b200", "lib")
GATEWAYS = ["rs_strength_mex", "rs_coarsening_mex", "rs_interpolation_mex",
            "cf_gauss_seidel_mex"]
MX_DOUBLE, MX_INT32 = 6, 12


def _build(name, outdir):
    so = os.path.join(outdir, f"{name}.so")
    cmd = ["gcc", "-std=c99", "-O2", "-Wall", "-Werror", "-shared", "-fPIC", f"-I{MEX}",
           f"-I{os.path.join(ROOT, 'include')}", os.path.join(MEX, f"{name}.c"),
           os.path.join(ROOT, "tests", "mex", "mxfake.c"), f"-L{LIBDIR}", "-lamg_b200",
           f"-Wl,-rpath,{LIBDIR}", "-o", so]
    subprocess.run(cmd, check=True, capture_output=True)
    lib = C.CDLL(so)
    vp, sz = C.c_void_p, C.c_size_t
    lib.mxfake_run.restype = C.c_int
    lib.mxfake_run.argtypes = [C.c_int, C.POINTER(vp), C.c_int, C.POINTER(vp)]
    lib.mxfake_error_id.restype = C.c_char_p
    lib.mxfake_sparse.restype = vp
    lib.mxfake_sparse.argtypes = [sz, sz, sz, vp, vp, vp]
    lib.mxfake_double.restype = vp
    lib.mxfake_double.argtypes = [sz, sz, vp]
    lib.mxfake_int32.restype = vp
    lib.mxfake_int32.argtypes = [C.c_int]
    for f in ("mxfake_m", "mxfake_n", "mxfake_nnz"):
        getattr(lib, f).restype = sz
        getattr(lib, f).argtypes = [vp]
    lib.mxfake_class.argtypes = [vp]
    lib.mxfake_is_sparse.argtypes = [vp]
    lib.mxfake_int32_value.argtypes = [vp]
    lib.mxfake_copy_sparse.argtypes = [vp, vp, vp, vp]
    lib.mxfake_copy_double.argtypes = [vp, vp]
    lib.mxfake_free.argtypes = [vp]
    return lib


@pytest.fixture(scope="module")
def gw(tmp_path_factory):
    amg.load_library()  # the gateways link libamg_b200.so
    d = str(tmp_path_factory.mktemp("mex"))
    return {g: _build(g, d) for g in GATEWAYS}


class Mx:
    """Builds inputs and reads outputs through the stand-in runtime."""

    def __init__(self, lib):
        self.lib = lib
        self.keep = []

    def sparse(self, indptr, indices, data, m, n):
        jc = np.ascontiguousarray(indptr, np.int64)
        ir = np.ascontiguousarray(indices, np.int64)
        pr = np.ascontiguousarray(data, np.float64)
        self.keep += [jc, ir, pr]
        return self.lib.mxfake_sparse(m, n, len(ir), jc.ctypes.data, ir.ctypes.data,
                                      pr.ctypes.data)

    def dense(self, v):
        v = np.ascontiguousarray(v, np.float64).reshape(-1)
        self.keep.append(v)
        return self.lib.mxfake_double(len(v), 1, v.ctypes.data)

    def run(self, nlhs, inputs):
        prhs = (C.c_void_p * max(len(inputs), 1))(*inputs)
        plhs = (C.c_void_p * max(nlhs, 1))()
        rc = self.lib.mxfake_run(nlhs, plhs, len(inputs), prhs)
        return rc, list(plhs)[:nlhs], self.lib.mxfake_error_id().decode()

    def read_sparse(self, a):
        n, nnz = self.lib.mxfake_n(a), self.lib.mxfake_nnz(a)
        jc, ir, pr = np.zeros(n + 1, np.int64), np.zeros(nnz, np.int64), np.zeros(nnz)
        self.lib.mxfake_copy_sparse(a, jc.ctypes.data, ir.ctypes.data, pr.ctypes.data)
        return jc, ir, pr

    def read_dense(self, a):
        out = np.zeros(self.lib.mxfake_m(a) * self.lib.mxfake_n(a))
        self.lib.mxfake_copy_double(a, out.ctypes.data)
        return out


def _net():
    return vascular_network(depth=8, n_nodes=3000, seed=4)


# ------------------------------------------------------------ CPU: arguments
@pytest.mark.parametrize("name,nrhs,errid", [
    ("rs_strength_mex", 1, "rs_str:nrhs"), ("rs_coarsening_mex", 3, "rs_coarsen:nrhs"),
    ("rs_interpolation_mex", 2, "rs_interp:nrhs"), ("cf_gauss_seidel_mex", 5, "cf_gs:nrhs")])
def test_argument_count_errors(gw, name, nrhs, errid):
    mx = Mx(gw[name])
    args = [mx.dense(np.ones(3)) for _ in range(nrhs)]
    rc, _, got = mx.run(1, args)
    assert rc == 1 and got == errid


@pytest.mark.parametrize("name,nrhs,errid", [
    ("rs_strength_mex", 2, "rs_str:notSparse"), ("rs_coarsening_mex", 2, "rs_coarsen:notSparse"),
    ("rs_interpolation_mex", 3, "rs_interp:A"), ("cf_gauss_seidel_mex", 6, "cf_gs:notSparse")])
def test_dense_matrix_rejected(gw, name, nrhs, errid):
    mx = Mx(gw[name])
    rc, _, got = mx.run(1, [mx.dense(np.ones(3)) for _ in range(nrhs)])
    assert rc == 1 and got == errid


def test_interpolation_sparse_s_and_lam_max_class(gw):
    net = _net()
    mx = Mx(gw["rs_interpolation_mex"])
    A = mx.sparse(net.indptr, net.indices, net.data, net.n, net.n)
    rc, _, got = mx.run(1, [A, mx.dense(np.ones(3)), mx.dense(np.ones(net.n))])
    assert rc == 1 and got == "rs_interp:S"
    mx = Mx(gw["rs_coarsening_mex"])
    S = mx.sparse(net.indptr, net.indices, net.data, net.n, net.n)
    rc, _, got = mx.run(1, [S, mx.dense(np.array([7.0]))])  # a double, not an int32
    assert rc == 1 and got == "rs_coarsen:badLamMax"


# ------------------------------------------------------------ GPU: values
def _dcsr(ia, ja, val, n, m=None):
    ia, ja, val = (np.ascontiguousarray(ia, np.int32), np.ascontiguousarray(ja, np.int32),
                   np.ascontiguousarray(val, np.float64))
    return amg.DcsrMat(n, n if m is None else m, int(ia[-1]),
                       ia.ctypes.data_as(C.POINTER(C.c_int)),
                       ja.ctypes.data_as(C.POINTER(C.c_int)),
                       val.ctypes.data_as(C.POINTER(C.c_double))), (ia, ja, val)


def _csr_out(m):
    return (np.ctypeslib.as_array(m.ia, shape=(m.row + 1,)).copy(),
            np.ctypeslib.as_array(m.ja, shape=(m.nnz,)).copy(),
            np.ctypeslib.as_array(m.val, shape=(m.nnz,)).copy())


def _csc_of(ia, ja, val, m, n):
    import scipy.sparse as sp
    c = sp.csr_matrix((val, ja, ia), shape=(m, n)).tocsc()
    c.has_sorted_indices = False
    c.sort_indices()
    return c.indptr.astype(np.int64), c.indices.astype(np.int64), c.data


@pytest.mark.gpu
def test_gateways_match_the_c_entry_points(gw):
    lib = amg.load_library()
    net = _net()
    n = net.n
    # [S, lam_max] = rs_strength_mex(A, 0.25)
    mx = Mx(gw["rs_strength_mex"])
    A = mx.sparse(net.indptr, net.indices, net.data, n, n)
    rc, (S_mx, lam_mx), eid = mx.run(2, [A, mx.dense(np.array([0.25]))])
    assert rc == 0, eid
    assert mx.lib.mxfake_is_sparse(S_mx) and mx.lib.mxfake_class(lam_mx) == MX_INT32
    Ad, keepA = _dcsr(net.indptr, net.indices, net.data, n)
    Sd = amg.DcsrMat()
    lam = C.c_int()
    lib.rs_strength(C.byref(Ad), 0.25, C.byref(Sd), C.byref(lam))
    S = _csr_out(Sd)
    assert mx.lib.mxfake_int32_value(lam_mx) == lam.value
    for a, b in zip(mx.read_sparse(S_mx), _csc_of(*S, n, n)):
        assert np.array_equal(a, b)
    # [cf, nc] = rs_coarsening_mex(S, lam_max)
    mx2 = Mx(gw["rs_coarsening_mex"])
    jc, ir, pr = mx.read_sparse(S_mx)
    S_in = mx2.sparse(jc, ir, pr, n, n)
    rc, (cf_mx, nc_mx), eid = mx2.run(2, [S_in, mx2.lib.mxfake_int32(lam.value)])
    assert rc == 0, eid
    cf = mx2.read_dense(cf_mx)
    cfd = np.zeros(n, np.int32)
    ncd = C.c_int()
    lib.rs_coarsening(C.byref(Sd), lam.value, amg._p(cfd), C.byref(ncd))
    assert np.array_equal(cf, cfd.astype(np.float64))
    assert mx2.read_dense(nc_mx)[0] == ncd.value
    # P = rs_interpolation_mex(A, S, cf)
    mx3 = Mx(gw["rs_interpolation_mex"])
    rc, (P_mx,), eid = mx3.run(1, [mx3.sparse(net.indptr, net.indices, net.data, n, n),
                                   mx3.sparse(jc, ir, pr, n, n), mx3.dense(cf)])
    assert rc == 0, eid
    Pd = amg.DcsrMat()
    lib.rs_standard_interpolation(C.byref(Ad), C.byref(Sd), amg._p(cfd), C.byref(Pd))
    P = _csr_out(Pd)
    assert mx3.lib.mxfake_m(P_mx) == n and mx3.lib.mxfake_n(P_mx) == Pd.col
    for a, b in zip(mx3.read_sparse(P_mx), _csc_of(*P, n, Pd.col)):
        assert np.array_equal(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("direction", [0, 1])
def test_cf_gauss_seidel_gateway(gw, direction):
    from test_gpu_ordered_gs import sequential
    net = _net()
    n = net.n
    rng = np.random.default_rng(9)
    b, x0 = rng.standard_normal(n), rng.standard_normal(n)
    c = rng.random(n) < 0.3
    order = np.concatenate([np.nonzero(c)[0], np.nonzero(~c)[0]])
    mx = Mx(gw["cf_gauss_seidel_mex"])
    rc, (x_mx,), eid = mx.run(1, [mx.sparse(net.indptr, net.indices, net.data, n, n),
                                  mx.dense(b), mx.dense(x0), mx.dense(order + 1.0),
                                  mx.dense(np.array([2.0])), mx.dense(np.array([float(direction)]))])
    assert rc == 0, eid
    want = sequential(net.indptr, net.indices, net.data, b, x0, order, 2, direction)
    assert mx.read_dense(x_mx).tobytes() == want.tobytes()
