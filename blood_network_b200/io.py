"""The reference's on-disk formats.

* COO text matrices (``C_amg1/src/io.c:71-124``) and right-hand-side files
  (``C_amg1/test_amg.c:126-148``): read by the library's C entry points
  ``amg_read_coo`` / ``amg_read_vector``.
* Network cases (``Matlab_amg/caseReaderMJ.m:1-33``): ``<prefix>.fMx`` faces
  (column 2 and 3: 1-based end nodes), ``.pMx`` node coordinates, ``.dia``
  diameters, ``.BC`` boundary rows (column 1: 1-based node, column 3:
  pressure).  ``case_network`` forms the Dirichlet-reduced system as
  ``Matlab_amg/read_nwk.m:17-36`` does with the Cartesian diffusive
  conductances of ``Matlab_amg/makeDiffusiveConductance.m:2-13``.
* Labelled solutions (``Matlab_amg/label_solution.m:41-44``).
"""
import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import amg
from .network import Network, assemble


def _lib():
    lib = amg.load_library()
    vp, i = C.c_void_p, C.c_int
    ip = C.POINTER(C.c_int)
    lib.amg_read_coo.restype = i
    lib.amg_read_coo.argtypes = [C.c_char_p, ip, ip, ip, C.POINTER(ip), C.POINTER(ip),
                                 C.POINTER(C.POINTER(C.c_double))]
    lib.amg_free_host.argtypes = [vp]
    lib.amg_free_host.restype = None
    lib.amg_read_vector.restype = i
    lib.amg_read_vector.argtypes = [C.c_char_p, i, vp]
    lib.amg_write_labeled_solution.restype = i
    lib.amg_write_labeled_solution.argtypes = [C.c_char_p, i, vp, vp]
    return lib


def read_coo(path):
    """(nrow, ncol, indptr, indices, data) of a COO text file, converted as
    the reference converts it (entries of a row in file order, duplicates
    kept)."""
    lib = _lib()
    m, n, nnz = C.c_int(), C.c_int(), C.c_int()
    ia, ja = C.POINTER(C.c_int)(), C.POINTER(C.c_int)()
    val = C.POINTER(C.c_double)()
    rc = lib.amg_read_coo(os.fsencode(path), C.byref(m), C.byref(n), C.byref(nnz), C.byref(ia),
                          C.byref(ja), C.byref(val))
    if rc != 0:
        raise amg.AMGError(rc, lib.amg_solver_last_error().decode())
    try:
        indptr = np.ctypeslib.as_array(ia, shape=(m.value + 1,)).copy()
        k = nnz.value
        indices = np.ctypeslib.as_array(ja, shape=(k,)).copy() if k else np.zeros(0, np.int32)
        data = np.ctypeslib.as_array(val, shape=(k,)).copy() if k else np.zeros(0)
    finally:
        for p in (ia, ja, val):
            lib.amg_free_host(C.cast(p, C.c_void_p))
    return m.value, n.value, indptr, indices, data


def read_vector(path, n):
    """The n values of a right-hand-side file ("n" then the values)."""
    lib = _lib()
    out = np.zeros(n)
    rc = lib.amg_read_vector(os.fsencode(path), n, out.ctypes.data)
    if rc != 0:
        raise amg.AMGError(rc, lib.amg_solver_last_error().decode())
    return out


def write_labeled_solution(path, interior_nodes, p):
    """One "%d %.16e" line per interior node: its 1-based id and pressure."""
    lib = _lib()
    node = np.ascontiguousarray(interior_nodes, np.int32)
    p = np.ascontiguousarray(p, np.float64)
    if node.shape != p.shape:
        raise ValueError("write_labeled_solution: one pressure per node")
    rc = lib.amg_write_labeled_solution(os.fsencode(path), node.shape[0], node.ctypes.data,
                                        p.ctypes.data)
    if rc != 0:
        raise amg.AMGError(rc, lib.amg_solver_last_error().decode())


# ------------------------------------------------------------ network cases
@dataclass
class Case:
    faces: np.ndarray    # faceMx, rows of the .fMx file (columns 2, 3: 1-based nodes)
    coords: np.ndarray   # ptCoordMx
    dia: np.ndarray
    bc: np.ndarray       # BC rows: node (1-based), type, pressure
    np_: int             # node count, MATLAB's length(ptCoordMx)
    nf: int
    nt: int


def _load(path):
    """MATLAB ``load`` of a numeric text file; an empty file is []."""
    if os.path.getsize(path) == 0:
        return np.zeros((0, 0))
    a = np.loadtxt(path, ndmin=2)
    return a


def read_case(prefix) -> Case:
    """caseReaderMJ.m: the four files of a network case."""
    faces = _load(prefix + ".fMx")
    coords = _load(prefix + ".pMx")
    dia = _load(prefix + ".dia")
    bc = _load(prefix + ".BC")
    npts = max(coords.shape) if coords.size else 0  # length(): the larger dimension
    nf = faces.shape[0]
    return Case(faces, coords, dia, bc, int(npts), int(nf), int(npts + nf))


def diffusive_conductance(faces, coords):
    """makeDiffusiveConductance.m: faces whose vector (end node minus start
    node) has a positive x, y or z component get hy*hz/hx, hx*hz/hy or
    hx*hy/hz (later directions win), h the length of the first such face;
    every other face gets NaN."""
    p1 = faces[:, 1].astype(np.int64) - 1
    p2 = faces[:, 2].astype(np.int64) - 1
    vec = coords[p2, :] - coords[p1, :]
    g = np.full(faces.shape[0], np.nan)
    h = []
    sel = []
    for d in range(3):
        idx = np.nonzero(vec[:, d] > 0)[0]
        sel.append(idx)
        h.append(np.sqrt(np.sum(vec[idx[0], :] ** 2)) if idx.size else np.nan)
    hx, hy, hz = h
    g[sel[0]] = hy * hz / hx
    g[sel[1]] = hx * hz / hy
    g[sel[2]] = hx * hy / hz
    return g


def case_network(prefix, conductance=None) -> Network:
    """read_nwk.m: LHS = C_I^T W C_I and RHS = -C_I^T W C_B p_B with W the
    diffusive conductances (or the given per-face ``conductance``)."""
    c = read_case(prefix)
    seg_u = c.faces[:, 1].astype(np.int64) - 1
    seg_v = c.faces[:, 2].astype(np.int64) - 1
    g = diffusive_conductance(c.faces, c.coords) if conductance is None else \
        np.asarray(conductance, np.float64)
    boundary = c.bc[:, 0].astype(np.int64) - 1
    return assemble(c.np_, seg_u, seg_v, g, boundary, c.bc[:, 2].astype(np.float64))
