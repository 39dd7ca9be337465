"""Seeded synthetic vascular networks and their Dirichlet-reduced pressure systems.

The reference ships no network data; its MATLAB layer assembles the pressure
system of a vessel network as

    LHS = C_I^T G C_I,     RHS = -C_I^T G C_B p_B

(``Matlab_amg/read_nwk.m:17-36``), where ``C`` is the segment/node incidence
matrix (``Matlab_amg/ConnectivityMx.m:10-13``), ``G`` the diagonal of segment
conductances and ``I``/``B`` the interior and Dirichlet node sets.  This module
builds networks of the same kind from a seed and assembles that system:

* an arterial binary tree and a mirrored venous binary tree, each with
  ``depth`` generations (``2**depth - 1`` nodes, heap order), joined at their
  leaves by a 3D capillary lattice;
* tree segment radius ``1 mm * 0.79**(g-1)`` at generation ``g`` with +-10%
  jitter; capillary (lattice and leaf connector) radius log-uniform between
  3 um and the radius of the last tree generation, so radii span 3 um - 1 mm;
* segment length uniform in [50, 500] um;
* Poiseuille conductance ``g = pi r^4 / (8 mu L)`` with mu = 3.5e-3 Pa s,
  optionally plus a diffusive term ``D pi r^2 / L`` (D = 2e-9 m^2/s) on a
  random fraction of segments;
* lattice: every x-edge is kept, y/z edges are dropped with probability
  ``lattice_drop`` (interior degree 4-6, mean 5) except a backbone (the z=0
  plane and the z-edges of the x=0 column) that keeps the lattice connected;
* Dirichlet pressures 13.3 kPa at the arterial root and 2 kPa at the venous
  root, eliminated exactly as ``read_nwk.m`` does.

The matrix is returned as 0-based CSR (int32 indices, float64 values, columns
sorted, diagonal stored), the layout the reference C API takes
(``C_amg1/src/amg_wrapper.c:51-97``).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

MU_BLOOD = 3.5e-3  # Pa s
D_DIFFUSION = 2e-9  # m^2 / s
P_INLET = 13.3e3  # Pa, arterial root
P_OUTLET = 2.0e3  # Pa, venous root


@dataclass
class Network:
    """A vessel network and its Dirichlet-reduced pressure system."""

    n: int                 # interior unknowns
    indptr: np.ndarray     # int32 [n+1]
    indices: np.ndarray    # int32 [nnz]
    data: np.ndarray       # float64 [nnz]
    rhs: np.ndarray        # float64 [n]
    # segment description (full node numbering, before elimination)
    seg_u: np.ndarray = field(repr=False, default=None)
    seg_v: np.ndarray = field(repr=False, default=None)
    radius: np.ndarray = field(repr=False, default=None)
    length: np.ndarray = field(repr=False, default=None)
    conductance: np.ndarray = field(repr=False, default=None)
    diffusive: np.ndarray = field(repr=False, default=None)  # bool mask
    n_total: int = 0                # nodes before elimination
    boundary: np.ndarray = field(repr=False, default=None)  # Dirichlet node ids
    p_boundary: np.ndarray = field(repr=False, default=None)
    interior_of: np.ndarray = field(repr=False, default=None)  # full id -> interior id or -1

    @property
    def nnz(self) -> int:
        return int(self.indptr[-1])

    @property
    def n_segments(self) -> int:
        return int(self.seg_u.shape[0])


def _lattice_dims(n_lat: int):
    side = max(2, int(round(n_lat ** (1.0 / 3.0))))
    nx = ny = side
    nz = max(2, int(np.ceil(n_lat / float(nx * ny))))
    return nx, ny, nz


def _tree_edges(T: int, offset: int):
    child = np.arange(1, T, dtype=np.int64)
    parent = (child - 1) // 2
    gen = np.floor(np.log2(child + 1)).astype(np.int64)  # generation of the child
    return parent + offset, child + offset, gen


def vascular_network(depth: int, n_nodes: int, seed: int = 0,
                     diffusive_fraction: float = 0.0,
                     lattice_drop: float = 0.25,
                     p_inlet: float = P_INLET, p_outlet: float = P_OUTLET,
                     keep_segments: bool = True) -> Network:
    """Build the pressure system of a seeded arterial-capillary-venous network.

    ``depth`` is the number of generations per tree; ``n_nodes`` the target
    node count (the lattice takes whatever the two trees leave).
    """
    if depth < 2:
        raise ValueError("depth must be >= 2")
    rng = np.random.default_rng(seed)
    T = (1 << depth) - 1
    n_lat_target = max(n_nodes - 2 * T, 8)
    nx, ny, nz = _lattice_dims(n_lat_target)
    n_lat = nx * ny * nz
    lat0 = T                 # first lattice node
    ven0 = T + n_lat         # venous root
    n_total = 2 * T + n_lat

    # ---- trees -------------------------------------------------------
    au, av, agen = _tree_edges(T, 0)
    vu, vv, vgen = _tree_edges(T, ven0)
    tree_gen = np.concatenate([agen, vgen])
    r_tree = 1e-3 * 0.79 ** (tree_gen - 1).astype(np.float64)
    r_tree *= rng.uniform(0.9, 1.1, size=r_tree.shape[0])
    r_leaf = 1e-3 * 0.79 ** (depth - 2)
    r_cap_hi = max(r_leaf, 3.0e-6 * 1.0001)

    # ---- leaf connectors ----------------------------------------------
    n_leaf = 1 << (depth - 1)
    leaf = np.arange(n_leaf, dtype=np.int64)
    a_leaf = (T // 2) + leaf
    v_leaf = ven0 + (T // 2) + leaf
    a_tgt = lat0 + (leaf * n_lat) // n_leaf
    v_tgt = lat0 + ((leaf * n_lat) // n_leaf + max(1, n_lat // (2 * n_leaf))) % n_lat

    # ---- lattice -------------------------------------------------------
    idx = np.arange(n_lat, dtype=np.int64)
    x = idx % nx
    y = (idx // nx) % ny
    z = idx // (nx * ny)
    ex = idx[x < nx - 1]
    lx_u, lx_v = ex, ex + 1
    ey = idx[y < ny - 1]
    keep_y = (rng.random(ey.shape[0]) >= lattice_drop) | (z[ey] == 0)
    ly_u, ly_v = ey[keep_y], ey[keep_y] + nx
    ez = idx[z < nz - 1]
    keep_z = (rng.random(ez.shape[0]) >= lattice_drop) | (x[ez] == 0)
    lz_u, lz_v = ez[keep_z], ez[keep_z] + nx * ny
    lat_u = lat0 + np.concatenate([lx_u, ly_u, lz_u])
    lat_v = lat0 + np.concatenate([lx_v, ly_v, lz_v])

    cap_u = np.concatenate([a_leaf, v_tgt, lat_u])
    cap_v = np.concatenate([a_tgt, v_leaf, lat_v])
    lo, hi = np.log(3.0e-6), np.log(r_cap_hi)
    r_cap = np.exp(rng.uniform(lo, hi, size=cap_u.shape[0]))

    seg_u = np.concatenate([au, vu, cap_u])
    seg_v = np.concatenate([av, vv, cap_v])
    radius = np.concatenate([r_tree, r_cap])
    m = seg_u.shape[0]
    length = rng.uniform(50e-6, 500e-6, size=m)
    g = np.pi * radius ** 4 / (8.0 * MU_BLOOD * length)
    diff_mask = np.zeros(m, dtype=bool)
    if diffusive_fraction > 0.0:
        diff_mask = rng.random(m) < diffusive_fraction
        g = g + np.where(diff_mask, D_DIFFUSION * np.pi * radius ** 2 / length, 0.0)

    net = assemble(n_total, seg_u, seg_v, g,
                   boundary=np.array([0, ven0], dtype=np.int64),
                   p_boundary=np.array([p_inlet, p_outlet]))
    if keep_segments:
        net.radius, net.length, net.diffusive = radius, length, diff_mask
    else:
        net.seg_u = net.seg_v = net.conductance = None
    return net


def assemble(n_total: int, seg_u: np.ndarray, seg_v: np.ndarray, g: np.ndarray,
             boundary: np.ndarray, p_boundary: np.ndarray) -> Network:
    """Dirichlet-reduced weighted graph Laplacian, as ``read_nwk.m:17-36``.

    Returns CSR of ``C_I^T G C_I`` and ``RHS = -C_I^T G C_B p_B``.
    """
    interior_of = np.full(n_total, -1, dtype=np.int64)
    is_b = np.zeros(n_total, dtype=bool)
    is_b[boundary] = True
    interior = np.nonzero(~is_b)[0]
    interior_of[interior] = np.arange(interior.shape[0])
    n = interior.shape[0]
    pb_full = np.zeros(n_total)
    pb_full[boundary] = p_boundary

    iu, iv = interior_of[seg_u], interior_of[seg_v]
    # diagonal: every segment contributes g to each interior endpoint
    diag = np.zeros(n)
    np.add.at(diag, iu[iu >= 0], g[iu >= 0])
    np.add.at(diag, iv[iv >= 0], g[iv >= 0])
    # rhs: segments with one Dirichlet end
    rhs = np.zeros(n)
    mu_ = (iu >= 0) & (iv < 0)
    np.add.at(rhs, iu[mu_], g[mu_] * pb_full[seg_v[mu_]])
    mv_ = (iv >= 0) & (iu < 0)
    np.add.at(rhs, iv[mv_], g[mv_] * pb_full[seg_u[mv_]])

    both = (iu >= 0) & (iv >= 0)
    ru = np.concatenate([iu[both], iv[both], np.arange(n)])
    rv = np.concatenate([iv[both], iu[both], np.arange(n)])
    vals = np.concatenate([-g[both], -g[both], diag])
    # sort by (row, col); duplicate (row, col) pairs are summed
    key = ru * n + rv
    order = np.argsort(key, kind="stable")
    key = key[order]
    vals = vals[order]
    uniq, start = np.unique(key, return_index=True)
    summed = np.add.reduceat(vals, start) if vals.shape[0] else vals
    rows = (uniq // n).astype(np.int64)
    cols = (uniq % n).astype(np.int32)
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(indptr, rows + 1, 1)
    indptr = np.cumsum(indptr)
    if indptr[-1] >= 2**31:
        raise ValueError("nnz exceeds int32 range")
    return Network(n=n, indptr=indptr.astype(np.int32), indices=cols,
                   data=summed.astype(np.float64), rhs=rhs,
                   seg_u=seg_u, seg_v=seg_v, conductance=g,
                   n_total=n_total, boundary=boundary, p_boundary=p_boundary,
                   interior_of=interior_of)


# Named workloads (node counts, tree depth, coarsening and threshold).
CONFIGS = {
    # ~20k nodes: trees of depth 12 + lattice; PMIS, theta 0.25
    "vascular_20k": dict(depth=12, n_nodes=20_000, diffusive_fraction=0.0,
                         coarsening="pmis", theta=0.25),
    # 2M nodes: trees of depth 19 + lattice; PMIS, theta 0.25
    "vascular_2m": dict(depth=19, n_nodes=2_000_000, diffusive_fraction=0.0,
                        coarsening="pmis", theta=0.25),
    # 20M nodes: trees of depth 22 + lattice, diffusive term on 30% of
    # segments; HMIS, theta 0.5
    "vascular_20m": dict(depth=22, n_nodes=20_000_000, diffusive_fraction=0.3,
                         coarsening="hmis", theta=0.5),
    # 5M nodes, the many-right-hand-side workload: trees of depth 20 + lattice
    "vascular_5m": dict(depth=20, n_nodes=5_000_000, diffusive_fraction=0.0,
                        coarsening="pmis", theta=0.25),
    # 4M nodes with the 20M network's options (profiling case: its fine
    # matrix, ~240 MB, is larger than the 126 MB L2 but small on the device)
    "vascular_4m": dict(depth=20, n_nodes=4_000_000, diffusive_fraction=0.3,
                        coarsening="hmis", theta=0.5),
}


def make_config(name: str, seed: int = 0, **kw) -> Network:
    c = dict(CONFIGS[name])
    c.pop("coarsening"), c.pop("theta")
    c.update(kw)
    return vascular_network(seed=seed, **c)


def block_diagonal(nets):
    """Independent networks packed into one block-diagonal system (the
    multi-network batch): returns (n, indptr, indices, data, rhs, seg_ptr),
    network k holding rows seg_ptr[k] .. seg_ptr[k+1]-1 in its own order."""
    sizes = np.array([nt.n for nt in nets], np.int64)
    seg_ptr = np.zeros(len(nets) + 1, np.int64)
    np.cumsum(sizes, out=seg_ptr[1:])
    nnzs = np.array([nt.nnz for nt in nets], np.int64)
    nz_ptr = np.zeros(len(nets) + 1, np.int64)
    np.cumsum(nnzs, out=nz_ptr[1:])
    if seg_ptr[-1] > np.iinfo(np.int32).max or nz_ptr[-1] > np.iinfo(np.int32).max:
        raise ValueError("block_diagonal: the packed system exceeds 32-bit CSR indices")
    indptr = np.concatenate([[0]] + [nt.indptr[1:].astype(np.int64) + nz_ptr[k]
                                     for k, nt in enumerate(nets)])
    indices = np.concatenate([nt.indices.astype(np.int64) + seg_ptr[k]
                              for k, nt in enumerate(nets)])
    data = np.concatenate([nt.data for nt in nets])
    rhs = np.concatenate([nt.rhs for nt in nets])
    return (int(seg_ptr[-1]), indptr.astype(np.int32), indices.astype(np.int32), data, rhs,
            seg_ptr.astype(np.int32))


def batch_networks(count: int = 256, lo: int = 5_000, hi: int = 200_000, seed: int = 0):
    """Independent networks of the multi-network batch: node counts
    log-uniform in [lo, hi], trees of depth round(log2(0.2 n)) (the depth
    the named configs use for their sizes), seeds seed+1 .. seed+count."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), count)).astype(np.int64)
    nets = []
    for k, m in enumerate(sizes):
        depth = max(4, int(round(np.log2(0.2 * m))))
        nets.append(vascular_network(depth=depth, n_nodes=int(m), seed=seed + 1 + k,
                                     keep_segments=False))
    return nets
