"""Synthetic vascular networks: the assembled system is the Dirichlet-reduced
graph Laplacian of read_nwk.m (LHS = C_I^T G C_I, RHS = -C_I^T G C_B p_B)."""
import numpy as np
import scipy.sparse as sp

from blood_network_b200.network import vascular_network, make_config, P_INLET, P_OUTLET


def test_laplacian_structure():
    net = vascular_network(depth=8, n_nodes=3000, seed=1, diffusive_fraction=0.3)
    A = sp.csr_matrix((net.data, net.indices, net.indptr), shape=(net.n, net.n))
    assert (A - A.T).nnz == 0 or abs(A - A.T).max() == 0.0
    assert net.indptr.dtype == np.int32 and net.indices.dtype == np.int32
    # sorted columns, diagonal present, off-diagonals negative
    for i in range(0, net.n, 97):
        cols = net.indices[net.indptr[i]:net.indptr[i + 1]]
        assert np.all(np.diff(cols) > 0) and i in cols
    off = A - sp.diags(A.diagonal())
    assert off.max() <= 0.0
    # row sums vanish except where a Dirichlet node was eliminated
    rs = np.asarray(A.sum(axis=1)).ravel()
    assert np.count_nonzero(np.abs(rs) > 1e-12 * A.diagonal()) == np.count_nonzero(net.rhs)
    # exact solution lies between the boundary pressures (maximum principle)
    x = sp.linalg.spsolve(A.tocsc(), net.rhs)
    assert x.min() >= P_OUTLET * (1 - 1e-9) and x.max() <= P_INLET * (1 + 1e-9)


def test_conductance_range_and_seed():
    a = vascular_network(depth=8, n_nodes=3000, seed=5)
    b = vascular_network(depth=8, n_nodes=3000, seed=5)
    assert np.array_equal(a.data, b.data) and np.array_equal(a.rhs, b.rhs)
    g = a.conductance
    assert g.max() / g.min() > 1e8        # many decades of conductance
    assert a.radius.min() >= 3e-6 * 0.99 and a.radius.max() <= 1.1e-3


def test_named_config_sizes():
    net = make_config("vascular_20k")
    assert 19_000 <= net.n <= 22_000
    assert net.nnz < 8 * net.n


def test_batch_networks_sizes_and_determinism():
    from blood_network_b200.network import batch_networks
    a = batch_networks(6, lo=2000, hi=20000, seed=4)
    b = batch_networks(6, lo=2000, hi=20000, seed=4)
    for x, y in zip(a, b):
        assert x.n == y.n and x.data.tobytes() == y.data.tobytes()
    # node counts within the range (interior = total minus the two Dirichlet roots)
    assert all(1000 <= x.n <= 25000 for x in a)


def test_adjoint_conductance_matches_generator():
    import torch
    from blood_network_b200.adjoint import conductance
    from blood_network_b200.network import vascular_network
    net = vascular_network(depth=6, n_nodes=800, seed=2, diffusive_fraction=0.3)
    g = conductance(torch.as_tensor(np.log(net.radius)), torch.as_tensor(net.length),
                    torch.as_tensor(net.diffusive.astype(np.float64))).numpy()
    assert np.allclose(g, net.conductance, rtol=1e-12, atol=0)
