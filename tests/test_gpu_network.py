"""Vessel networks on the device: assembly of the Dirichlet-reduced system
(read_nwk.m:17-36) against the host assembly, flows, and the adjoint gradient
of a flow-matching loss with respect to log-radius against an FP64 reference
gradient (direct solves) and against central finite differences."""
import math

import numpy as np
import pytest

from blood_network_b200.network import MU_BLOOD, D_DIFFUSION, make_config, vascular_network

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _system(net):
    from blood_network_b200 import adjoint
    dnet = adjoint.DeviceNetwork.from_network(net)
    g = torch.as_tensor(net.conductance, dtype=torch.float64, device="cuda")
    return adjoint.System(g, dnet), dnet, g


def _dev(ptr, n, typestr="<f8"):
    from blood_network_b200.adjoint import _DevicePtr
    return torch.as_tensor(_DevicePtr(ptr, n, typestr), device="cuda").cpu().numpy()


def test_assembly_matches_host():
    net = make_config("vascular_20k")
    S, dnet, g = _system(net)
    try:
        sys = S.sys
        assert sys.n == net.n and sys.nnz == net.nnz
        assert np.array_equal(_dev(sys.ia, net.n + 1, "<i4"), net.indptr)
        assert np.array_equal(_dev(sys.ja, net.nnz, "<i4"), net.indices)
        assert _dev(sys.val, net.nnz).tobytes() == net.data.tobytes()
        assert _dev(sys.rhs, net.n).tobytes() == net.rhs.tobytes()
        assert np.array_equal(S.interior_of().cpu().numpy(), net.interior_of)
    finally:
        S.close()


def test_flows():
    net = make_config("vascular_20k")
    S, dnet, g = _system(net)
    try:
        p = S.solve(S.rhs())
        q = S.flows(g, p).cpu().numpy()
        P = np.zeros(net.n_total)
        io = net.interior_of
        P[io >= 0] = p.cpu().numpy()[io[io >= 0]]
        P[net.boundary] = net.p_boundary
        want = net.conductance * (P[net.seg_u] - P[net.seg_v])
        assert q.tobytes() == want.tobytes()
    finally:
        S.close()


def _conductance(logr, length, diff):
    r = torch.exp(logr)
    g = math.pi * r ** 4 / (8.0 * MU_BLOOD * length)
    return g + diff * (D_DIFFUSION * math.pi * r ** 2 / length)


def _loss(logr, net, dnet, length, diff, obs, qhat, io):
    from blood_network_b200 import adjoint
    g = _conductance(logr, length, diff)
    p = adjoint.network_pressure(g, dnet, tol=1e-13)
    P = adjoint.full_pressure(p, dnet, io)
    q = g * (P[dnet.u.long()] - P[dnet.v.long()])
    return ((q[obs] - qhat) ** 2).sum()


def test_adjoint_gradient_against_reference_and_fd():
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    from blood_network_b200.network import assemble
    net = vascular_network(depth=8, n_nodes=3000, seed=11, diffusive_fraction=0.3)
    dnet_np = net
    rng = np.random.default_rng(3)
    logr0 = np.log(net.radius)
    length = torch.as_tensor(net.length, device="cuda")
    diff = torch.as_tensor(net.diffusive.astype(np.float64), device="cuda")
    from blood_network_b200 import adjoint
    dnet = adjoint.DeviceNetwork.from_network(net)
    io = torch.as_tensor(net.interior_of, device="cuda")
    m = net.n_segments
    obs = torch.as_tensor(np.sort(rng.choice(m, max(50, m // 20), replace=False)), device="cuda")
    # targets: flows at radii perturbed by log-normal noise (sigma 0.1)
    with torch.no_grad():
        lr_t = torch.as_tensor(logr0 + rng.normal(0.0, 0.1, m), device="cuda")
        g_t = _conductance(lr_t, length, diff)
        p_t = adjoint.network_pressure(g_t, dnet, tol=1e-13)
        P_t = adjoint.full_pressure(p_t, dnet, io)
        qhat = (g_t * (P_t[dnet.u.long()] - P_t[dnet.v.long()]))[obs]
    logr = torch.as_tensor(logr0, device="cuda").requires_grad_(True)
    L = _loss(logr, net, dnet, length, diff, obs, qhat, io)
    L.backward()
    grad = logr.grad.cpu().numpy()

    # FP64 reference: direct solves on the host assembly
    gpois = math.pi * net.radius ** 4 / (8.0 * MU_BLOOD * net.length)
    gdiff = np.where(net.diffusive, D_DIFFUSION * math.pi * net.radius ** 2 / net.length, 0.0)
    gn = gpois + gdiff
    sysn = assemble(net.n_total, net.seg_u, net.seg_v, gn, net.boundary, net.p_boundary)
    A = sp.csr_matrix((sysn.data, sysn.indices, sysn.indptr), shape=(sysn.n, sysn.n)).tocsc()
    lu = spla.splu(A)
    p = lu.solve(sysn.rhs)
    P = np.zeros(net.n_total)
    P[net.interior_of >= 0] = p[net.interior_of[net.interior_of >= 0]]
    P[net.boundary] = net.p_boundary
    dP = P[net.seg_u] - P[net.seg_v]
    q = gn * dP
    o = obs.cpu().numpy()
    dLdq = np.zeros(m)
    dLdq[o] = 2.0 * (q[o] - qhat.cpu().numpy())
    dLdP = np.zeros(net.n_total)
    np.add.at(dLdP, net.seg_u, dLdq * gn)
    np.add.at(dLdP, net.seg_v, -dLdq * gn)
    lam = lu.solve(dLdP[net.interior_of >= 0][np.argsort(net.interior_of[net.interior_of >= 0])])
    Lam = np.zeros(net.n_total)
    Lam[net.interior_of >= 0] = lam[net.interior_of[net.interior_of >= 0]]
    dLdg = dLdq * dP - (Lam[net.seg_u] - Lam[net.seg_v]) * dP
    ref = dLdg * (4.0 * gpois + 2.0 * gdiff)
    err = np.linalg.norm(grad - ref) / np.linalg.norm(ref)
    assert err < 1e-6, err

    # central finite differences on 50 random segments
    h = 1e-6
    pick = rng.choice(m, 50, replace=False)
    fd = []
    with torch.no_grad():
        for k in pick:
            e = torch.zeros(m, dtype=torch.float64, device="cuda")
            e[k] = h
            lp = _loss(logr.detach() + e, net, dnet, length, diff, obs, qhat, io).item()
            lm = _loss(logr.detach() - e, net, dnet, length, diff, obs, qhat, io).item()
            fd.append((lp - lm) / (2 * h))
    fd = np.array(fd)
    scale = np.abs(ref).max()
    assert np.all(np.abs(fd - grad[pick]) <= 1e-4 * scale + 1e-3 * np.abs(grad[pick])), \
        np.max(np.abs(fd - grad[pick])) / scale
