"""Pressure of a vessel network as a differentiable function of its segment
conductances, for checking the adjoint entry points.

``NetworkPressure.apply(g, net)`` assembles the Dirichlet-reduced system on the
device (``amg_network_assemble_device``), solves it with the AMG-PCG solver and
returns the interior pressures; its backward pass is one adjoint solve on the
same hierarchy (``amg_network_adjoint_device``: A is symmetric), giving
dL/dg_e = -(lambda_u - lambda_v)(P_u - P_v).  Everything stays on the GPU; torch
carries the chain rule around it (conductance from radius, flows, loss).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import amg


@dataclass
class DeviceNetwork:
    """Segments and Dirichlet data of a network as CUDA tensors."""
    n_nodes: int
    u: "torch.Tensor"      # int32 [n_seg]
    v: "torch.Tensor"      # int32 [n_seg]
    bnd: "torch.Tensor"    # int32 [n_bnd]
    p_bnd: "torch.Tensor"  # float64 [n_bnd]

    @classmethod
    def from_network(cls, net, device="cuda"):
        import torch
        t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=device)
        return cls(int(net.n_total), t(net.seg_u, torch.int32), t(net.seg_v, torch.int32),
                   t(net.boundary, torch.int32), t(net.p_boundary, torch.float64))


class System:
    """A device-assembled pressure system and the solver built on it."""

    def __init__(self, g, net: DeviceNetwork, threshold=0.25, coarsening=amg.COARSEN_PMIS,
                 tol=1e-12, maxiter=500):
        import torch
        self.lib = amg.load_library()
        self.net = net
        self.tol, self.maxiter = tol, maxiter
        self.sys = amg.NetworkSystem()
        g = g.contiguous()
        rc = self.lib.amg_network_assemble_device(
            net.n_nodes, int(net.u.numel()), net.u.data_ptr(), net.v.data_ptr(), g.data_ptr(),
            int(net.bnd.numel()), net.bnd.data_ptr(), net.p_bnd.data_ptr(), C.byref(self.sys))
        if rc != 0:
            raise amg.AMGError(rc, self.lib.amg_solver_last_error().decode())
        o = amg.default_options(threshold=threshold, coarsening=coarsening,
                                stop=amg.STOP_RELRES)
        torch.cuda.synchronize()
        self.h = self.lib.amg_solver_create_device(self.sys.n, self.sys.nnz, self.sys.ia,
                                                   self.sys.ja, self.sys.val, C.byref(o))
        if not self.h:
            raise amg.AMGError(self.lib.amg_solver_last_status(),
                               self.lib.amg_solver_last_error().decode())
        self.n = self.sys.n

    def rhs(self):
        """f on the device (a copy of the library's array)."""
        import torch
        return torch.as_tensor(_DevicePtr(self.sys.rhs, self.n), device=self.net.u.device).clone()

    def interior_of(self):
        """node -> interior unknown (-1 at Dirichlet nodes), int32 on the device (a copy)."""
        import torch
        return torch.as_tensor(_DevicePtr(self.sys.interior_of, self.net.n_nodes, "<i4"),
                               device=self.net.u.device).clone()

    def solve(self, b):
        import torch
        x = torch.zeros_like(b)
        torch.cuda.synchronize()
        it = self.lib.amg_solver_solve_device(self.h, C.c_void_p(b.data_ptr()),
                                              C.c_void_p(x.data_ptr()), self.tol, self.maxiter, 0)
        if it <= 0:
            raise amg.AMGError(self.lib.amg_solver_last_status(), "solve did not converge")
        return x

    def adjoint(self, p, dLdp):
        import torch
        lam = torch.empty_like(p)
        dLdg = torch.empty(self.net.u.numel(), dtype=torch.float64, device=p.device)
        it = C.c_int()
        torch.cuda.synchronize()
        rc = self.lib.amg_network_adjoint_device(
            self.h, C.byref(self.sys), int(self.net.u.numel()), self.net.u.data_ptr(),
            self.net.v.data_ptr(), p.contiguous().data_ptr(), dLdp.contiguous().data_ptr(),
            self.tol, self.maxiter, lam.data_ptr(), dLdg.data_ptr(), C.byref(it))
        if rc != 0 or it.value <= 0:
            raise amg.AMGError(rc, self.lib.amg_solver_last_error().decode())
        return dLdg, lam

    def flows(self, g, p):
        import torch
        q = torch.empty_like(g)
        torch.cuda.synchronize()
        rc = self.lib.amg_network_flows_device(C.byref(self.sys), int(self.net.u.numel()),
                                               self.net.u.data_ptr(), self.net.v.data_ptr(),
                                               g.contiguous().data_ptr(),
                                               p.contiguous().data_ptr(), q.data_ptr())
        if rc != 0:
            raise amg.AMGError(rc, self.lib.amg_solver_last_error().decode())
        return q

    def close(self):
        if getattr(self, "h", None):
            self.lib.amg_solver_free(self.h)
            self.h = None
        if getattr(self, "sys", None) is not None and self.sys.owner:
            self.lib.amg_network_system_free(C.byref(self.sys))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _DevicePtr:
    """__cuda_array_interface__ over a device array the library owns."""

    def __init__(self, ptr, n, typestr="<f8"):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr,
                                         "data": (ptr, False), "version": 3, "strides": None}


def _network_pressure():
    import torch

    class NetworkPressure(torch.autograd.Function):
        @staticmethod
        def forward(ctx, g, net: DeviceNetwork, tol=1e-12):
            S = System(g.detach(), net, tol=tol)
            f = torch.as_tensor(_DevicePtr(S.sys.rhs, S.n), device=g.device).clone()
            p = S.solve(f)
            ctx.S = S
            ctx.save_for_backward(p)
            return p

        @staticmethod
        def backward(ctx, dLdp):
            (p,) = ctx.saved_tensors
            dLdg, _ = ctx.S.adjoint(p, dLdp.contiguous())
            ctx.S.close()
            return dLdg, None, None

    return NetworkPressure


def network_pressure(g, net: DeviceNetwork, tol=1e-12):
    """Interior pressures p(g) (CUDA float64), differentiable in g."""
    return _network_pressure().apply(g, net, tol)


def full_pressure(p, net: DeviceNetwork, interior_of):
    """Pressures of all nodes: p at interior nodes, p_B at Dirichlet nodes."""
    import torch
    P = torch.zeros(net.n_nodes, dtype=torch.float64, device=p.device)
    io = interior_of
    mask = io >= 0
    P[mask] = p[io[mask]]
    P[net.bnd.long()] = net.p_bnd
    return P


def conductance(logr, length, diffusive):
    """Segment conductances from log-radius (torch, differentiable): the
    Poiseuille term pi r^4 / (8 mu L) plus, on diffusive segments (mask 1.0),
    D pi r^2 / L."""
    import math
    import torch
    from .network import D_DIFFUSION, MU_BLOOD
    r = torch.exp(logr)
    g = math.pi * r ** 4 / (8.0 * MU_BLOOD * length)
    return g + diffusive * (D_DIFFUSION * math.pi * r ** 2 / length)


def flow_misfit(logr, dnet: DeviceNetwork, length, diffusive, obs, qhat, interior_of,
                tol=1e-12):
    """L = sum over observed segments of (q_e - qhat_e)^2 with q = g (P_u - P_v)."""
    g = conductance(logr, length, diffusive)
    p = network_pressure(g, dnet, tol=tol)
    P = full_pressure(p, dnet, interior_of)
    q = g * (P[dnet.u.long()] - P[dnet.v.long()])
    return ((q[obs] - qhat) ** 2).sum()
