"""Differentiable Field::solve (the elliptic map forcing -> solution) and
DNS time steps (the discrete adjoint over the C ABI), as
torch.autograd.Functions.

Field::solve.  The map (src/field.cpp:598-809 with the z transforms of elliptic/helmholtz.cpp:
29-52) is affine, u = A f + b: b comes from the boundary conditions and
A = I S F, with F / I the packed real DFT pair and S, per plane, the
condensed Helmholtz solve S = -P H^-1 P^T M (P: global -> element-local
copy, H the symmetric assembled Helmholtz matrix of the plane's mode, M the
element-local mass Q4).  The packed DFT pair satisfies F^T = I W^-1 / N and
I^T = N W F with W = diag(1, 1, 2, 2, ...), a per-plane weight that commutes
with the per-plane S^T = -M P H^-1 P^T, and M commutes with the z transforms,
so
        A^T g = M (A (M^-1 g) - b)  =  Q4 * (solve(g / Q4) - solve(0)):
the gradient reuses the forward solve, its condensed factors included.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import FORWARD, INVERSE, _torch
from ._lib import check, lib


class _Work:
    """Device buffers and constants of one system, kept on the system."""

    def __init__(self, system):
        torch = _torch()
        ctx = system.ctx
        self.F = ctx.new_field("adj_f")
        self.U = ctx.new_field("adj_u")
        q4 = np.empty(ctx.nel * ctx.np * ctx.np)
        check(lib().stx_mesh_mass(ctx.handle, C.c_void_p(q4.ctypes.data)))
        self.q4 = torch.from_numpy(q4.reshape(1, ctx.nel, ctx.np, ctx.np)).to(self.F.data.device)
        self.offset = None


def _work(system):
    w = getattr(system, "_adjoint_work", None)
    if w is None:
        w = _Work(system)
        system._adjoint_work = w
    return w


def solve_physical(system, f):
    """u = Field::solve of the physical forcing f (device tensor [nz, nel, np, np],
    float64) with the system's BCs; returns a new device tensor."""
    torch = _torch()
    ctx = system.ctx
    w = _work(system)
    n = ctx.nel * ctx.np * ctx.np
    shape = (ctx.nz, ctx.nel, ctx.np, ctx.np)
    if tuple(f.shape) != shape:
        raise ValueError(f"forcing shape {tuple(f.shape)} != {shape}")
    w.F.data.zero_()
    w.F.data[:, :n] = f.reshape(ctx.nz, n).to(torch.float64)
    torch.cuda.synchronize(w.F.data.device)
    w.F.transform(FORWARD).zero_nyquist()
    w.U.data.zero_()
    torch.cuda.synchronize(w.U.data.device)
    w.U.solve(w.F, system)
    w.U.transform(INVERSE)
    ctx.sync()
    return w.U.data[:, :n].clone().reshape(shape)


def _helmholtz_solve():
    torch = _torch()

    class HelmholtzSolve(torch.autograd.Function):
        @staticmethod
        def forward(actx, f, system):
            actx.system = system
            return solve_physical(system, f)

        @staticmethod
        def backward(actx, g):
            system = actx.system
            w = _work(system)
            # b = solve(0), the BC part of the affine map, taken afresh each
            # time: stx_field_bc_evaluate may have changed the BC values
            # (time-dependent BCs) since the forward call
            offset = solve_physical(system, torch.zeros_like(g))
            x = solve_physical(system, g / w.q4) - offset
            return w.q4 * x, None

    return HelmholtzSolve


_FN = None


def helmholtz_solve(f, system):
    """Differentiable u = Field::solve(f) for a DIRECT (or MIXED) ModalMatrixSys."""
    global _FN
    if _FN is None:
        _FN = _helmholtz_solve()
    return _FN.apply(f, system)


def _dns_steps():
    torch = _torch()

    class DNSSteps(torch.autograd.Function):
        @staticmethod
        def forward(actx, u0, adjoint, nsteps, t0):
            dns = adjoint.dns
            a = u0.detach().to("cpu", torch.float64).numpy()
            dns.restart({c: a[i] for i, c in enumerate(adjoint.components)}, t0)
            adjoint.record(nsteps)
            out = np.stack([dns.field(c) for c in adjoint.components])
            actx.adjoint = adjoint
            actx.device = u0.device
            return torch.from_numpy(out).to(u0.device)

        @staticmethod
        def backward(actx, g):
            adj = actx.adjoint
            gn = g.detach().to("cpu", torch.float64).numpy()
            r = adj.backward({c: gn[i] for i, c in enumerate(adj.components)})
            grad = torch.from_numpy(np.stack([r[c] for c in adj.components])).to(actx.device)
            return grad, None, None, None

    return DNSSteps


_DNS_FN = None


def dns_steps(u0, adjoint, nsteps: int, t0: float = 0.0):
    """Differentiable final velocity of `nsteps` DNS time steps (integrate(),
    dns/integrate.cpp:138-200) from the initial velocity u0 (tensor
    [ncom, nz, nel, np, np], float64, physical; the DNS restarts from it at
    time t0 with empty history).  `adjoint` is a semtex_b200.DNSAdjoint of
    the DNS: the forward call records the run (checkpoints every
    checkpoint_every steps on the device), backward runs its discrete
    adjoint, whose solves reuse the step's condensed factors."""
    global _DNS_FN
    if _DNS_FN is None:
        _DNS_FN = _dns_steps()
    return _DNS_FN.apply(u0, adjoint, nsteps, t0)
