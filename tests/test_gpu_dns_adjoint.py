"""Discrete adjoint and tangent-linear model of the DNS time step
(stx_dns_adjoint_*, semtex_b200.DNSAdjoint, autograd.dns_steps).

- The dot-product identity <T x, y> = <x, A y> between the tangent-linear
  model T and the adjoint A, over runs that cross the start-up orders and
  several checkpoint segments: every nonlinear form, periodic Taylor-Green
  and the channel with high-order pressure walls, 2D and 3D, N_TIME 1..3.
  Both sides are built independently (T runs the forward kernels on the
  perturbation, A the transposed kernels), so the identity checks every
  transposed sub-step to round-off.
- T against central differences of the forward DNS (h = 1e-6).
- The channel workload: 16x8 quads, N_P = 9, N_Z = 32, Re = 500,
  D_T = 5e-3, 100 steps, checkpoints every 10; objective the perturbation
  kinetic energy at the end; the gradient w.r.t. the initial velocity
  against central differences (h = 1e-6, 1e-6 relative) and against the
  tangent-linear directional derivative.
- The gradient does not depend on the checkpoint interval; the
  torch.autograd path gives the same gradient; options that are not
  differentiated are rejected.
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

import semtex_b200 as S
from semtex_b200 import _lib, sessions
from semtex_b200.autograd import dns_steps

from conftest import GOLDEN

sys.path.insert(0, GOLDEN)
import make_baseline_fixtures as FX  # noqa: E402

pytestmark = pytest.mark.gpu


def _q4(ctx):
    q = np.empty(ctx.nel * ctx.np * ctx.np)
    _lib.check(_lib.lib().stx_mesh_mass(ctx.handle, C.c_void_p(q.ctypes.data)))
    return q.reshape(1, ctx.nel, ctx.np, ctx.np)


def _tg(tmp_path, name, nz=8, extra=None):
    p = sessions.taylor_green_session(str(tmp_path / name), 3, 6, nz, re=100.0, dt=2e-3, extra=extra)
    ctx = S.Context(p)
    x, y = ctx.mesh_coords()
    z = (np.arange(ctx.nz) * 2 * np.pi / ctx.nz)[:, None, None, None]
    ic = {"u": np.sin(x) * np.cos(y) * np.cos(z), "v": -np.cos(x) * np.sin(y) * np.cos(z),
          "w": 0.3 * np.sin(x) * np.sin(y) * np.sin(z) + 0 * x}
    return ctx, {c: np.broadcast_to(v, (ctx.nz, ctx.nel, ctx.np, ctx.np)).copy() for c, v in ic.items()}


def _channel(tmp_path, name, nz=8, ntime=3, amplitude=0.05, re=200.0, dt=5e-3, extra=None):
    p = sessions.channel_session(str(tmp_path / name), 4, 2, 6, nz, re=re, dt=dt, ntime=ntime, extra=extra)
    ctx = S.Context(p)
    x, y = ctx.mesh_coords()
    ic = sessions.channel_initial(x, y, np.arange(ctx.nz) * 2 * np.pi / ctx.nz, amplitude=amplitude)
    return ctx, {c: ic[c] for c in ctx.fields[:-1]}


CASES = {
    # name: (builder, kwargs, advection)
    "tg_skew": (_tg, {}, 0),
    "tg_alternating": (_tg, {}, 1),
    "tg_convective": (_tg, {}, 2),
    "tg_stokes": (_tg, {}, 3),
    "channel_alternating": (_channel, {}, 1),
    "channel_skew": (_channel, {}, 0),
    "channel_order1": (_channel, {"ntime": 1}, 1),
    "channel_order2": (_channel, {"ntime": 2}, 2),
    "channel_2d": (_channel, {"nz": 1}, 1),
    "channel_nz2": (_channel, {"nz": 2}, 1),
    # Jacobi-PCG velocity solves forward; the derivatives solve exactly
    "channel_iterative": (_channel, {"extra": {"ITERATIVE": 1}}, 1),
}


def _inner(a, b):
    return sum(float(np.vdot(a[c], b[c])) for c in a)


@pytest.mark.parametrize("name", sorted(CASES))
def test_tangent_adjoint_dot_product(tmp_path, name):
    build, kw, adv = CASES[name]
    ctx, ic = build(tmp_path, name, **kw)
    D = S.DNS(ctx, adv)
    D.restart(ic, 0.0)
    A = S.DNSAdjoint(D, checkpoint_every=4)
    A.record(11)  # start-up orders, then three segments (4, 4, 3)
    assert A.info()[:2] == (0, 11)
    shape = (ctx.nz, ctx.nel, ctx.np, ctx.np)
    rng = np.random.default_rng(11)
    x = {c: rng.standard_normal(shape) for c in A.components}
    y = {c: rng.standard_normal(shape) for c in A.components}
    tx = A.tangent(x)
    ay = A.backward(y)
    lhs, rhs = _inner(tx, y), _inner(x, ay)
    assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), abs(rhs)), (lhs, rhs)
    assert D.state()[0] == 11  # left at the end of the record
    A.close()
    D.close()


def _run(ctx, ic, steps, adv=1):
    D = S.DNS(ctx, adv)
    D.restart(ic, 0.0)
    D.advance(steps)
    out = {c: D.field(c) for c in ic}
    D.close()
    return out


@pytest.mark.parametrize("name", ["tg_alternating", "channel_alternating"])
def test_tangent_matches_central_differences(tmp_path, name):
    build, kw, adv = CASES[name]
    ctx, ic = build(tmp_path, name, **kw)
    steps, h = 12, 1e-6
    rng = np.random.default_rng(5)
    shape = (ctx.nz, ctx.nel, ctx.np, ctx.np)
    d = {c: rng.uniform(-1, 1, shape) for c in ic}
    D = S.DNS(ctx, adv)
    D.restart(ic, 0.0)
    A = S.DNSAdjoint(D, checkpoint_every=5)
    A.record(steps)
    t = A.tangent(d)
    A.close()
    D.close()
    up = _run(ctx, {c: ic[c] + h * d[c] for c in ic}, steps, adv)
    um = _run(ctx, {c: ic[c] - h * d[c] for c in ic}, steps, adv)
    fd = {c: (up[c] - um[c]) / (2 * h) for c in ic}
    num = np.sqrt(sum(np.sum((fd[c] - t[c]) ** 2) for c in ic))
    den = np.sqrt(sum(np.sum(t[c] ** 2) for c in ic))
    assert num <= 1e-6 * den, num / den


def _perturbation_energy(q4, u, base):
    """0.5 * sum over planes of the Q4-weighted |u - base|^2 (perturbation
    kinetic energy up to the constant plane spacing) and its gradient."""
    e = 0.0
    g = {}
    for c, v in u.items():
        w = v - base[c]
        e += 0.5 * float(np.sum(q4 * w * w))
        g[c] = q4 * w
    return e, g


def _c5(tmp_path):
    p = FX.c5_session(str(tmp_path))
    ctx = S.Context(p)
    x, y = ctx.mesh_coords()
    ic = FX.c5_initial(x, y, ctx.nz)
    vel = {c: ic[c] for c in "uvw"}
    shape = (ctx.nz, ctx.nel, ctx.np, ctx.np)
    base = {"u": np.broadcast_to(1 - y * y, shape), "v": np.zeros(shape), "w": np.zeros(shape)}
    # a second divergence-free perturbation of the same family as the
    # direction, scaled to unit amplitude (max |d| = 1), so that the central
    # difference step h = 1e-6 perturbs the initial velocity by 1e-6
    alt = sessions.channel_initial(x, y, np.arange(ctx.nz) * 2 * np.pi / ctx.nz, seed=7)
    direction = {c: alt[c] - base[c] for c in "uvw"}
    amp = max(float(np.abs(v).max()) for v in direction.values())
    direction = {c: v / amp for c, v in direction.items()}
    return ctx, vel, base, direction


def test_c5_gradient_matches_central_differences_and_tangent(tmp_path):
    ctx, u0, base, dirn = _c5(tmp_path)
    q4 = _q4(ctx)
    steps, every = 100, 10
    D = S.DNS(ctx, 1)
    D.restart(u0, 0.0)
    A = S.DNSAdjoint(D, checkpoint_every=every)
    A.record(steps)
    uT = {c: D.field(c) for c in "uvw"}
    E, dE = _perturbation_energy(q4, uT, base)
    grad = A.backward(dE)
    dot = _inner(grad, dirn)
    # tangent-linear directional derivative: <dE/du_T, T d>
    tl = _inner(dE, A.tangent(dirn))
    assert abs(dot - tl) <= 1e-10 * abs(tl), (dot, tl)
    _, _, ck = A.info()
    assert ck > 0
    A.close()
    D.close()
    # central differences of the nonlinear forward run, h = 1e-6
    h = 1e-6
    Ep, _ = _perturbation_energy(q4, _run(ctx, {c: u0[c] + h * dirn[c] for c in u0}, steps), base)
    Em, _ = _perturbation_energy(q4, _run(ctx, {c: u0[c] - h * dirn[c] for c in u0}, steps), base)
    fd = (Ep - Em) / (2 * h)
    assert abs(fd - dot) <= 1e-6 * abs(fd), (fd, dot)


def test_gradient_independent_of_checkpoint_interval(tmp_path):
    ctx, ic = _channel(tmp_path, "ck")
    rng = np.random.default_rng(2)
    shape = (ctx.nz, ctx.nel, ctx.np, ctx.np)
    seed = {c: rng.standard_normal(shape) for c in ic}
    grads = []
    for every in (1, 7, 30):
        D = S.DNS(ctx, 1)
        D.restart(ic, 0.0)
        A = S.DNSAdjoint(D, checkpoint_every=every)
        A.record(23)
        grads.append(A.backward(seed))
        A.close()
        D.close()
    scale = np.sqrt(sum(np.sum(grads[0][c] ** 2) for c in ic))
    for g in grads[1:]:
        err = np.sqrt(sum(np.sum((g[c] - grads[0][c]) ** 2) for c in ic))
        assert err <= 1e-12 * scale


def test_torch_autograd_dns_steps(tmp_path):
    import torch
    ctx, ic = _channel(tmp_path, "ta")
    q4 = torch.from_numpy(_q4(ctx)).cuda()
    D = S.DNS(ctx, 1)
    A = S.DNSAdjoint(D, checkpoint_every=6)
    u0 = torch.from_numpy(np.stack([ic[c] for c in A.components])).cuda().requires_grad_(True)
    uT = dns_steps(u0, A, 15)
    loss = 0.5 * (q4 * uT ** 2).sum()
    loss.backward()
    g = A.backward({c: (q4 * uT[i]).detach().cpu().numpy() for i, c in enumerate(A.components)})
    want = np.stack([g[c] for c in A.components])
    got = u0.grad.cpu().numpy()
    assert np.linalg.norm(got - want) <= 1e-12 * np.linalg.norm(want)
    A.close()
    D.close()


def test_options_not_differentiated_are_rejected(tmp_path):
    p = sessions.taylor_green_session(str(tmp_path / "dl"), 3, 6, 8, extra={"DEALIAS": 1})
    ctx = S.Context(p)
    D = S.DNS(ctx, 1)
    with pytest.raises(_lib.StxError, match="DEALIAS"):
        S.DNSAdjoint(D)
    with pytest.raises(_lib.StxError, match="no recorded run"):
        D2 = S.DNS(S.Context(sessions.taylor_green_session(str(tmp_path / "nr"), 3, 6, 8)), 1)
        A = S.DNSAdjoint(D2)
        A.backward({c: np.zeros((8, 9, 6, 6)) for c in "uvw"})
