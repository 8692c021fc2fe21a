"""The two-level systems formed on the device (batched block sweeps, the
default) against the same systems formed on the host (session token
STX_SETUP_HOST = 1): the solutions agree to round-off.  Cases cover several
geometry families (a perturbed mesh), mixed (Robin) BCs, a singular pinned
k=0 system, patch families without interior nodes, and the mixed-precision
(FP32 packed) form.  Both are also checked against the oracle elsewhere."""
import os

import numpy as np
import pytest

import semtex_oracle as O
import semtex_b200 as S
from semtex_b200 import sessions

from conftest import SESSIONS

pytestmark = pytest.mark.gpu


def _solve(path, f, lambda2, host, method=S.DIRECT, field="c", extra=None):
    ov = dict(extra or {})
    if host:
        ov["STX_SETUP_HOST"] = 1
    ctx = S.Context(path, ov or None)
    sysm = S.ModalMatrixSys(ctx, field, lambda2, method=method)
    u = sysm.solve_host(f)
    assert sysm.status() == 0
    sysm.close()
    ctx.close()
    return u


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("n,np_,nz,perturb", [(6, 7, 8, 0.0), (5, 6, 4, 0.3), (12, 5, 2, 0.0), (3, 9, 1, 0.0)])
def test_device_setup_matches_host(tmp_path, n, np_, nz, perturb):
    rng = np.random.default_rng(n * 31 + np_)
    xs = ys = None
    if perturb:
        xs = np.linspace(0, 1, n + 1)
        ys = np.linspace(0, 1, n + 1)
        xs[1:-1] += perturb * rng.uniform(-1, 1, n - 1) / n
        ys[1:-1] += perturb * rng.uniform(-1, 1, n - 1) / n
    p = sessions.helmholtz_session(str(tmp_path / "s"), n, np_, nz=nz, lambda2=1.0, beta=1.0, xs=xs, ys=ys)
    f = rng.uniform(-1, 1, (nz, n * n, np_, np_))
    dev = _solve(p, f, 1.0, host=False)
    host = _solve(p, f, 1.0, host=True)
    assert _rel(dev, host) < 1e-12
    _, U = O.elliptic(p, forcing_phys=f)
    assert _rel(dev, U) < 1e-10


def test_device_setup_mixed_bc():
    path = os.path.join(SESSIONS, "mixed1")
    ctx = S.Context(path)
    shape = (ctx.nz, ctx.nel, ctx.np, ctx.np)
    lam = ctx.token("LAMBDA2")
    field = ctx.fields[0]
    ctx.close()
    f = np.random.default_rng(3).uniform(-1, 1, shape)
    dev = _solve(path, f, lam, host=False, field=field)
    host = _solve(path, f, lam, host=True, field=field)
    assert _rel(dev, host) < 1e-12


def test_device_setup_singular_pressure(tmp_path):
    # periodic Taylor-Green pressure system: k = 0 singular, its pinned node
    # an identity row of the interface matrix
    p = sessions.taylor_green_session(str(tmp_path / "tg"), 4, 6, 8)
    ctx = S.Context(p)
    shape = (ctx.nz, ctx.nel, ctx.np, ctx.np)
    ctx.close()
    f = np.random.default_rng(5).uniform(-1, 1, shape)
    f -= f.mean()
    dev = _solve(p, f, 0.0, host=False, field="p")
    host = _solve(p, f, 0.0, host=True, field="p")
    assert _rel(dev, host) < 1e-11


def test_device_setup_fp32_pack(tmp_path):
    p = sessions.helmholtz_session(str(tmp_path / "m"), 8, 7, nz=8, lambda2=1.0, beta=1.0)
    f = np.random.default_rng(9).uniform(-1, 1, (8, 64, 7, 7))
    dev = _solve(p, f, 1.0, host=False, method=S.MIXED)
    host = _solve(p, f, 1.0, host=True, method=S.MIXED)
    assert _rel(dev, host) < 1e-12
