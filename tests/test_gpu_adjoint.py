"""Gradient of the elliptic solve (semtex_b200.autograd.helmholtz_solve)
against central finite differences (h = 1e-6, agreement to 1e-6 relative)
and the exact adjoint identity w^T (A(f + e) - A(f)) = (A^T w)^T e, with
inhomogeneous Dirichlet and mixed (Robin) boundaries, in 2D and 3D."""
import numpy as np
import pytest

import semtex_b200 as S
from semtex_b200 import sessions
from semtex_b200.autograd import helmholtz_solve, solve_physical

pytestmark = pytest.mark.gpu


def _session(tmp_path, nz):
    p = sessions.rect_session(str(tmp_path / f"adj{nz}"), 4, 3,
                              tokens={"N_P": 6, "N_Z": nz, "BETA": 1.0, "LAMBDA2": 2.0, "TOL_REL": 1e-14},
                              periodic_x=True, bcs={"w": {"c": "<M> 1.5;0.2"}})
    txt = open(p).read()
    txt = txt.replace("<GROUPS NUMBER=1>", "<GROUPS NUMBER=2>\n\t2\tz\tclamp")
    bc = "0.3+0.1*cos(z)" if nz > 1 else "0.3"
    txt = txt.replace("<BCS NUMBER=1>", f"<BCS NUMBER=2>\n\t2\tz\t1\n\t\t<D>\tc = {bc}\t</D>")
    out = []
    for ln in txt.splitlines():
        parts = ln.split("\t")
        if len(parts) >= 4 and parts[3] == "1" and "<B>" in ln:
            ln = ln.replace("<B>\tw\t</B>", "<B>\tz\t</B>")
        out.append(ln)
    open(p, "w").write("\n".join(out) + "\n")
    return p


@pytest.mark.parametrize("nz", [1, 8])
def test_solve_gradient(tmp_path, nz):
    import torch
    p = _session(tmp_path, nz)
    ctx = S.Context(p)
    sysm = S.ModalMatrixSys(ctx, "c", 2.0)
    dev = "cuda:0"
    rng = np.random.default_rng(nz)
    shape = (ctx.nz, ctx.nel, ctx.np, ctx.np)
    f0 = torch.tensor(rng.uniform(-1, 1, shape), device=dev)
    w = torch.tensor(rng.uniform(-1, 1, shape), device=dev)
    f = f0.clone().requires_grad_(True)
    u = helmholtz_solve(f, sysm)
    (w * u).sum().backward()
    grad = f.grad.detach()
    L = lambda x: float((w * solve_physical(sysm, x)).sum())
    for k in range(3):
        e = torch.tensor(rng.uniform(-1, 1, shape), device=dev)
        ge = float((grad * e).sum())
        lin = float((w * (solve_physical(sysm, f0 + e) - solve_physical(sysm, f0))).sum())
        assert abs(lin - ge) <= 1e-11 * abs(ge), (lin, ge)
        h = 1e-6
        fd = (L(f0 + h * e) - L(f0 - h * e)) / (2 * h)
        assert abs(fd - ge) <= 1e-6 * abs(ge), (fd, ge)
    sysm.close()
    ctx.close()
