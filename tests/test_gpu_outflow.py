"""Computed outflow BCs <O> on the device against the oracle's restatement
(src/bcmgr.cpp:998-1633): a channel with a parabolic inflow, no-slip walls and
an outflow exit, in 2D and 3D, with a sharp switch (Poiseuille flow kept to
round-off) and a smooth one (the kinetic-energy term acting), started from a
perturbed state so that every term (gradients, div u, the z-derivative of w,
the extrapolated edge velocities) carries data.  Bar: relative L2 <= 1e-10
(pressure 1e-9 of its scale), as the other DNS parity tests."""
import numpy as np
import pytest

import semtex_oracle as O
import semtex_b200 as S
from semtex_b200 import sessions

pytestmark = pytest.mark.gpu


def _channel(path, nz, u0, perturb):
    fields = "uvwp" if nz > 1 else "uvp"
    bcs = {"v": {"u": "<D> 1-y*y", "v": "<D> 0", "p": "<H> 0"},
           "w": {"u": "<D> 0", "v": "<D> 0", "p": "<H> 0"},
           "o": {"u": "<O> 0", "v": "<O> 0", "p": "<O> 0"}}
    if nz > 1:
        for g in bcs:
            bcs[g]["w"] = "<O> 0" if g == "o" else "<D> 0"
    if perturb:
        user = ["u = 1-y*y+0.05*sin(PI*x/2)*(1-y*y)*cos(z)", "v = 0.03*(1-y*y)*sin(PI*x/4)*sin(z)",
                "p = 0.2*(4-x)"] + (["w = 0.02*(1-y*y)*x*(4-x)*cos(2*z)"] if nz > 1 else [])
        if nz == 1:
            user = [u.replace("*cos(z)", "").replace("*sin(z)", "") for u in user]
    else:
        user = ["u = 1-y*y", "v = 0", "p = 0.2*(4-x)"] + (["w = 0"] if nz > 1 else [])
    return sessions.rect_session(path, 4, 2, x=(0.0, 4.0), y=(-1.0, 1.0),
                                 tokens={"N_P": 6, "N_Z": nz, "N_TIME": 2, "D_T": 0.01, "KINVIS": 0.1,
                                         "N_STEP": 12, "TOL_REL": 1e-14, "U0Delta": u0},
                                 fields=fields, bcs=bcs, side_groups={"left": "v", "right": "o"},
                                 group_names={"o": "outflow"}, user=user)


def _compare(gpu, D, tol=1e-10, ptol=1e-9):
    phys = D.physical()
    scale = max(np.linalg.norm(phys[c]) for c in D.vel)
    for c in D.vel:
        err = np.linalg.norm(gpu[c] - phys[c]) / scale
        assert err < tol, (c, err)
    pc = D.pname
    pscale = max(np.linalg.norm(phys[pc]), np.linalg.norm(sum(phys[c] ** 2 for c in D.vel)))
    assert np.linalg.norm(gpu[pc] - phys[pc]) / pscale < ptol


@pytest.mark.parametrize("nz", [1, 4])
@pytest.mark.parametrize("u0,perturb", [(1e-8, False), (0.05, True)])
def test_outflow_gpu_matches_oracle(tmp_path, nz, u0, perturb):
    p = _channel(str(tmp_path / "ch"), nz, u0, perturb)
    gpu, _ = S.dns(p)
    D = O.dns_session(p)
    assert len(D.oedges) == 2
    _compare(gpu, D)
    if not perturb:   # Poiseuille flow through the exit, kept to round-off
        y = D.P.M.y[None]
        assert np.abs(gpu["u"] - (1 - y * y)).max() < 1e-11


def test_outflow_ntime3_graph_and_checkpoint(tmp_path):
    # third-order steps, enough of them for the steady-step graph replay; the
    # outflow levels also travel in a checkpoint
    p = _channel(str(tmp_path / "ch3"), 4, 0.05, True)
    txt = open(p).read().replace("N_TIME = 2", "N_TIME = 3").replace("N_STEP = 12", "N_STEP = 110")
    open(p, "w").write(txt)
    ctx = S.Context(p)
    funcs = S._user_functions(p)
    ic = {c: ctx.evaluate(funcs[c], 0.0) for c in ctx.fields if c in funcs}
    A = S.DNS(ctx, 1)
    A.restart(ic, 0.0)
    A.advance(20)
    buf = A.checkpoint()
    A.advance(90)   # the steady cycle (42 steps with pressure-BC and outflow levels) is captured
    gpu = {c: A.field(c) for c in ctx.fields}
    assert A.graph_info()[1] > 0   # steady steps were replayed as a graph
    A.close()
    D = O.dns_session(p)
    _compare(gpu, D)
    B = S.DNS(ctx, 1)
    B.restart(ic, 0.0)
    B.restore(buf)
    B.advance(90)
    cont = {c: B.field(c) for c in ctx.fields}
    scale = max(np.linalg.norm(gpu[c]) for c in "uvw")
    for c in "uvw":
        assert np.linalg.norm(cont[c] - gpu[c]) <= 1e-12 * scale, c
    assert np.linalg.norm(cont["p"] - gpu["p"]) <= 1e-10 * np.linalg.norm(gpu["p"])
    B.close()
