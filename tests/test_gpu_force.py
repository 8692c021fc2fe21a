"""GPU parity of the DNS body forcing (<FORCE>; FieldForce and its classes,
dns/fieldforce.cpp) against the oracle's restatement, through the C ABI.

Tolerances as the other DNS tests: velocities 1e-10 relative to the largest
component, pressure 1e-9 relative to max(|p|, |u|^2).
"""
import numpy as np
import pytest

import semtex_oracle as O
import semtex_b200 as S
from semtex_b200 import sessions


pytestmark = pytest.mark.gpu


def _compare(gpu, D, tol=1e-10, ptol=1e-9):
    phys = D.physical()
    scale = max(np.linalg.norm(phys[c]) for c in D.vel)
    for c in D.vel:
        err = np.linalg.norm(gpu[c] - phys[c]) / scale
        assert err < tol, (c, err)
    pc = D.pname
    pscale = max(np.linalg.norm(phys[pc]), np.linalg.norm(sum(phys[c] ** 2 for c in D.vel)))
    perr = np.linalg.norm(gpu[pc] - phys[pc]) / pscale
    assert perr < ptol, (pc, perr)


# every physical-space class, time-dependent ones included, and ConstForce
EVERY = ["STEADY_X = 0.1*sin(y)", "MOD_A_Y = cos(x)", "MOD_ALPHA_Y = 0.5+t",
         "SPATIOTEMP_ALPHA_Z = 0.2*sin(x+z-t)", "SPONGE_M = 0.3*heav(x-4)", "SPONGE_U = 0.1",
         "DRAG_M = 0.05", "CORIOLIS_OMEGA_Z = 0.4", "CORIOLIS_OMEGA_X = 0.1", "SFD_DELTA = 0.5",
         "SFD_CHI = 0.2", "CONST_Z = 0.01"]


def _tg(tmp_path, force, nstep=6, extra=None, name="tgf"):
    ex = {"TOL_REL": 1e-14}
    ex.update(extra or {})
    return sessions.taylor_green_session(str(tmp_path / name), 3, 6, 8, re=100.0, dt=2e-3, nstep=nstep, extra=ex,
                                         force=force)


@pytest.mark.parametrize("advection", [0, 1, 3])
def test_every_force_class(tmp_path, advection):
    p = _tg(tmp_path, EVERY)
    gpu, _ = S.dns(p, advection=advection)
    D = O.dns_session(p, advection=advection)
    _compare(gpu, D)
    plain = O.dns_session(_tg(tmp_path, None, name="tg0"), advection=advection).physical()
    assert max(np.abs(plain[c] - gpu[c]).max() for c in "uvw") > 1e-6   # the forcing acted


def test_every_force_class_dealiased(tmp_path):
    # with DEALIAS the force is added on the 3/2-padded grid of the products
    p = _tg(tmp_path, EVERY, extra={"DEALIAS": 1})
    gpu, _ = S.dns(p)
    D = O.dns_session(p)
    assert D.dealias
    _compare(gpu, D)


def test_stokes_dealiased_force(tmp_path):
    p = _tg(tmp_path, ["STEADY_X = 0.1*sin(y)*cos(z)", "DRAG_M = 0.05"], extra={"DEALIAS": 1})
    gpu, _ = S.dns(p, advection=3)
    _compare(gpu, O.dns_session(p, advection=3))


@pytest.mark.parametrize("nz", [1, 8])
def test_poiseuille_const_force(tmp_path, nz):
    # u = 1 - y^2 driven by CONST_X = 2 KINVIS (ConstForce, mode 0) is an
    # exact steady solution: the GPU run keeps it and agrees with the oracle
    fields = "uvwp" if nz > 1 else "uvp"
    bc = {"u": "<D> 0", "v": "<D> 0", "p": "<H> 0"}
    if nz > 1:
        bc["w"] = "<D> 0"
    user = ["u = 1-y*y", "v = 0", "p = 0"] + (["w = 0"] if nz > 1 else [])
    p = sessions.rect_session(str(tmp_path / "pois"), 4, 3, x=(0.0, 2.0), y=(-1.0, 1.0),
                              tokens={"N_P": 6, "N_Z": nz, "N_TIME": 3, "D_T": 0.01, "KINVIS": 0.1, "N_STEP": 12,
                                      "TOL_REL": 1e-14},
                              fields=fields, periodic_x=True, bcs={"w": bc}, user=user,
                              force=["CONST_X = 2*KINVIS"])
    gpu, _ = S.dns(p)
    D = O.dns_session(p)
    yy = np.broadcast_to(D.P.M.y, gpu["u"].shape)
    assert np.abs(gpu["u"] - (1 - yy ** 2)).max() < 1e-12
    assert np.abs(gpu["v"]).max() < 1e-12
    _compare(gpu, D)


def test_unsteady_coriolis(tmp_path):
    force = ["CORIOLIS_UNSTEADY = 1", "CORIOLIS_OMEGA_Z = 0.3+0.1*t", "CORIOLIS_DOMEGA_Z_DT = 0.1",
             "CORIOLIS_OMEGA_X = 0.2*cos(t)", "CORIOLIS_DOMEGA_X_DT = -0.2*sin(t)", "CORIOLIS_OMEGA_Y = 0.05"]
    p = _tg(tmp_path, force)
    gpu, _ = S.dns(p)
    _compare(gpu, O.dns_session(p))


def test_forcing_2d_channel(tmp_path):
    # 2-D: the Coriolis term as the reference forms it with two components,
    # drag, sponge and SFD near walls with high-order pressure BCs
    force = ["CORIOLIS_OMEGA_Z = 0.5", "DRAG_M = 0.1*(1-y*y)", "SPONGE_M = 0.5*heav(x-3)", "SPONGE_V = 0.01",
             "SFD_DELTA = 0.3", "SFD_CHI = 0.5", "STEADY_Y = 0.02*cos(x)"]
    p = sessions.rect_session(str(tmp_path / "ch2"), 4, 3, x=(0.0, 2 * np.pi), y=(-1.0, 1.0),
                              tokens={"N_P": 6, "N_TIME": 2, "D_T": 0.01, "KINVIS": 0.1, "N_STEP": 8,
                                      "TOL_REL": 1e-14},
                              fields="uvp", periodic_x=True,
                              bcs={"w": {"u": "<D> 0", "v": "<D> 0", "p": "<H> 0"}},
                              user=["u = 1-y*y+0.1*sin(x)*(1-y*y)", "v = 0.05*(1-y*y)*cos(x)", "p = 0"],
                              force=force)
    gpu, _ = S.dns(p)
    _compare(gpu, O.dns_session(p))


def test_sponge_update_and_file_forcing(tmp_path):
    # SPONGE_UPDATE re-evaluates a time-dependent mask every 2 steps;
    # STEADY_FILE / MOD_A_FILE read u and w from a field file (v absent: zero)
    ctx = S.Context(_tg(tmp_path, None, name="tmp"))
    x, y = ctx.mesh_coords()
    nz, nel, np_ = ctx.nz, ctx.nel, ctx.np
    ctx.close()
    z = (np.arange(nz) * 2 * np.pi / nz)[:, None, None, None]
    fu = 0.05 * np.sin(y)[None] * np.cos(z) + 0 * x[None]
    fw = 0.02 * np.cos(x)[None] + 0 * z
    ffile = str(tmp_path / "forcing.fld")
    S.write_field(ffile, "forcing", np_, nz, nel, 0, 0.0, 0.0, 0.0, 1.0, {"u": fu, "w": fw})
    force = ["SPONGE_M = 0.2*(1+cos(x-t))", "SPONGE_UPDATE = 2", "SPONGE_W = 0.05",
             f"STEADY_FILE ={ffile}", f"MOD_A_FILE ={ffile}", "MOD_ALPHA_X = 0.3", "MOD_ALPHA_Z = 2*t"]
    p = _tg(tmp_path, force)
    gpu, _ = S.dns(p)
    _compare(gpu, O.dns_session(p))


def _run(p, steps, graph):
    ctx = S.Context(p, {"STX_DNS_GRAPH": int(graph)})
    funcs = S._user_functions(p)
    ic = {c: ctx.evaluate(funcs[c], 0.0) for c in ctx.fields if c in funcs}
    D = S.DNS(ctx, 1)
    D.restart(ic, 0.0)
    D.advance(steps)
    period, launches = D.graph_info()
    out = {c: D.field(c) for c in ctx.fields}
    D.close()
    ctx.close()
    return out, period, launches


def test_forced_graph_replay(tmp_path):
    # forcing constant in time: the step cycle is replayed as a CUDA graph and
    # gives the direct steps' fields; a time-dependent term runs every step
    # directly
    p = _tg(tmp_path, ["CONST_X = 0.01", "STEADY_Y = 0.1*sin(x)", "DRAG_M = 0.05", "SFD_DELTA = 0.5",
                       "SFD_CHI = 0.2", "CORIOLIS_OMEGA_Z = 0.3"], nstep=100)
    g, period, launches = _run(p, 100, True)
    d, _, dl = _run(p, 100, False)
    assert period > 0 and launches > 0 and dl == 0
    for c in g:
        tol = 1e-10 if c == "p" else 1e-12
        err = np.linalg.norm(g[c] - d[c]) / max(np.linalg.norm(d[c]), 1e-300)
        assert err < tol, (c, err)
    p2 = _tg(tmp_path, ["MOD_A_X = 1", "MOD_ALPHA_X = 0.1*t"], nstep=100, name="tgt")
    _, period2, launches2 = _run(p2, 100, True)
    assert period2 == 0 and launches2 == 0


@pytest.mark.parametrize("force,code", [(["WHITE_EPS_X = 0.1"], 6), (["SFD_DELTA = 0.5"], 2),
                                        (["STEADY_FILE = no_such_file.fld"], 2)])
def test_force_rejections(tmp_path, force, code):
    p = _tg(tmp_path, force)
    ctx = S.Context(p)
    try:
        with pytest.raises(S.StxError) as e:
            S.DNS(ctx, 1)
        assert e.value.code == code
    finally:
        ctx.close()
