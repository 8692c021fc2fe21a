"""GPU parity of the spectral-vanishing-viscosity systems (src/svv.cpp,
src/element.cpp:1454-1455, src/matrix.cpp:78-83) against the oracle: the
viscous (lambda2 > 0) Helmholtz systems take the SVV derivative in the plane
and SVV-scaled beta^2 k^2 across the Fourier modes, in the direct and the
Jacobi-PCG solves and in the DNS viscous step.  Bar as the other solve
tests: 1e-10 relative L2 (PCG 1e-9)."""
import numpy as np
import pytest

import semtex_oracle as O
import semtex_b200 as S
from semtex_b200 import sessions

pytestmark = pytest.mark.gpu

SVV = {"SVV_MN": 3, "SVV_EPSN": 0.1, "SVV_MZ": 1, "SVV_EPSZ": 0.05, "KINVIS": 0.5}


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("method", [S.DIRECT, S.JACPCG])
@pytest.mark.parametrize("nz", [1, 8])
def test_svv_helmholtz(tmp_path, method, nz):
    # essential values varying along the boundary exercise -H g with the SVV
    # operator; random forcing every mode
    tok = {"N_P": 7, "N_Z": nz, "LAMBDA2": 2.0, "BETA": 1.0, "TOL_REL": 1e-14, "STEP_MAX": 2000}
    tok.update(SVV)
    if method == S.JACPCG:
        tok["ITERATIVE"] = 1
    p = sessions.rect_session(str(tmp_path / "svv"), 4, 3, tokens=tok, fields="c",
                              bcs={"w": {"c": "<D> 1+x*y"}})
    ctx = S.Context(p)
    rng = np.random.default_rng(11)
    f = rng.uniform(-1, 1, (nz, ctx.nel, ctx.np, ctx.np))
    u = S.ModalMatrixSys(ctx, "c", 2.0, method=method).solve_host(f)
    ctx.close()
    _, U = O.elliptic(p, forcing_phys=f)
    assert rel_l2(u, U) < (1e-9 if method == S.JACPCG else 1e-10)
    _, U0 = O.elliptic(p, {k: (-1 if k.endswith(("MN", "MZ")) else 0.0) for k in SVV if k.startswith("SVV")},
                       forcing_phys=f)
    assert rel_l2(U0, U) > 1e-6                                   # SVV changed the solution


@pytest.mark.parametrize("ntime", [1, 3])
def test_svv_dns(tmp_path, ntime):
    # the start-up steps use Jacobi-PCG viscous systems, the later ones the
    # direct ones: both with SVV
    ex = {"TOL_REL": 1e-14, "N_TIME": ntime, "SVV_MN": 3, "SVV_EPSN": 0.02, "SVV_MZ": 1, "SVV_EPSZ": 0.01}
    p = sessions.taylor_green_session(str(tmp_path / "tgs"), 3, 6, 8, re=100.0, dt=2e-3, nstep=6, extra=ex)
    gpu, _ = S.dns(p)
    D = O.dns_session(p)
    phys = D.physical()
    scale = max(np.linalg.norm(phys[c]) for c in D.vel)
    for c in D.vel:
        assert np.linalg.norm(gpu[c] - phys[c]) / scale < 1e-10, c
    pscale = max(np.linalg.norm(phys["p"]), np.linalg.norm(sum(phys[c] ** 2 for c in D.vel)))
    assert np.linalg.norm(gpu["p"] - phys["p"]) / pscale < 1e-9
