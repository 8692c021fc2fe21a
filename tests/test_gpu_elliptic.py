"""GPU parity of the condensed Helmholtz solve against the oracle (FP64).

Bar: relative L2 difference <= 1e-10 between the CUDA path (through the C
ABI) and the oracle's restatement of Field::solve on the same session and
forcing; plus agreement with the analytic solutions the sessions carry.
"""
import os

import numpy as np
import pytest

import semtex_oracle as O
import semtex_b200 as S
from semtex_b200 import sessions

from conftest import SESSIONS

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("name", ["helmholtz1", "poisson1", "laplace1", "laplace4", "laplace3", "mixed1"])
@pytest.mark.parametrize("iterative", [False, True])
def test_reference_sessions(name, iterative):
    path = os.path.join(SESSIONS, name)
    ov = {"ITERATIVE": 1, "TOL_REL": 1e-14} if iterative else None
    u = S.elliptic(path, overrides=ov, iterative=iterative)
    P, U = O.elliptic(path, ov)
    assert rel_l2(u, U) < (1e-9 if iterative else TOL)


def _random_case(tmp_path, n, np_, nz, seed, perturb=0.0):
    rng = np.random.default_rng(seed)
    xs = ys = None
    if perturb:
        xs = np.linspace(0, 1, n + 1)
        ys = np.linspace(0, 1, n + 1)
        xs[1:-1] += perturb * rng.uniform(-1, 1, n - 1) / n
        ys[1:-1] += perturb * rng.uniform(-1, 1, n - 1) / n
    p = sessions.helmholtz_session(str(tmp_path / f"r{seed}"), n, np_, nz=nz, lambda2=1.0, beta=1.0,
                                   xs=xs, ys=ys)
    ctx = S.Context(p)
    x, y = ctx.mesh_coords()
    f = rng.uniform(-1, 1, (nz, n * n, np_, np_))
    return p, ctx, f


@pytest.mark.parametrize("n,np_,nz,perturb", [(4, 6, 8, 0.0), (5, 7, 6, 0.3), (3, 11, 4, 0.0), (6, 5, 1, 0.25)])
def test_random_forcing_fourier(tmp_path, n, np_, nz, perturb):
    p, ctx, f = _random_case(tmp_path, n, np_, nz, seed=n * 100 + np_, perturb=perturb)
    sysm = S.ModalMatrixSys(ctx, "c", 1.0)
    u = sysm.solve_host(f)
    P, U = O.elliptic(p, forcing_phys=f)
    assert rel_l2(u, U) < TOL
    if perturb:
        assert ctx.families() > 1


def test_two_calls_in_a_row_identical(tmp_path):
    p, ctx, f = _random_case(tmp_path, 4, 6, 8, seed=7)
    sysm = S.ModalMatrixSys(ctx, "c", 1.0)
    u1 = sysm.solve_host(f).copy()
    u2 = sysm.solve_host(f)
    assert rel_l2(u1, u2) < 1e-14
    assert sysm.status() == 0   # every bounded wait met its copy


def test_device_solve_and_transform(tmp_path):
    import torch
    p, ctx, f = _random_case(tmp_path, 4, 6, 8, seed=11)
    F = ctx.new_field("f").load_physical(f)
    F.transform(S.FORWARD)
    fo = O.dft_forward(f)
    got = F.to_numpy()
    assert rel_l2(got, fo) < 1e-14
    F.zero_nyquist()
    U = ctx.new_field("c")
    sysm = S.ModalMatrixSys(ctx, "c", 1.0)
    U.solve(F, sysm)
    U.transform(S.INVERSE)
    P, Uo = O.elliptic(p, forcing_phys=f)
    assert rel_l2(U.to_numpy(), Uo) < TOL


@pytest.mark.parametrize("nz", [4, 6, 10, 12, 14, 64, 96])
def test_transform_roundtrip_odd_factors(tmp_path, nz):
    # radix 4/2/3/5 FFT paths, and the DFT for a factor outside 2, 3, 5 (14)
    p = sessions.helmholtz_session(str(tmp_path / "t"), 2, 5, nz=nz)
    ctx = S.Context(p)
    rng = np.random.default_rng(nz)
    f = rng.standard_normal((nz, 4, 5, 5))
    F = ctx.new_field().load_physical(f)
    F.transform(S.FORWARD)
    assert rel_l2(F.to_numpy(), O.dft_forward(f)) < 1e-14
    F.transform(S.INVERSE)
    assert rel_l2(F.to_numpy(), f) < 1e-14


@pytest.mark.parametrize("n,np_,nz,perturb", [(8, 9, 8, 0.0), (8, 7, 6, 0.3)])
def test_mixed_precision_refined(tmp_path, n, np_, nz, perturb):
    """STX_MIXED: FP32 skeleton matrices (FP64 sums) with FP64 iterative
    refinement on the skeleton system reaches the FP64 oracle to 1e-10 (the
    default two refinements); without refinement (STX_REFINE = 0) the FP32
    matrices alone leave an error above 1e-9, so the refinement does the work."""
    p, ctx, f = _random_case(tmp_path, n, np_, nz, seed=n * 10 + np_, perturb=perturb)
    plain = S.ModalMatrixSys(ctx, "c", 1.0).solve_host(f)
    mixed = S.ModalMatrixSys(ctx, "c", 1.0, method=S.MIXED).solve_host(f)
    P, U = O.elliptic(p, forcing_phys=f)
    assert rel_l2(plain, U) < TOL
    assert rel_l2(mixed, U) < TOL, rel_l2(mixed, U)
    ctx0 = S.Context(p, overrides={"STX_REFINE": 0})
    none = S.ModalMatrixSys(ctx0, "c", 1.0, method=S.MIXED).solve_host(f)
    assert rel_l2(none, U) > 1e-9, rel_l2(none, U)


def test_mixed_precision_rejects_singular_systems():
    ctx = S.Context(os.path.join(SESSIONS, "taylor2"))
    with pytest.raises(S.StxError):
        S.ModalMatrixSys(ctx, "p", 0.0, method=S.MIXED)


@pytest.mark.parametrize("nf", [3, 2])
def test_multi_field_solve_matches_single(tmp_path, nf):
    """stx_field_solve_multi: velocity systems that share their matrices are
    solved with one skeleton pass for all fields; the results equal the
    one-by-one solves (round-off) and the oracle (1e-10)."""
    p = sessions.channel_session(str(tmp_path / "mf"), 4, 3, 7, 8, extra={"TOL_REL": 1e-14})
    ctx = S.Context(p)
    lam = 3.7
    names = "uvw"[:nf]
    systems = [S.ModalMatrixSys(ctx, c, lam) for c in names]
    rng = np.random.default_rng(nf)
    fs, single, multi, phys = [], [], [], []
    for c in names:
        f = rng.uniform(-1, 1, (ctx.nz, ctx.nel, ctx.np, ctx.np))
        phys.append(f)
        fs.append(ctx.new_field("f" + c).load_physical(f).transform(S.FORWARD).zero_nyquist())
        single.append(ctx.new_field("s" + c))
        multi.append(ctx.new_field("m" + c))
    for sys_, F, U in zip(systems, fs, single):
        U.solve(F, sys_)
    S.solve_multi(systems, fs, multi)
    P = O.Problem(O.read_session(p))
    for i, c in enumerate(names):
        a, b = multi[i].to_numpy(), single[i].to_numpy()
        assert rel_l2(a, b) < 1e-13, (c, rel_l2(a, b))
        F = O.dft_forward(phys[i])
        F[1] = 0.0
        Uo = P.solve(c, F, np.zeros_like(F), P.modal_systems(c, lam), P.bc_lines(c))
        Uo[1] = 0.0
        assert rel_l2(a, Uo) < TOL, (c, rel_l2(a, Uo))
    for sys_ in systems:
        sys_.close()
    ctx.close()



def _robin_session(path, nx, ny, np_, nz, K, C):
    """Periodic in x, Dirichlet 0 at y = 0, mixed dc/dn + K (c - C) = 0 at y = 1."""
    p = sessions.rect_session(path, nx, ny, tokens={"N_P": np_, "N_Z": nz, "BETA": 1.0, "LAMBDA2": 1.0,
                                                     "TOL_REL": 1e-14},
                              periodic_x=True, bcs={"w": {"c": f"<M> {K};{C}"}})
    txt = open(p).read()
    txt = txt.replace("<GROUPS NUMBER=1>", "<GROUPS NUMBER=2>\n\t2\tz\tclamp")
    txt = txt.replace("<BCS NUMBER=1>", "<BCS NUMBER=2>\n\t2\tz\t1\n\t\t<D>\tc = 0\t</D>")
    out = []
    for ln in txt.splitlines():
        parts = ln.split("\t")
        if len(parts) >= 4 and parts[3] == "1" and "<B>" in ln:   # side 1: bottom
            ln = ln.replace("<B>\tw\t</B>", "<B>\tz\t</B>")
        out.append(ln)
    open(p, "w").write("\n".join(out) + "\n")
    return p


@pytest.mark.parametrize("solver", ["twolevel", "band", "pcg"])
def test_mixed_bc_fourier(tmp_path, solver):
    """Mixed (Robin) BCs (src/condition.cpp:295-435) in 3D, against the oracle:
    K C <1, w> on every plane, K <c, w> on the boundary-system diagonal."""
    p = _robin_session(str(tmp_path / "rb"), 8, 6, 7, 8, 2.5, 0.3)
    ov = {"STX_TWOLEVEL": 0} if solver == "band" else ({"ITERATIVE": 1} if solver == "pcg" else None)
    ctx = S.Context(p, ov)
    rng = np.random.default_rng(5)
    f = rng.uniform(-1, 1, (ctx.nz, ctx.nel, ctx.np, ctx.np))
    sysm = S.ModalMatrixSys(ctx, "c", 1.0, method=S.JACPCG if solver == "pcg" else S.DIRECT)
    u = sysm.solve_host(f)
    P, U = O.elliptic(p, {"ITERATIVE": 1} if solver == "pcg" else None, forcing_phys=f)
    assert rel_l2(u, U) < (1e-9 if solver == "pcg" else TOL), rel_l2(u, U)
    with pytest.raises(S.StxError):
        S.ModalMatrixSys(ctx, "c", 1.0, method=S.MIXED)
    sysm.close()
    ctx.close()


@pytest.mark.parametrize("n,np_,nz", [(4, 2, 4), (3, 3, 8), (5, 4, 2), (1, 5, 4), (2, 2, 1)])
def test_edge_sizes(tmp_path, n, np_, nz):
    """Linear elements (N_P = 2: no interior nodes), quadratics, N_Z = 2 (mean
    and Nyquist planes only), a single element; direct and PCG."""
    p, ctx, f = _random_case(tmp_path, n, np_, nz, seed=n * 1000 + np_ * 10 + nz)
    P, U = O.elliptic(p, forcing_phys=f)
    u = S.ModalMatrixSys(ctx, "c", 1.0).solve_host(f)
    assert rel_l2(u, U) < TOL, rel_l2(u, U)
    ctx2 = S.Context(p, {"ITERATIVE": 1, "TOL_REL": 1e-14})
    ui = S.ModalMatrixSys(ctx2, "c", 1.0, method=S.JACPCG).solve_host(f)
    assert rel_l2(ui, U) < 1e-9, rel_l2(ui, U)
