"""The oracle's analysis restatements on flows with known answers (CPU):
the wall forces and tractions of plane Poiseuille flow (Field::
normTraction / tangTraction / traction, src/field.cpp:392-593), the
AVERAGE 3 correlations of a uniform shear (Statistics::update,
src/statistics.cpp:247-391) and history-point probes of a smooth field
(AuxField::probe, src/auxfield.cpp:1621-1700).  The device paths are checked against these
restatements by the GPU tests."""
import numpy as np

import semtex_oracle as O
from semtex_b200 import sessions


def _channel(tmp_path, nz, extra=None):
    p = sessions.channel_session(str(tmp_path / "pois"), 4, 2, 7, nz, re=50.0, extra=extra)
    S = O.read_session(p)
    P = O.Problem(S)
    D = O.DNS(P)
    y = P.M.y
    shape = (P.nz, P.nel, P.np, P.np)
    phys = {c: np.zeros(shape) for c in S.fields}
    phys["u"] = np.broadcast_to(1.0 - y * y, shape).copy()
    phys["p"] = np.broadcast_to(0.3 + 0.0 * y, shape).copy()
    for c, v in phys.items():
        f = O.dft_forward(v) if P.nz > 1 else v
        if P.nz > 1:
            f[1] = 0.0
        D.u[c] = f
    return S, P, D


def test_poiseuille_wall_forces_and_tractions(tmp_path):
    for nz in (1, 4):
        S, P, D = _channel(tmp_path, nz)
        mu = S.tokens["KINVIS"]
        lx = 2 * np.pi
        pf, vf = D.wall_forces()
        # du/dy = -2y: a shear stress 2 mu on each wall, both pulled along +x;
        # the uniform pressure pushes the two walls apart equally
        assert abs(vf[0] - 2 * 2 * mu * lx) < 1e-10 and abs(vf[1]) < 1e-10 and abs(vf[2]) < 1e-10
        assert abs(pf[0]) < 1e-10 and abs(pf[1]) < 1e-10
        T = D.wall_traction()
        walls = [(e, s) for (e, s, k, g) in S.surfaces if k == "B" and S.groups.get(g) == "wall"]
        for b, (e, s) in enumerate(walls):
            sl = slice(b * P.np, (b + 1) * P.np)
            bottom = P.M.y[e].ravel()[P.M.side_nodes(s)].mean() < 0
            assert np.allclose(T[0][:, sl], 0.3, atol=1e-12)                       # normal: the pressure
            assert np.allclose(T[1][:, sl], 2 * mu if bottom else -2 * mu, atol=1e-10)
            assert np.allclose(T[2][:, sl], 0.0, atol=1e-12)


def test_uniform_shear_energy_correlations(tmp_path):
    # u = y, v = w = 0: S_xy = 1/2, S_ij S_ij = 2 S_xy^2 = 1/2, q = y^2 / 2,
    # S_ij u_j = (0, y / 2, 0), q u = y^3 / 2
    S, P, D = _channel(tmp_path, 4, extra={"AVERAGE": 3})
    y = np.broadcast_to(P.M.y, (P.nz,) + P.M.y.shape)
    D.u["u"] = O.dft_forward(y.copy())
    D.u["u"][1] = 0.0
    D.u["p"] = np.zeros_like(D.u["p"])
    D.stats_init(3)
    D.stats_update()
    A = D.stats_physical()
    assert len(A) == 27
    expect = {"H": 0.5 + 0 * y, "d": 0.5 + 0 * y, "G": 0 * y, "I": 0 * y, "L": 0 * y, "J": 0 * y, "K": 0 * y,
              "a": 0 * y, "b": 0.5 * y, "c": 0 * y, "q": 0.5 * y * y, "r": 0.5 * y ** 3, "s": 0 * y, "t": 0 * y,
              "A": y * y, "m": 0 * y}
    for c, v in expect.items():
        assert np.abs(A[c] - v).max() < 1e-10, c


def test_probe_reproduces_a_smooth_field(tmp_path):
    # AuxField::probe on u = sin(x) cos(y) (cos z + 0.5 sin 2z): the
    # interpolants and the Fourier series reproduce it to the resolution
    p = sessions.taylor_green_session(str(tmp_path / "tgp"), 4, 11, 8)
    S = O.read_session(p)
    P = O.Problem(S)
    D = O.DNS(P)
    x, y = P.M.x, P.M.y
    z = (np.arange(P.nz) * 2 * np.pi / P.nz)[:, None, None, None]
    u = np.sin(x) * np.cos(y) * (np.cos(z) + 0.5 * np.sin(2 * z))
    for c in S.fields:
        f = O.dft_forward(u if c == "u" else 0 * u)
        f[1] = 0.0
        D.u[c] = f
    rng = np.random.default_rng(3)
    pts = np.column_stack([rng.uniform(0, 2 * np.pi, 12), rng.uniform(0, 2 * np.pi, 12), rng.uniform(-3, 9, 12)])
    got = D.probe(pts)
    want = np.sin(pts[:, 0]) * np.cos(pts[:, 1]) * (np.cos(pts[:, 2]) + 0.5 * np.sin(2 * pts[:, 2]))
    assert np.abs(got[:, 0] - want).max() < 1e-6
    assert np.abs(got[:, 1:]).max() == 0.0
