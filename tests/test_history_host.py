"""History-point location on the host (stx_mesh_locate_host; HistoryPoint::
locate / Element::locate, src/history.cpp:45-63, src/element.cpp:
1061-1183) and the relocation of moved particles (stx_mesh_relocate_host;
src/particle.cpp:155-175) against the oracle's restatement, on a mesh of
skewed quads; the oracle's Lagrange interpolants against polynomials and
its particle integrator on a uniform flow."""
import ctypes as C
import re

import numpy as np
import pytest

import semtex_oracle as O
from semtex_b200 import _lib, sessions


@pytest.mark.parametrize("np_", [4, 7, 11])
def test_lagrange_interpolants_reproduce_polynomials(np_):
    z, _, _ = O.gll(np_)
    rng = np.random.default_rng(np_)
    c = rng.standard_normal(np_)           # degree np_ - 1
    p, dp = np.polynomial.polynomial.Polynomial(c), np.polynomial.polynomial.Polynomial(c).deriv()
    for x in rng.uniform(-1, 1, 5):
        h, dh = O.lagrange_interpolants(z, x)
        assert abs(h @ p(z) - p(x)) <= 1e-12 * max(1.0, abs(p(x)))
        assert abs(dh @ p(z) - dp(x)) <= 1e-10 * max(1.0, abs(dp(x)))


def _skewed_session(path, n=4, np_=7):
    """A 4x4-element session on [0, 1]^2 whose interior vertices are moved
    off the grid, so that the elements are general straight-sided quads."""
    sessions.rect_session(path, n, n, tokens={"N_P": np_}, fields="c", bcs={"w": {"c": "<D> 0"}})
    text = open(path).read()
    rng = np.random.default_rng(3)

    def move(m):
        i, x, y = int(m.group(1)), float(m.group(2)), float(m.group(3))
        if 0.0 < x < 1.0 and 0.0 < y < 1.0:
            dx, dy = rng.uniform(-0.3, 0.3, 2) / n
            x, y = x + dx, y + dy
        return f"\t{i}\t{x:.17g}\t{y:.17g}\t0"

    body = re.search(r"<NODES[^>]*>(.*?)</NODES>", text, re.S)
    new = re.sub(r"^\t(\d+)\t(\S+)\t(\S+)\t0$", move, body.group(1), flags=re.M)
    open(path, "w").write(text[:body.start(1)] + new + text[body.end(1):])
    return path


def test_locate_matches_oracle_on_skewed_quads(tmp_path):
    path = _skewed_session(str(tmp_path / "skew"))
    S = O.read_session(path)
    M = O.Problem(S).M
    rng = np.random.default_rng(9)
    pts = np.concatenate([rng.uniform(0.02, 0.98, (40, 2)), [[1.5, 0.5], [-0.2, 0.1]]])
    el = np.empty(len(pts), dtype=np.int32)
    rs = np.empty((len(pts), 2))
    _lib.check(_lib.lib().stx_mesh_locate_host(path.encode(), None, len(pts), C.c_void_p(pts.ctypes.data),
                                               C.c_void_p(el.ctypes.data), C.c_void_p(rs.ctypes.data)))
    for i, (x, y) in enumerate(pts):
        want = O.locate(M, x, y)
        if want is None:
            assert el[i] == -1
            continue
        e, r, s = want
        assert el[i] == e
        assert abs(rs[i, 0] - r) < 1e-12 and abs(rs[i, 1] - s) < 1e-12
        # the located (r, s) maps back to the point
        ir, _ = O.lagrange_interpolants(M.z, rs[i, 0])
        is_, _ = O.lagrange_interpolants(M.z, rs[i, 1])
        assert abs(is_ @ M.x[e] @ ir - x) < 1e-9 and abs(is_ @ M.y[e] @ ir - y) < 1e-9
    assert (el[:40] >= 0).all() and (el[40:] == -1).all()


def test_relocate_matches_oracle(tmp_path):
    path = _skewed_session(str(tmp_path / "skew"))
    S = O.read_session(path)
    M = O.Problem(S).M
    rng = np.random.default_rng(4)
    start = rng.uniform(0.05, 0.95, (30, 2))
    moved = np.clip(start + rng.uniform(-0.08, 0.08, start.shape), 0.0, 1.0)
    moved[0] = (1.2, 0.5)   # left the mesh
    moved = np.ascontiguousarray(moved)
    el = np.empty(len(start), dtype=np.int32)
    rs = np.empty((len(start), 2))
    lib = _lib.lib()
    _lib.check(lib.stx_mesh_locate_host(path.encode(), None, len(start), C.c_void_p(np.ascontiguousarray(start).ctypes.data),
                                        C.c_void_p(el.ctypes.data), C.c_void_p(rs.ctypes.data)))
    want = [O.relocate(M, x, y, int(e), r, s) for (x, y), e, (r, s) in zip(moved, el, rs)]
    _lib.check(lib.stx_mesh_relocate_host(path.encode(), None, len(start), C.c_void_p(moved.ctypes.data),
                                          C.c_void_p(el.ctypes.data), C.c_void_p(rs.ctypes.data)))
    for i, w in enumerate(want):
        if w is None:
            assert el[i] == -1
            continue
        assert el[i] == w[0]
        assert abs(rs[i, 0] - w[1]) < 1e-12 and abs(rs[i, 1] - w[2]) < 1e-12
    assert (el[1:] >= 0).all() and el[0] == -1


def test_particles_follow_a_uniform_flow(tmp_path):
    # the predictor and corrector weights of every order sum to one: a
    # particle in a uniform flow moves by dt * velocity each step
    path = sessions.rect_session(str(tmp_path / "uf"), 4, 4, x=(0.0, 4.0), y=(0.0, 4.0),
                                 tokens={"N_P": 5, "N_Z": 4, "D_T": 0.01, "N_TIME": 3}, fields="uvwp",
                                 periodic_x=True, periodic_y=True)
    S = O.read_session(path)
    M = O.Problem(S).M
    T = O.FluidParticles(M, S.tokens, 4)
    assert T.make(1, (0.5, 0.7, 6.2), 0.0) and not T.make(2, (5.0, 1.0, 0.0), 0.0)
    for _ in range(5):
        T.integrate(lambda e, r, s, z: (1.0, 0.5, 0.25))
    q = T.parts[0]
    assert abs(q["x"] - (0.5 + 0.05)) < 1e-12 and abs(q["y"] - (0.7 + 0.025)) < 1e-12
    assert abs(q["z"] - ((6.2 + 0.0125) % (2 * np.pi))) < 1e-12 and q["e"] is not None
