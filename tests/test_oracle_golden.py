"""The oracle pinned against the reference's own known answers (CPU).

* regress/*.ok goldens (test/testregress:14-30): `compare -n` ∞-norm errors
  after `dns -chk` on the Taylor-flow sessions, 5 significant digits.
* analytic solutions of the elliptic test sessions (elliptic/testsuite).
"""
import json
import os

import numpy as np
import pytest

import semtex_oracle as O

from conftest import GOLDEN, SESSIONS

GOLD = json.load(open(os.path.join(GOLDEN, "regress_ok.json")))["goldens"]


@pytest.mark.parametrize("name,fields", [
    ("taylor2", "uv"), ("taylor3", "uvw"), ("taylor4", "uvw"), ("taylor5", "uvwp"),
])
def test_dns_regress_goldens(name, fields):
    D = O.dns_session(os.path.join(SESSIONS, name))
    got = O.compare_errors(D)
    for c in fields:
        assert got[c] == GOLD[name][c], (name, c, got[c], GOLD[name][c])


def test_taylor3_mpi_golden_velocity():
    D = O.dns_session(os.path.join(SESSIONS, "taylor3"))
    got = O.compare_errors(D)
    for c in "uvw":
        assert got[c] == GOLD["MPI/taylor3"][c]


@pytest.mark.parametrize("name,tol", [
    ("helmholtz1", 1e-13), ("poisson1", 1e-13), ("laplace4", 1e-13), ("laplace1", 2e-10),
])
def test_elliptic_exact(name, tol):
    P, U = O.elliptic(os.path.join(SESSIONS, name))
    assert np.abs(U - O.exact_field(P)).max() < tol


def test_elliptic_exact_3d_fourier():
    P, U = O.elliptic(os.path.join(SESSIONS, "laplace3"))
    ex = P.evaluate("exp(sqrt(2.0)*x)*sin(y)*sin(z)")
    assert np.abs(U - ex).max() < 1e-11


def test_elliptic_pcg_matches_direct():
    P, U = O.elliptic(os.path.join(SESSIONS, "laplace4"), {"ITERATIVE": 1, "TOL_REL": 1e-14})
    P2, U2 = O.elliptic(os.path.join(SESSIONS, "laplace4"))
    assert np.abs(U - U2).max() < 1e-11


def test_dft_roundtrip_and_convention():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((12, 5))
    f = O.dft_forward(x)
    assert np.allclose(f[0], x.mean(0))
    n = np.arange(12)[:, None]
    assert np.allclose(f[2], (x * np.cos(2 * np.pi * n / 12)).sum(0) / 12)
    assert np.allclose(f[3], -(x * np.sin(2 * np.pi * n / 12)).sum(0) / 12)
    assert np.allclose(O.dft_inverse(f), x)


def test_gll_operators():
    z, w, D = O.gll(9)
    assert abs(w.sum() - 2) < 1e-14
    for p in range(8):
        assert np.abs(D @ z ** p - (p * z ** (p - 1) if p else 0 * z)).max() < 1e-12
