"""Host-side cylindrical coordinates against the oracle (CPU): r-weighted
element Helmholtz matrices with betak2 / r^2 + lambda2 (src/element.cpp:
1389-1399, 1411-1481) and the axis-BC numberings of Fourier modes 0, 1, 2+
(src/bcmgr.cpp:153-180, 550-583), through the host-only C-ABI entries."""
import os

import numpy as np
import pytest

import semtex_oracle as O
import semtex_b200 as S

from conftest import SESSIONS


@pytest.mark.parametrize("name", ["tc1", "cylkov2", "laplace8", "tube1", "taylor3"])
def test_element_matrices(name):
    path = os.path.join(SESSIONS, name)
    P = O.Problem(O.read_session(path))
    for e in sorted({0, P.nel // 2, P.nel - 1}):
        for lam, bk2 in ((2.5, 1.7), (0.0, 4.0), (1e3, 0.0)):
            H = S.element_matrix(path, e, lam, bk2)
            Ho = O.helmholtz_matrix(P.M, e, lam, bk2)
            assert np.abs(H - Ho).max() <= 1e-12 * np.abs(Ho).max(), (name, e, lam, bk2)


@pytest.mark.parametrize("name", ["cylkov2", "laplace8", "tube2", "tc1"])
def test_axis_numberings(name):
    path = os.path.join(SESSIONS, name)
    P = O.Problem(O.read_session(path))
    for c in P.S.fields:
        for m in (0, 1, 2, 5):
            n = S.numbering(path, c, mode=m)
            N, _ = P.nb(c, m)
            assert (n["nglobal"], n["nsolve"]) == (N.nglobal, N.nsolve), (name, c, m)
            assert int(n["bmask"].sum()) == int(N.bmask.sum()), (name, c, m)
            if N.nsolve == N.nglobal:        # no essential nodes: enumerate -O3, node for node
                np.testing.assert_array_equal(n["btog"], N.btog)


def test_axis_classes():
    # cylkov2 reaches the axis: u and p natural there in mode 0 only, w~ in
    # mode 1 only, v~ never
    path = os.path.join(SESSIONS, "cylkov2")
    ns = {(c, m): S.numbering(path, c, mode=m)["nsolve"] for c in "uvwp" for m in (0, 1, 2)}
    assert ns[("u", 0)] > ns[("u", 1)] == ns[("u", 2)]
    assert ns[("p", 0)] > ns[("p", 1)] == ns[("p", 2)]
    assert ns[("w", 1)] > ns[("w", 0)] == ns[("w", 2)]
    assert ns[("v", 0)] == ns[("v", 1)] == ns[("v", 2)]
