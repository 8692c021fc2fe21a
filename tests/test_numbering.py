"""The host numbering (`stx_numbering_host`, no GPU) against the oracle.

Fields without essential nodes take the reference's `enumerate -O3`
numbering in both codes (utility/enumerate.cpp:694-964): identical global
numbers, hence the same pinned node of the singular k=0 system.  Fields with
essential nodes: the same node sets and counts (the orderings are each
code's own reverse Cuthill--McKee).
"""
import os

import numpy as np
import pytest

import semtex_oracle as O
import semtex_b200 as S

from conftest import SESSIONS


@pytest.mark.parametrize("name", ["kovas1", "kovas3", "kovas5", "taylor2", "taylor4", "tgreen"])
def test_essential_free_fields_match_enumerate(name):
    path = os.path.join(SESSIONS, name)
    P = O.Problem(O.read_session(path))
    for c in P.S.fields:
        N = P.N[c]
        r = S.numbering(path, c)
        assert (r["nglobal"], r["nsolve"]) == (N.nglobal, N.nsolve)
        if N.nglobal == N.nsolve:
            assert np.array_equal(r["btog"], N.btog), (name, c)
            assert r["nband"] == N.nband
            assert not r["bmask"].any()


@pytest.mark.parametrize("name", ["kovas2", "helmholtz1", "laplace1"])
def test_fields_with_essential_nodes(name):
    path = os.path.join(SESSIONS, name)
    P = O.Problem(O.read_session(path))
    for c in P.S.fields:
        N = P.N[c]
        r = S.numbering(path, c)
        assert (r["nglobal"], r["nsolve"]) == (N.nglobal, N.nsolve)
        assert np.array_equal(r["bmask"], N.bmask)
        # the same nodes are identified: equal numbers in one code are equal in the other
        a, b = r["btog"].ravel(), N.btog.ravel()
        pairs = set(zip(a.tolist(), b.tolist()))
        assert len(pairs) == N.nglobal


def test_high_order_bc_on_velocity_is_rejected(tmp_path):
    from semtex_b200 import sessions
    p = sessions.rect_session(str(tmp_path / "bad"), 2, 2, tokens={"N_P": 4}, fields="uvp",
                              bcs={"w": {"u": "<H> 0", "v": "<D> 0", "p": "<H> 0"}})
    with pytest.raises(S.StxError):
        S.numbering(p, "u")
