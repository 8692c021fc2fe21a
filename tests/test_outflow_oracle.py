"""The oracle's computed outflow BCs <O> (Dong, Karniadakis & Chryssostomidis
2014; src/bcmgr.cpp:1036-1633) on the CPU.  The reference ships no golden for
them; the check is an exact solution: fully developed Poiseuille flow with a
parabolic inflow, no-slip walls and an outflow exit, which the outflow
conditions keep to round-off when the switch function S0 is sharp (U0Delta
-> 0: the kinetic-energy term vanishes at every exit node), and to the size of
that term otherwise."""
import numpy as np
import pytest

import semtex_oracle as O
from semtex_b200 import sessions


def _channel(path, nz, u0):
    fields = "uvwp" if nz > 1 else "uvp"
    bcs = {"v": {"u": "<D> 1-y*y", "v": "<D> 0", "p": "<H> 0"},
           "w": {"u": "<D> 0", "v": "<D> 0", "p": "<H> 0"},
           "o": {"u": "<O> 0", "v": "<O> 0", "p": "<O> 0"}}
    if nz > 1:
        for g in bcs:
            bcs[g]["w"] = "<O> 0" if g == "o" else "<D> 0"
    return sessions.rect_session(path, 4, 2, x=(0.0, 4.0), y=(-1.0, 1.0),
                                 tokens={"N_P": 6, "N_Z": nz, "N_TIME": 2, "D_T": 0.01, "KINVIS": 0.1,
                                         "N_STEP": 20, "TOL_REL": 1e-14, "U0Delta": u0},
                                 fields=fields, bcs=bcs, side_groups={"left": "v", "right": "o"},
                                 group_names={"o": "outflow"},
                                 user=["u = 1-y*y", "v = 0", "p = 0.2*(4-x)"] + (["w = 0"] if nz > 1 else []))


@pytest.mark.parametrize("nz", [1, 4])
def test_poiseuille_through_outflow_exit(tmp_path, nz):
    D = O.dns_session(_channel(str(tmp_path / "ch"), nz, 1e-8))
    assert len(D.oedges) == 2
    ph = D.physical()
    y, x = D.P.M.y[None], D.P.M.x[None]
    assert np.abs(ph["u"] - (1 - y * y)).max() < 1e-12
    assert np.abs(ph["v"]).max() < 1e-12
    assert np.abs(ph["p"] - 0.2 * (4 - x)).max() < 1e-12


def test_outflow_energy_term_acts(tmp_path):
    # a smooth switch: near the walls the exit carries KE S0 != 0
    D = O.dns_session(_channel(str(tmp_path / "ch"), 1, 0.05))
    y = D.P.M.y[None]
    err = np.abs(D.physical()["u"] - (1 - y * y)).max()
    assert 1e-8 < err < 1e-4


@pytest.mark.parametrize("nz", [1, 4])
def test_outflow_numbering_host_matches_oracle(tmp_path, nz):
    # the library's host numbering classifies outflow edges as the oracle
    # does: pressure essential, u and v natural (computed), w natural zero
    import semtex_b200 as S
    p = _channel(str(tmp_path / "ch"), nz, 0.05)
    P = O.Problem(O.read_session(p))
    for c in P.S.fields:
        n = S.numbering(p, c)
        N = P.N[c]
        assert (n["nglobal"], n["nsolve"], int(n["bmask"].sum())) == (N.nglobal, N.nsolve, int(N.bmask.sum())), c
    assert S.numbering(p, "p")["nsolve"] < S.numbering(p, "p")["nglobal"]    # the exit pins the pressure


def test_outflow_needs_outflow_group(tmp_path):
    # BCmgr rejects a type 'O' BC whose group is not described as "outflow"
    # (src/bcmgr.cpp:418-419); the oracle and the host numbering do the same
    import semtex_b200 as S
    fields = "uvp"
    bcs = {"v": {"u": "<D> 1-y*y", "v": "<D> 0", "p": "<H> 0"},
           "w": {"u": "<D> 0", "v": "<D> 0", "p": "<H> 0"},
           "o": {"u": "<O> 0", "v": "<O> 0", "p": "<O> 0"}}
    p = sessions.rect_session(str(tmp_path / "bad"), 4, 2, x=(0.0, 4.0), y=(-1.0, 1.0),
                              tokens={"N_P": 5, "N_Z": 1, "N_TIME": 2, "D_T": 0.01, "KINVIS": 0.1},
                              fields=fields, bcs=bcs, side_groups={"left": "v", "right": "o"},
                              group_names={"o": "exit"}, user=["u = 1-y*y", "v = 0", "p = 0"])
    with pytest.raises(ValueError, match="outflow"):
        O.Problem(O.read_session(p))
    with pytest.raises(RuntimeError, match="outflow"):
        S.numbering(p, "p")
