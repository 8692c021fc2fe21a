"""Session writer produces the benchmark workloads' shapes (CPU, oracle numbering)."""
import numpy as np

import semtex_oracle as O
from semtex_b200 import sessions


def test_c1_shape_and_exact(tmp_path):
    p = sessions.helmholtz_session(str(tmp_path / "c1"), 4, 9, user=[
        "forcing -(2.0*PI*PI+LAMBDA2)*sin(PI*x)*sin(PI*y)", "exact sin(PI*x)*sin(PI*y)"])
    P, U = O.elliptic(p)
    assert P.N["c"].nsolve == 177 and P.N["c"].nglobal == 305
    assert np.abs(U - O.exact_field(P)).max() < 1e-12


def test_tg_periodic_numbering(tmp_path):
    p = sessions.taylor_green_session(str(tmp_path / "tg"), 3, 5, 4)
    S = O.read_session(p)
    P = O.Problem(S)
    # fully periodic: every boundary node is solved for, 3x3 grid of 4x4 edges
    assert P.N["u"].nglobal == 3 * 3 * (1 + 2 * 3)
