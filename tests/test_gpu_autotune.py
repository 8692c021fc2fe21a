"""The autotuner on the device: every knob value it may pick gives the same
solution (to round-off), and a tuning run records a winner no slower than
the defaults, which then solves correctly."""
import numpy as np
import pytest

import semtex_b200 as S
from semtex_b200 import autotune as A, sessions

pytestmark = pytest.mark.gpu


def _solve(p, ov, f):
    ctx = S.Context(p, ov or None)
    sysm = S.ModalMatrixSys(ctx, "c", 1.0)
    u = sysm.solve_host(f)
    assert sysm.status() == 0
    sysm.close()
    ctx.close()
    return u


@pytest.mark.parametrize("ov", [{"STX_PATCH_CAP": 8}, {"STX_PATCH_CAP": 64}, {"STX_CHUNK": 8},
                                {"STX_CHUNK": 3}, {"STX_MODE_GROUPS": 3}, {"STX_SYM_WARPS": 1},
                                {"STX_SYM_WARPS": 8, "STX_SYM_REGCAP": 1}, {"STX_SYM_OCC": 10},
                                {"STX_SYM_OCC": 400}, {"STX_SYM_REGCAP": 1}])
def test_knobs_do_not_change_the_solution(tmp_path, ov):
    p = sessions.helmholtz_session(str(tmp_path / "k"), 8, 7, nz=8, lambda2=1.0, beta=1.0)
    f = np.random.default_rng(2).uniform(-1, 1, (8, 64, 7, 7))
    ref = _solve(p, {}, f)
    got = _solve(p, ov, f)
    assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref)


@pytest.mark.parametrize("ov", [{"STX_ELEM_TWOBLOCK": 1}, {"STX_ELEM_TWOBLOCK": 1, "STX_CHUNK": 16},
                                {"STX_STAGGER": 1}])
def test_element_tiers_do_not_change_the_solution(tmp_path, ov):
    # N_P = 11 with 32-element chunks: the recovery's operator rows exceed the
    # two-block tier unless split into row blocks
    p = sessions.helmholtz_session(str(tmp_path / "t"), 6, 11, nz=4, lambda2=1.0, beta=1.0)
    f = np.random.default_rng(3).uniform(-1, 1, (4, 36, 11, 11))
    ref = _solve(p, {}, f)
    got = _solve(p, ov, f)
    assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref)


def test_tune_records_winner(tmp_path):
    p = sessions.helmholtz_session(str(tmp_path / "t"), 8, 7, nz=8, lambda2=1.0, beta=1.0)
    table = str(tmp_path / "table.json")
    space = {"STX_CHUNK": [None, 8], "STX_SYM_WARPS": [None, 2]}
    e = A.tune(p, "c", 1.0, space=space, reps=3, path=table)
    assert e["best_ms"] <= e["default_ms"] and len(e["trials"]) == 3
    ov = A.tuned_overrides(p, "c", 1.0, table)
    assert ov == e["best"]
    f = np.random.default_rng(4).uniform(-1, 1, (8, 64, 7, 7))
    assert np.linalg.norm(_solve(p, ov, f) - _solve(p, {}, f)) <= 1e-12 * np.linalg.norm(_solve(p, {}, f))


def test_tune_batch_records_one_setting(tmp_path):
    specs = [{"n": 3, "np": 6, "lambda2": 1.0, "seed": 1}, {"n": 5, "np": 8, "lambda2": 10.0, "seed": 2},
             {"n": 4, "np": 7, "lambda2": 0.5, "seed": 3}]
    table = str(tmp_path / "table.json")
    e = A.tune_batch(specs, space={"STX_CHUNK": [None, 8]}, reps=3, path=table)
    assert e["best_ms"] <= e["default_ms"] and len(e["trials"]) == 2
    assert A.tuned_batch_overrides(specs, table) == e["best"]
    assert A.tuned_batch_overrides(specs[:2], table) == {}
