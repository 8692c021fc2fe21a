"""stx_field_solve_noalloc: the solve for callers that cannot allocate.

Hosts that own all device memory through their own allocator, or loops that
cannot take the synchronisation a cudaMalloc may imply, need a solve that
allocates nothing.  This entry point uses a fixed 8 MiB device array for its
scratch instead of growing a workspace.  Checked here against stx_field_solve
on the same inputs, on two calls in a row (the array keeps the previous
call's contents, which must not leak into the next result), and for the
error it returns when a problem needs more scratch than the array holds.
Collected last on purpose: a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

import semtex_b200 as S
from semtex_b200 import _lib, sessions

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_noalloc_matches_solve_twice(tmp_path):
    p = sessions.helmholtz_session(str(tmp_path / "na"), 5, 7, nz=8, lambda2=1.0, beta=1.0)
    ctx = S.Context(p)
    rng = np.random.default_rng(42)
    f = rng.uniform(-1, 1, (ctx.nz, ctx.nel, ctx.np, ctx.np))
    F = ctx.new_field("f").load_physical(f).transform(S.FORWARD).zero_nyquist()
    sysm = S.ModalMatrixSys(ctx, "c", 1.0)
    ref = ctx.new_field("c").solve(F, sysm).to_numpy()
    L = _lib.lib()
    for _ in range(2):
        U = ctx.new_field("c")
        _lib.check(L.stx_field_solve_noalloc(sysm.handle, F.ptr(), U.ptr()))
        got = U.to_numpy()
        assert _rel(got, ref) < TOL


def test_noalloc_rejects_oversize(tmp_path):
    # 20x20 quads at N_P=5 have 2961 global boundary nodes; with N_Z=256 the
    # solve needs 2 * 2976 * 256 doubles, more than the 2^20 available.
    p = sessions.helmholtz_session(str(tmp_path / "big"), 20, 5, nz=256, lambda2=1.0, beta=1.0)
    ctx = S.Context(p)
    sysm = S.ModalMatrixSys(ctx, "c", 1.0)
    F, U = ctx.new_field("f"), ctx.new_field("c")
    rc = _lib.lib().stx_field_solve_noalloc(sysm.handle, F.ptr(), U.ptr())
    assert rc == _lib.STX_EINVAL
    assert b"static maximum" in _lib.lib().stx_last_error()
