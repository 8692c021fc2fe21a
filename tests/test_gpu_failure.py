"""Failure paths on the GPU, none of which faults, traps or hangs the device.

- A bounded wait that runs out: session token STX_WAIT_NS = 0 makes every
  first wait of the element and skeleton kernels one non-blocking probe, which
  a bulk copy issued just before misses.  The kernels record the error in the
  system's status word, drain their copies with the default bound and return;
  the host reads the word (stx_modal_status, stx_elliptic_solve_host) and the
  context stays usable: a system with the default bound then solves correctly.
- STX_ENOCONV: a Jacobi-PCG solve stopped at STEP_MAX (src/field.cpp:790,
  where the reference prints "step limit exceeded" and carries on).
- STX_ENUMERIC: a system that is not positive definite, whose Cholesky
  factorisation fails during setup (the reference's dpbtrf check,
  src/matrix.cpp:254, stops the run).
"""
import ctypes as C

import numpy as np
import pytest

import semtex_b200 as S
from semtex_b200 import _lib, sessions

pytestmark = pytest.mark.gpu


def _case(tmp_path, name, overrides=None, n=4, np_=7, nz=8, lambda2=1.0):
    p = sessions.helmholtz_session(str(tmp_path / name), n, np_, nz=nz, lambda2=lambda2, beta=1.0)
    ctx = S.Context(p, overrides)
    f = np.random.default_rng(7).uniform(-1, 1, (ctx.nz, ctx.nel, ctx.np, ctx.np))
    return p, ctx, f


def test_expired_wait_is_reported_and_context_survives(tmp_path):
    p, ctx, f = _case(tmp_path, "w0", {"STX_WAIT_NS": 0})
    sysm = S.ModalMatrixSys(ctx, "c", 1.0)
    # asynchronous device-buffer solve: the word is read afterwards
    F = ctx.new_field("f").load_physical(f).transform(S.FORWARD).zero_nyquist()
    U = ctx.new_field("c")
    _lib.check(_lib.lib().stx_field_solve(sysm.handle, F.ptr(), U.ptr(), C.c_double(0.0), 0, None))
    assert sysm.status() in (3, 4)  # element kernel or packed skeleton product
    # the host-buffer solve reads the word itself and fails
    with pytest.raises(_lib.StxError, match="bounded wait"):
        sysm.solve_host(f)
    # the device stays usable: a context with the default bound solves, and
    # the first context (every system of which has the zero bound) still
    # runs work without bulk-copy waits -- a Jacobi-PCG solve -- correctly
    _, ctx2, _ = _case(tmp_path, "w1")
    good = S.ModalMatrixSys(ctx2, "c", 2.0)
    u = good.solve_host(f)
    assert good.status() == 0
    pcg = S.ModalMatrixSys(ctx, "c", 2.0, method=S.JACPCG)
    F1 = ctx.new_field("f").load_physical(f).transform(S.FORWARD).zero_nyquist()
    U1 = ctx.new_field("c").solve(F1, pcg, tol_rel=1e-14, step_max=5000)
    U1.transform(S.INVERSE)
    u1 = U1.to_numpy()
    assert np.linalg.norm(u1 - u) <= 1e-10 * np.linalg.norm(u)


def test_wait_token_rejects_negative(tmp_path):
    _, ctx, _ = _case(tmp_path, "wneg", {"STX_WAIT_NS": -1})
    with pytest.raises(_lib.StxError, match="STX_WAIT_NS"):
        S.ModalMatrixSys(ctx, "c", 1.0)


def test_pcg_step_limit_is_enoconv(tmp_path):
    p, ctx, f = _case(tmp_path, "pcg")
    sysm = S.ModalMatrixSys(ctx, "c", 1.0, method=S.JACPCG)
    F = ctx.new_field("f").load_physical(f).transform(S.FORWARD).zero_nyquist()
    U = ctx.new_field("c")
    iters = (C.c_int * ctx.nz)()
    rc = _lib.lib().stx_field_solve(sysm.handle, F.ptr(), U.ptr(), C.c_double(1e-14), 1, iters)
    assert rc == _lib.STX_ENOCONV
    assert b"step limit" in _lib.lib().stx_last_error()
    # the Python mirror warns and carries on, as the reference does
    with pytest.warns(UserWarning, match="step limit"):
        ctx.new_field("c").solve(F, sysm, tol_rel=1e-14, step_max=1)
    # with room to converge the same system meets the tolerance
    rc = _lib.lib().stx_field_solve(sysm.handle, F.ptr(), U.ptr(), C.c_double(1e-12), 5000, iters)
    assert rc == _lib.STX_OK


def test_indefinite_system_is_enumeric(tmp_path):
    # a Helmholtz constant lambda2 = -1e6, far below minus the smallest
    # Laplacian eigenvalue: the operator -div grad + lambda2 is negative
    # definite, so is every condensed block, and the first Cholesky pivot fails
    p, ctx, f = _case(tmp_path, "neg", n=3, np_=5, nz=1)
    h = C.c_void_p()
    rc = _lib.lib().stx_modal_create(ctx.handle, b"c", C.c_double(-1.0e6), C.c_double(1.0), 0, 1,
                                     S.DIRECT, C.byref(h))
    assert rc == _lib.STX_ENUMERIC, _lib.lib().stx_last_error()
