"""stx_field_solve_noalloc: the solve for callers that cannot allocate.

Hosts that own all device memory through their own allocator, or loops that
cannot take the synchronisation a cudaMalloc may imply, need a solve that
allocates nothing.  This entry point uses a fixed 8 MiB device array for its
scratch instead of growing a workspace.  Checked here:
- on a fresh context, after one set-up call, a second call changes the
  device's free memory by nothing (cudaMemGetInfo before and after);
- two calls in a row (the array keeps the previous call's contents, which
  must not leak into the next result) agree with stx_field_solve and with the
  oracle, and leave the system's status word at 0;
- a problem needing more scratch than the array holds is rejected.
Collected last on purpose: a failure here leaves every other test already run.
"""
import numpy as np
import pytest

import semtex_oracle as O
import semtex_b200 as S
from semtex_b200 import _lib, sessions

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_noalloc_allocates_nothing_and_matches(tmp_path):
    import torch
    p = sessions.helmholtz_session(str(tmp_path / "na"), 5, 7, nz=8, lambda2=1.0, beta=1.0)
    ctx = S.Context(p)
    rng = np.random.default_rng(42)
    f = rng.uniform(-1, 1, (ctx.nz, ctx.nel, ctx.np, ctx.np))
    F = ctx.new_field("f").load_physical(f).transform(S.FORWARD).zero_nyquist()
    sysm = S.ModalMatrixSys(ctx, "c", 1.0)
    outs = [ctx.new_field("c") for _ in range(3)]
    L = _lib.lib()
    dev = torch.device(f"cuda:{ctx.device}")
    # set-up call: maps the static array on this device (lazy module load)
    _lib.check(L.stx_field_solve_noalloc(sysm.handle, F.ptr(), outs[0].ptr()))
    torch.cuda.synchronize(dev)
    got = []
    for k in (1, 2):
        free0, _ = torch.cuda.mem_get_info(dev)
        _lib.check(L.stx_field_solve_noalloc(sysm.handle, F.ptr(), outs[k].ptr()))
        torch.cuda.synchronize(dev)
        free1, _ = torch.cuda.mem_get_info(dev)
        assert free1 == free0, f"call {k} changed free device memory by {free0 - free1} bytes"
    assert sysm.status() == 0
    # only now the allocating entry point, for the comparison
    ref = ctx.new_field("c").solve(F, sysm).to_numpy()
    for k in (1, 2):
        got = outs[k].to_numpy()
        assert _rel(got, ref) < TOL
    # and the oracle, in physical space
    outs[2].transform(S.INVERSE)
    _, U = O.elliptic(p, forcing_phys=f)
    assert _rel(outs[2].to_numpy(), U) < TOL


def test_noalloc_rejects_oversize(tmp_path):
    # 20x20 quads at N_P=5 have 2961 global boundary nodes; with N_Z=256 the
    # two-level solve needs 3 * 2976 * 256 doubles, more than the 2^20 available.
    p = sessions.helmholtz_session(str(tmp_path / "big"), 20, 5, nz=256, lambda2=1.0, beta=1.0)
    ctx = S.Context(p)
    sysm = S.ModalMatrixSys(ctx, "c", 1.0)
    F, U = ctx.new_field("f"), ctx.new_field("c")
    rc = _lib.lib().stx_field_solve_noalloc(sysm.handle, F.ptr(), U.ptr())
    assert rc == _lib.STX_EINVAL
    assert b"static maximum" in _lib.lib().stx_last_error()
