"""stx_elliptic_solve_host_batch: several whole elliptic solves from host
memory with the copies of neighbouring solves overlapping each solve.  Every
result equals the one-call-at-a-time host-buffer solve of the same forcing
(and so the oracle's, which tests/test_gpu_elliptic.py checks), with pinned
and with pageable host buffers, for odd and even counts."""
import numpy as np
import pytest

import semtex_oracle as O
import semtex_b200 as S
from semtex_b200 import sessions

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,pinned", [(5, True), (4, False), (1, True)])
def test_batch_matches_single_calls(tmp_path, n, pinned):
    import torch
    p = sessions.helmholtz_session(str(tmp_path / "b"), 6, 7, nz=8, lambda2=1.0, beta=1.0)
    ctx = S.Context(p)
    sysm = S.ModalMatrixSys(ctx, "c", 1.0)
    rng = np.random.default_rng(11)
    shape = (ctx.nz, ctx.nel, ctx.np, ctx.np)
    fs = [rng.uniform(-1, 1, shape) for _ in range(n)]
    ref = [sysm.solve_host(f) for f in fs]
    if pinned:
        fin = [torch.from_numpy(f).pin_memory() for f in fs]
        fout = [torch.zeros(shape, dtype=torch.float64).pin_memory() for _ in range(n)]
        S.solve_host_batch(sysm, fin, fout)
        got = [t.numpy() for t in fout]
    else:
        got = [np.zeros(shape) for _ in range(n)]
        S.solve_host_batch(sysm, fs, got)
    for g, r in zip(got, ref):
        assert np.linalg.norm(g - r) <= 1e-14 * np.linalg.norm(r)
    _, U = O.elliptic(p, forcing_phys=fs[-1])
    assert np.linalg.norm(got[-1] - U) <= 1e-10 * np.linalg.norm(U)
