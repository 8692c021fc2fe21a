"""The DNS with mixed-precision steady velocity solves (token STX_DNS_MIXED:
FP32 packed skeleton inverses, FP64 sums and refinement) against the plain
FP64 DNS on the same run: every field within 1e-10 relative after the
start-up and 20 steady steps; the adjoint rejects it."""
import numpy as np
import pytest

import semtex_b200 as S
from semtex_b200 import _lib, sessions

pytestmark = pytest.mark.gpu


def _run(path, overrides, steps):
    ctx = S.Context(path, overrides=overrides)
    x, y = ctx.mesh_coords()
    ic = sessions.channel_initial(x, y, np.arange(ctx.nz) * 2 * np.pi / ctx.nz, amplitude=0.05)
    D = S.DNS(ctx, 1)
    D.restart({c: ic[c] for c in ctx.fields[:-1]}, 0.0)
    D.advance(steps)
    out = {c: D.field(c) for c in ctx.fields}
    D.close()
    return out


def test_mixed_velocity_solves_match_fp64(tmp_path):
    path = sessions.channel_session(str(tmp_path / "chm"), 4, 2, 8, 8, re=200.0, dt=5e-3)
    ref = _run(path, None, 22)
    mix = _run(path, {"STX_DNS_MIXED": 1}, 22)
    for c in ref:
        err = np.linalg.norm(mix[c] - ref[c]) / np.linalg.norm(ref[c])
        assert err < 1e-10, (c, err)


def test_adjoint_rejects_mixed(tmp_path):
    path = sessions.channel_session(str(tmp_path / "cha"), 4, 2, 6, 8)
    D = S.DNS(S.Context(path, overrides={"STX_DNS_MIXED": 1}), 1)
    with pytest.raises(_lib.StxError, match="STX_DNS_MIXED"):
        S.DNSAdjoint(D)
    D.close()
