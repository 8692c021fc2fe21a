"""Full-state DNS checkpoints: a run interrupted at step k, saved, loaded
into a fresh DNS of the same session and continued, ends where the
uninterrupted run ends (to round-off) -- the multistep history, the high-order pressure BC
levels and the alternating form's switch travel with the fields (the
reference's restart zeroes the history instead, dns/integrate.cpp:130-136).
Also: a checkpoint of another layout is rejected."""
import numpy as np
import pytest

import semtex_b200 as S
from semtex_b200 import _lib, sessions

pytestmark = pytest.mark.gpu


def _channel(tmp_path, name="c", extra=None):
    p = sessions.channel_session(str(tmp_path / name), 4, 2, 6, 8, nstep=40, extra=extra)
    ctx = S.Context(p)
    x, y = ctx.mesh_coords()
    ic = sessions.channel_initial(x, y, np.arange(ctx.nz) * 2 * np.pi / ctx.nz, amplitude=0.05)
    return ctx, ic


@pytest.mark.parametrize("k,total", [(1, 6), (4, 9), (5, 40)])
def test_checkpoint_continues_exactly(tmp_path, k, total):
    ctx, ic = _channel(tmp_path)
    A = S.DNS(ctx, 1)
    A.restart(ic, 0.0)
    A.advance(total)
    ref = {c: A.field(c) for c in ctx.fields}
    A.close()
    B = S.DNS(ctx, 1)
    B.restart(ic, 0.0)
    B.advance(k)
    buf = B.checkpoint()
    B.close()
    C = S.DNS(ctx, 1)
    C.restart({c: np.zeros_like(v) for c, v in ic.items()}, 0.0)
    C.restore(buf)
    assert C.state()[0] == k
    C.advance(total - k)
    assert C.state()[0] == total
    _same(ctx, {c: C.field(c) for c in ctx.fields}, ref)
    C.close()


def _same(ctx, got, ref):
    # the same steps to round-off (the skeleton products sum with atomics,
    # so two runs agree to rounding, not bit for bit); the pressure of a
    # pinned singular system is compared on the dynamic-pressure scale
    vel = ctx.fields[:-1]
    scale = max(np.linalg.norm(ref[c]) for c in vel)
    for c in vel:
        assert np.linalg.norm(got[c] - ref[c]) <= 1e-12 * scale, c
    p = ctx.fields[-1]
    pscale = max(np.linalg.norm(ref[p]), np.linalg.norm(sum(ref[c] ** 2 for c in vel)))
    assert np.linalg.norm(got[p] - ref[p]) <= 1e-10 * pscale


def test_checkpoint_of_other_layout_rejected(tmp_path):
    ctx, ic = _channel(tmp_path)
    D = S.DNS(ctx, 1)
    D.restart(ic, 0.0)
    D.advance(2)
    buf = D.checkpoint()
    ctx2, ic2 = _channel(tmp_path, "d", extra={"N_TIME": 2})
    E = S.DNS(ctx2, 1)
    E.restart(ic2, 0.0)
    with pytest.raises(_lib.StxError, match="different"):
        E.restore(buf)
    bad = buf.copy()
    bad[0] = 0.0
    with pytest.raises(_lib.StxError, match="not a DNS checkpoint"):
        D.restore(bad)
