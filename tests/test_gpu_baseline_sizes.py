"""GPU parity with the oracle at the benchmark sizes.

The benchmark workloads, built by the same seeded builders the benchmark
uses, run through the C ABI at full size and are compared with the oracle's
results on the same inputs, reduced to checksums (tests/golden/baseline/*.npz,
made by tests/golden/make_baseline_fixtures.py: the field norm, four seeded
Gaussian projections, 256 sampled values).  Each error is relative to the
field scale the other parity tests use (velocity: the largest velocity
component norm; pressure: the larger of its norm and the dynamic-pressure
scale ||u.u||); the bar is 1e-10 (pressure 1e-9).

- c2: 16x16 quads, N_P=11, N_Z=64 (32 modes in two mode groups), the
  device-buffer solve and the host-buffer call;
- c3: Taylor-Green 24x24, N_P=9, N_Z=96, five steps (two start-up PCG steps,
  three direct), plain and with 3/2-rule products;
- c5: the channel 16x8, N_P=9, N_Z=32 with high-order pressure walls, ten
  steps;
- c4: all 64 problems of the uneven batch through its CUDA graph.
"""
import os
import sys

import numpy as np
import pytest

import semtex_b200 as S
from semtex_b200 import sessions

from conftest import GOLDEN

sys.path.insert(0, GOLDEN)
import make_baseline_fixtures as FX  # noqa: E402

pytestmark = pytest.mark.gpu
TOL, PTOL = 1e-10, 1e-9


def _check(got, ref, scale=None, tol=TOL, what=""):
    e = FX.errors(got, ref, scale)
    assert max(e.values()) < tol, (what, e)
    return e


def test_c2_full_size(tmp_path):
    ref = FX.load("c2")["c"]
    p = FX.c2_session(str(tmp_path))
    ctx = S.Context(p)
    x, y = ctx.mesh_coords()
    f, _ = sessions.forcing_per_unique_node(x, y, ctx.nz, FX.C2["seed"])
    sysm = S.ModalMatrixSys(ctx, "c", FX.C2["lambda2"], FX.C2["beta"])
    # the device-buffer path the benchmark times
    F = ctx.new_field("f").load_physical(f).transform(S.FORWARD).zero_nyquist()
    U = ctx.new_field("c").solve(F, sysm)
    assert sysm.status() == 0
    U.transform(S.INVERSE)
    _check(U.to_numpy(), ref, what="device solve")
    # the host-buffer call of the end-to-end measurement
    _check(sysm.solve_host(f), ref, what="host solve")


def _dns(ctx, ic, steps):
    D = S.DNS(ctx, 1)
    D.restart(ic, 0.0)
    D.advance(steps)
    assert D.status() == 0
    out = {c: D.field(c) for c in ctx.fields}
    t = D.state()
    D.close()
    return out, t


def _compare_dns(gpu, ref, vel, pname):
    scale = max(float(ref[c]["norm"]) for c in vel)
    for c in vel:
        _check(gpu[c], ref[c], scale, TOL, c)
    pscale = max(float(ref[pname]["norm"]), float(np.linalg.norm(sum(gpu[c] ** 2 for c in vel))))
    _check(gpu[pname], ref[pname], pscale, PTOL, pname)


@pytest.mark.parametrize("name", ["c3", "c3d"])
def test_c3_taylor_green_full_size(tmp_path, name):
    ref = FX.load(name)
    p = FX.c3_session(str(tmp_path), name == "c3d")
    ctx = S.Context(p)
    funcs = S._user_functions(p)
    ic = {c: ctx.evaluate(funcs[c], 0.0) for c in ctx.fields if c in funcs}
    gpu, _ = _dns(ctx, ic, int(ref["meta"]["steps"]))
    _compare_dns(gpu, ref, "uvw", "p")
    ctx.close()


def test_c5_channel_full_size(tmp_path):
    ref = FX.load("c5")
    p = FX.c5_session(str(tmp_path))
    ctx = S.Context(p)
    x, y = ctx.mesh_coords()
    gpu, _ = _dns(ctx, FX.c5_initial(x, y, ctx.nz), int(ref["meta"]["steps"]))
    _compare_dns(gpu, ref, "uvw", "p")
    ctx.close()


def test_c4_uneven_batch_full(tmp_path):
    ref = FX.load("c4")
    specs = sessions.uneven_batch()
    items, ctxs = [], []
    for i, sp in enumerate(specs):
        ctx = S.Context(FX.c4_problem(str(tmp_path), i, sp))
        x, y = ctx.mesh_coords()
        f, _ = sessions.forcing_per_unique_node(x, y, 1, sp["seed"])
        items.append((S.ModalMatrixSys(ctx, "c", sp["lambda2"]), ctx.new_field("f").load_physical(f),
                      ctx.new_field("u")))
        ctxs.append(ctx)
    assert max(sp["n"] for sp in specs) == 32 and max(sp["np"] for sp in specs) == 13
    import torch
    B = S.Batch(items)   # runs every solve once outside the capture
    for _, _, u in items:
        u.data.zero_()
    torch.cuda.synchronize()
    B.launch()           # the replay alone must rewrite every solution
    torch.cuda.synchronize()
    worst = 0.0
    for i, (sysm, _, u) in enumerate(items):
        assert sysm.status() == 0
        e = _check(u.to_numpy(), ref[f"p{i}"], what=f"problem {i}")
        worst = max(worst, max(e.values()))
    B.close()
    for s, _, _ in items:
        s.close()
    for c in ctxs:
        c.close()
    assert worst < TOL
