"""Independent DIRECT solves replayed as one CUDA graph (stx_batch_*).

Problems of uneven size and order (the uneven-batch workload at small
sizes): the graph replay must give the same solutions as the individual
stx_field_solve calls (relative L2 <= 1e-12: the solve accumulates with
floating-point atomics, so two runs agree to round-off, not bit for bit), and
match the oracle's `elliptic` solve of each problem (relative L2 <= 1e-10).
"""
import os

import numpy as np
import pytest

import semtex_oracle as O
import semtex_b200 as S
from semtex_b200 import sessions

pytestmark = pytest.mark.gpu


def _problems(tmp_path, count, n_range, order_range):
    out = []
    for i, spec in enumerate(sessions.uneven_batch(count, seed=7, n_range=n_range, order_range=order_range)):
        path = sessions.helmholtz_session(str(tmp_path / f"p{i}"), spec["n"], spec["np"],
                                          lambda2=spec["lambda2"])
        ctx = S.Context(path)
        x, y = ctx.mesh_coords()
        f, _ = sessions.forcing_per_unique_node(x, y, 1, spec["seed"])
        sys_ = S.ModalMatrixSys(ctx, "c", spec["lambda2"])
        F = ctx.new_field("f").load_physical(f)
        U = ctx.new_field("u")
        out.append((path, ctx, sys_, F, U, f))
    return out


def test_batch_graph_matches_individual_solves_and_oracle(tmp_path):
    probs = _problems(tmp_path, 6, (2, 5), (4, 9))
    ref = []
    for path, ctx, sys_, F, U, f in probs:
        U.solve(F, sys_)
        ref.append(U.to_numpy().copy())
    B = S.Batch([(sys_, F, U) for _, _, sys_, F, U, _ in probs])
    assert B.nsystems == 6 and B.kernel_nodes > 0
    for *_, U, _ in probs:
        U.data.zero_()
    import torch
    torch.cuda.synchronize()
    for _ in range(2):
        B.launch()
    torch.cuda.synchronize()
    for (path, ctx, sys_, F, U, f), r in zip(probs, ref):
        got = U.to_numpy()
        d = np.linalg.norm(got - r) / np.linalg.norm(r)
        assert d < 1e-12, (path, d)
        P, Uo = O.elliptic(path, forcing_phys=f)
        err = np.linalg.norm(got - Uo) / np.linalg.norm(Uo)
        assert err < 1e-10, (path, err)
    B.close()
    for _, ctx, sys_, *_ in probs:
        sys_.close()
        ctx.close()


def test_batch_rejects_iterative_systems(tmp_path):
    path = sessions.helmholtz_session(str(tmp_path / "it"), 2, 5)
    ctx = S.Context(path)
    sys_ = S.ModalMatrixSys(ctx, "c", 1.0, method=S.JACPCG)
    F, U = ctx.new_field("f"), ctx.new_field("u")
    with pytest.raises(S.StxError):
        S.Batch([(sys_, F, U)])
    sys_.close()
    ctx.close()
