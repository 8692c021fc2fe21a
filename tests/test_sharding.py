"""Fourier-mode sharding plumbing on the CPU: the reference's plane layout
checks (src/geometry.cpp:70-110) and its block-transpose exchange
(femlib/message.c:121-286) over two gloo ranks, with the sharded z
transform equal to the single-process one."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from semtex_b200.sharding import plane_layout  # noqa: E402


def test_plane_layout_rules():
    L = plane_layout(30, 8, 2, rank=1)
    assert (L.psize, L.nz_local, L.base_plane, L.base_mode, L.nmode_local) == (32, 4, 4, 2, 2)
    assert plane_layout(32, 8, 2).psize == 36          # padded by 2 nproc even when divisible
    assert plane_layout(31, 8, 1).psize == 32
    assert plane_layout(30, 16, 4, rank=3).base_plane == 12
    for nplane, nz, nproc in ((30, 8, 3), (30, 4, 4), (30, 12, 4), (30, 7, 1)):
        with pytest.raises(ValueError):
            plane_layout(nplane, nz, nproc)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch
    import torch.distributed as dist
    import semtex_oracle as O
    from semtex_b200.sharding import exchange, plane_layout, transform_sharded
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        nz, nplane = 8, 30
        L = plane_layout(nplane, nz, ws, rank)
        g = np.random.default_rng(5).standard_normal((nz, L.psize))
        g[:, nplane:] = 0.0
        mine = torch.from_numpy(g[L.base_plane:L.base_plane + L.nz_local].copy()).reshape(-1)
        fwd = exchange(mine, L.nz_local, L.psize, +1)
        nb = L.psize // ws
        ok_fwd = np.array_equal(fwd.numpy(), g[:, rank * nb:(rank + 1) * nb])
        back = exchange(fwd, L.nz_local, L.psize, -1)
        ok_back = np.array_equal(back.numpy(), mine.numpy())

        def dft(a):  # the packed real DFT along z of every point of the block
            return torch.from_numpy(O.dft_forward(a.numpy()[:, :, None, None])[:, :, 0, 0].copy())

        t = transform_sharded(mine, L.nz_local, L.psize, dft).numpy().reshape(L.nz_local, L.psize)
        ref = O.dft_forward(g[:, :, None, None])[:, :, 0, 0][L.base_plane:L.base_plane + L.nz_local]
        out.put((rank, ok_fwd, ok_back, float(np.abs(t - ref).max())))
    finally:
        dist.destroy_process_group()


def test_exchange_and_sharded_transform_two_gloo_ranks():
    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, ok_fwd, ok_back, err in got:
        assert ok_fwd and ok_back, r
        assert err < 1e-14, (r, err)
