"""Fourier-mode sharding plumbing: the reference's parallel decomposition over
z planes (Geometry::set, src/geometry.cpp:70-110) and its block-transpose
exchange around every z transform (message_dexchange, femlib/message.c:
121-286; AuxField::transform, src/auxfield.cpp:1186-1191).

Each rank holds nz / nproc consecutive planes (rank 0 planes 0 and 1: mode 0
and the Nyquist plane), every plane padded to `psize` points so that it
splits into nproc equal blocks.  The forward exchange leaves each rank all
nz planes of its block of points, ready for the 1-D transforms along z; the
inverse exchange undoes it.  Both run as one all-to-all over
torch.distributed (NCCL between GPUs, gloo on the CPU) on a tensor of the
caller's device; the in-processor reordering is a tensor transpose.
"""

from __future__ import annotations

from dataclasses import dataclass

import torch
import torch.distributed as dist


@dataclass(frozen=True)
class PlaneLayout:
    nproc: int
    nz: int          # planes in all
    nz_local: int    # planes per rank
    nplane: int      # nodes per plane
    psize: int       # padded plane length
    base_plane: int  # first plane of this rank
    base_mode: int   # first Fourier mode of this rank
    nmode_local: int


def plane_layout(nplane: int, nz: int, nproc: int, rank: int = 0) -> PlaneLayout:
    """Geometry::set (src/geometry.cpp:70-110): the checks on the process
    count and the padded plane length.  With more than one process the plane
    is padded to the next multiple of 2 nproc -- by a whole 2 nproc when it
    already is one, as the reference pads it."""
    if nz > 1 and nz % 2:
        raise ValueError(f"N_Z must be even ({nz})")
    if nproc > 1:
        if nproc % 2:
            raise ValueError(f"No. of processors must be even ({nproc})")
        if 2 * nproc > nz:
            raise ValueError(f"No. of processors ({nproc}) can at most be half N_Z ({nz})")
        if nz % (2 * nproc):
            raise ValueError(f"No. of planes ({nz}) per processor ({nproc}) must be even")
        psize = nplane + 2 * nproc - nplane % (2 * nproc)
    else:
        psize = nplane + nplane % 2
    if not 0 <= rank < nproc:
        raise ValueError("rank out of range")
    nzl = nz // nproc
    nml = max(1, (nz + 1) // 2 // nproc)
    return PlaneLayout(nproc, nz, nzl, nplane, psize, rank * nzl, rank * nml, nml)


def exchange(data: torch.Tensor, nz_local: int, psize: int, sign: int, group=None) -> torch.Tensor:
    """message_dexchange (femlib/message.c:121-286).  sign +1: `data` holds
    this rank's nz_local planes of psize points ([nz_local * psize]); the
    result holds all nproc * nz_local planes of this rank's block of
    psize / nproc points ([nz, psize / nproc], global plane order).  sign -1
    inverts it.  Every rank of `group` must call it with the same sizes."""
    P = dist.get_world_size(group)
    if psize % P:
        raise ValueError("plane length must split into equal blocks")
    nb = psize // P
    if P == 1:
        return data.reshape(nz_local, psize).clone() if sign > 0 else data.reshape(nz_local * psize).clone()
    if sign > 0:
        # in-processor scatter: block index slowest, then the z index
        send = data.reshape(nz_local, P, nb).transpose(0, 1).contiguous()
        recv = torch.empty_like(send)
        dist.all_to_all_single(recv.view(-1), send.view(-1), group=group)
        return recv.view(P * nz_local, nb)
    send = data.reshape(P * nz_local, nb).contiguous()
    recv = torch.empty_like(send)
    dist.all_to_all_single(recv.view(-1), send.view(-1), group=group)
    return recv.view(P, nz_local, nb).transpose(0, 1).contiguous().view(nz_local * psize)


def transform_sharded(data: torch.Tensor, nz_local: int, psize: int, fn, group=None) -> torch.Tensor:
    """AuxField::transform over mode-sharded planes (src/auxfield.cpp:
    1186-1191): forward exchange, `fn` on the [nz, block] array (a transform
    along its first axis), inverse exchange."""
    return exchange(fn(exchange(data, nz_local, psize, +1, group)), nz_local, psize, -1, group)
