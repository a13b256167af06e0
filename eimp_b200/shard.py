"""Targets over the GPUs of one node: one process per GPU.

Targets (phasing) and target haplotypes (imputation) are independent given
the read-only panel, so the multi-GPU form has no data-path collective: every
rank holds the panel and phases and imputes its own contiguous block of the
targets -- the reference deals target blocks to its GPUs the same way
(GPUHandler.cpp:36-56, PBWTPhaser.cpp:476-520) -- and the blocks' results
are gathered once at the end.  The helpers below are the host side of that:
the block of a rank, the gather of the per-rank result rows in target order
and the maximum over ranks of a device time.  They run on any
torch.distributed backend: NCCL with CUDA tensors on the GPUs, gloo with CPU
tensors in the CPU tests.
"""
from __future__ import annotations

import numpy as np


def target_shard(n: int, world: int, rank: int) -> tuple[int, int]:
    """[start, stop) of rank's contiguous block of n targets; block sizes
    differ by at most one, the larger blocks first."""
    if world <= 0 or not 0 <= rank < world or n < 0:
        raise ValueError("bad shard request")
    q, r = divmod(n, world)
    start = rank * q + min(rank, r)
    return start, start + q + (rank < r)


def _dist():
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        raise RuntimeError("torch.distributed is not initialised")
    return dist


def gather_rows(local: np.ndarray, n: int, device=None) -> np.ndarray:
    """All-gather of per-rank row blocks (rank r holds the rows of
    target_shard(n, world, r)) into the n rows in target order, on every rank.
    Rows of any fixed shape and dtype; blocks are padded to the largest."""
    import torch
    dist = _dist()
    world, rank = dist.get_world_size(), dist.get_rank()
    a = np.ascontiguousarray(local)
    start, stop = target_shard(n, world, rank)
    if a.shape[0] != stop - start:
        raise ValueError(f"rank {rank} holds {a.shape[0]} rows, its block has {stop - start}")
    width = (n + world - 1) // world
    rb = int(np.prod(a.shape[1:], dtype=np.int64)) * a.dtype.itemsize   # bytes of each row
    row = a.view(np.uint8).reshape(a.shape[0], rb)
    buf = np.zeros((width, rb), np.uint8)
    buf[:a.shape[0]] = row
    t = torch.from_numpy(buf)
    if device is not None:
        t = t.to(device)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t)
    out = np.empty((n, rb), np.uint8)
    for r, p in enumerate(parts):
        s0, s1 = target_shard(n, world, r)
        out[s0:s1] = p.cpu().numpy()[:s1 - s0]
    return out.view(a.dtype).reshape((n,) + a.shape[1:])


def max_over_ranks(x: float, device=None) -> float:
    """The maximum of a per-rank value (a device time) over the ranks."""
    import torch
    dist = _dist()
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def phase_impute_sharded(ctx, hapmajor, sitemajor, cm, params, gt, sitemajor_full, af_full, typed,
                         nhaps_full, device=None):
    """Phasing and imputation of all targets of gt, each rank on its block
    (the context is the rank's GPU), gathered in target order on every rank:
    (mats, pats, dosages 2N x Mref, allele bits 2N x W(Mref))."""
    from .bits import W
    from .engine import PBWTImputer, Phaser
    dist = _dist()
    world, rank = dist.get_world_size(), dist.get_rank()
    n, M = gt.shape
    s0, s1 = target_shard(n, world, rank)
    mine = np.ascontiguousarray(gt[s0:s1])
    Mref = sitemajor_full.shape[0]
    if s1 > s0:
        mats, pats, _, _, _, _ = Phaser(ctx, hapmajor, sitemajor, cm).phase(params, mine)
        ph = np.empty((2 * (s1 - s0), W(M)), np.uint64)
        ph[0::2], ph[1::2] = mats, pats
        imp = PBWTImputer(ctx, sitemajor_full, af_full, typed, sitemajor, nhaps_full)
        imp.prepareImputation(ph, mine)
        bits, dos = imp.impute_window(0, Mref)
        per = np.concatenate([mats, pats], axis=1)
        dos2 = dos.reshape(s1 - s0, 2 * Mref)
        bits2 = bits.reshape(s1 - s0, -1)
    else:
        per = np.zeros((0, 2 * W(M)), np.uint64)
        dos2 = np.zeros((0, 2 * Mref), np.float32)
        bits2 = np.zeros((0, 2 * W(Mref)), np.uint64)
    per = gather_rows(per, n, device)
    dos2 = gather_rows(dos2, n, device)
    bits2 = gather_rows(bits2, n, device)
    wM = W(M)
    return per[:, :wM], per[:, wM:], dos2.reshape(2 * n, Mref), bits2.reshape(2 * n, -1)
