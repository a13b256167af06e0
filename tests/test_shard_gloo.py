"""The multi-GPU host side (eimp_b200/shard.py) with world size 3 on the gloo
backend (CPU): every target in exactly one rank's block, the gather of
per-rank result rows back into target order on every rank (ragged blocks,
an empty block), and the maximum over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from eimp_b200.shard import target_shard


def test_target_shard_covers_each_target_once():
    for n in (0, 1, 5, 999, 1000, 1001):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                s0, s1 = target_shard(n, world, r)
                assert 0 <= s0 <= s1 <= n
                seen += list(range(s0, s1))
            assert seen == list(range(n))
            sizes = [target_shard(n, world, r)[1] - target_shard(n, world, r)[0] for r in range(world)]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        target_shard(10, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, ns, q):
    import torch.distributed as dist
    from datetime import timedelta
    from eimp_b200.shard import gather_rows, max_over_ranks, target_shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        out = []
        for n in ns:
            s0, s1 = target_shard(n, world, rank)
            # a per-target result of the rank's block: rows of two dtypes
            ids = np.arange(s0, s1)
            rows_u64 = np.stack([ids * 3 + 1, ids ^ 0x5555], axis=1).astype(np.uint64)
            rows_f32 = (ids[:, None] * 0.5 + np.arange(7)[None, :]).astype(np.float32)
            out.append((n, gather_rows(rows_u64, n), gather_rows(rows_f32, n)))
        q.put((rank, out, max_over_ranks(10.0 + rank)))
    finally:
        dist.destroy_process_group()


def test_gather_and_max_over_ranks_gloo():
    """World size 3: ragged blocks (11 targets), a rank with an empty block
    (2 targets) and 1000 targets."""
    world, ns = 3, (11, 2, 1000)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, ns, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, out, mx in res:
        assert mx == 10.0 + world - 1
        for n, g1, g2 in out:
            ids = np.arange(n)
            np.testing.assert_array_equal(g1, np.stack([ids * 3 + 1, ids ^ 0x5555], axis=1).astype(np.uint64))
            np.testing.assert_array_equal(g2, (ids[:, None] * 0.5 + np.arange(7)[None, :]).astype(np.float32))
