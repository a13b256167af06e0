"""Host-side planning of the batched step, on the CPU: the phasing batch sizes
derived from the free device memory (bench.py phase_batch_targets) and the
order in which a step enqueues its density groups (eimp_b200/batch.py
step_order)."""
import types

import numpy as np

import bench
from eimp_b200 import synth
from eimp_b200.batch import step_order


def _groups(sizes):
    """Target sets of the cfg3 shape: (targets, typed sites) per group."""
    out = []
    for nt, M in sizes:
        out.append(synth.Targets(np.arange(M, dtype=np.int64), np.zeros((nt, M), np.uint8),
                                 np.zeros((2 * nt, M), np.uint8)))
    return out


CFG3 = synth.CONFIGS["cfg3"]
SIZES = [(3334, 4000), (3333, 12000), (3333, 32000)]


def test_one_batch_per_group_when_the_rows_fit():
    tg = _groups(SIZES)
    b = bench.phase_batch_targets(CFG3, tg, 400000, 20000, 190e9)
    assert b == [3334, 3333, 3333]


def test_batches_shrink_in_proportion_when_memory_is_short():
    tg = _groups(SIZES)
    full = bench.phase_batch_targets(CFG3, tg, 400000, 20000, 190e9)
    b = bench.phase_batch_targets(CFG3, tg, 400000, 20000, 110e9)
    assert all(x < y for x, y in zip(b, full))
    # the same share of every group's targets (one scale for all)
    frac = [x / n for x, (n, _) in zip(b, SIZES)]
    assert max(frac) - min(frac) < 1e-3
    # never fewer than 64 targets, even without any memory to spare
    assert bench.phase_batch_targets(CFG3, tg, 400000, 20000, 1e9) == [64, 64, 64]


def test_step_order_puts_the_most_rows_first():
    gs = [types.SimpleNamespace(rows=r) for r in ([5, 5], [40], [7, 1], [41])]
    assert step_order(gs) == [3, 1, 0, 2]
    # stable for equal work
    assert step_order([types.SimpleNamespace(rows=[3])] * 3) == [0, 1, 2]
