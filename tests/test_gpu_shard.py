"""GPU: the sharded phase+impute entry (eimp_b200/shard.py) in a one-rank
process group equals the unsharded calls on the golden panel (the blocks,
row reshapes and gathers around the kernels; more ranks need more GPUs and
are covered by the gloo tests of the host side)."""
import os
import socket

import numpy as np
import pytest

from conftest import golden_path
from eimp_b200.bits import W

pytestmark = pytest.mark.gpu


def test_sharded_equals_unsharded_one_rank(ctx):
    import torch.distributed as dist
    from datetime import timedelta
    from eimp_b200.engine import PBWTImputer, PhaseParams, Phaser
    from eimp_b200.shard import phase_impute_sharded
    g = np.load(golden_path("golden_tiny.npz"))
    hm, sm, cm, gt = g["hapmajor_typed"], g["sitemajor_typed"], g["cm_typed"], g["gt"]
    p = PhaseParams(K=64, beamwidth=16)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=0, world_size=1, timeout=timedelta(seconds=60))
    try:
        mats, pats, dos, bits = phase_impute_sharded(ctx, hm, sm, cm, p, gt, g["sitemajor_full"], g["af_full"],
                                                     g["typed"], int(g["nhaps"]))
    finally:
        dist.destroy_process_group()
    m2, p2, _, _, _, _ = Phaser(ctx, hm, sm, cm).phase(p, gt)
    np.testing.assert_array_equal(mats, m2)
    np.testing.assert_array_equal(pats, p2)
    ph = np.empty((2 * gt.shape[0], W(gt.shape[1])), np.uint64)
    ph[0::2], ph[1::2] = m2, p2
    imp = PBWTImputer(ctx, g["sitemajor_full"], g["af_full"], g["typed"], sm, int(g["nhaps"]))
    imp.prepareImputation(ph, gt)
    b2, d2 = imp.impute_window(0, int(g["Mref"]))
    np.testing.assert_array_equal(dos, d2)
    np.testing.assert_array_equal(bits, b2)
