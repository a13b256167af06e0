"""GPU: the serving loop (eimp_b200/serving.py) with two slots on one device.
Requests of different sizes arrive together and while others run; every
request's phased haplotypes, imputed bits and dosages must equal those of the
same targets phased and imputed alone (bit-exact)."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_serving_results_equal_alone(smalltest):
    from eimp_b200.engine import Context, PBWTImputer, PhaseParams, Phaser
    from eimp_b200.serving import GpuSlot, Server, device_bytes_per_target
    from eimp_b200.synth import typed_views
    from eimp_b200.bits import W
    panel, groups = smalltest
    tg = groups[0]
    hm, sm, cm = typed_views(panel, tg.typed)
    params = PhaseParams(K=200, beamwidth=32)
    M, Mref = len(tg.typed), panel.nsites
    slots = [GpuSlot(0, hm, sm, cm, panel.sitemajor, panel.af.astype(np.float32), tg.typed, panel.nhaps, params)
             for _ in range(2)]
    bpt = device_bytes_per_target(M, Mref, 200, P=64)
    srv = Server(slots, max_batch_targets=4, mem_budget=bpt * 8, bytes_per_target=bpt)
    gt = tg.gt
    cuts = [(0, 2), (2, 3), (3, 5), (5, 6), (6, gt.shape[0])]
    futs = [srv.submit(gt[a:b]) for a, b in cuts[:3]]
    time.sleep(0.05)   # the rest arrives while the first launches run
    futs += [srv.submit(gt[a:b]) for a, b in cuts[3:]]
    res = [f.result(timeout=600) for f in futs]
    lat = srv.latencies()
    srv.close()
    assert len(lat) == len(cuts)

    ctx = Context(0)
    ph = Phaser(ctx, hm, sm, cm)
    imp = PBWTImputer(ctx, panel.sitemajor, panel.af.astype(np.float32), tg.typed, sm, panel.nhaps)
    for (a, b), r in zip(cuts, res):
        mats, pats, _, _, _, _ = ph.phase(params, gt[a:b])
        np.testing.assert_array_equal(r.mats, mats)
        np.testing.assert_array_equal(r.pats, pats)
        phased = np.empty((2 * (b - a), W(M)), np.uint64)
        phased[0::2], phased[1::2] = mats, pats
        imp.prepareImputation(phased, gt[a:b])
        bits, dos = imp.impute_window(0, Mref)
        np.testing.assert_array_equal(r.bits, bits)
        np.testing.assert_array_equal(r.dosages, dos)
    ctx.close()
