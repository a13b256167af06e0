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


def test_window_requests_equal_alone_and_plain():
    """Serving requests with their own typed sites in windows of a resident
    panel (the cfg5 shape at cfg1 scale): every request's phased haplotypes,
    imputed bits and dosages equal those of the same request run alone on
    one slot, and those of the plain calls on the window's sub-panel
    (Phaser / PBWTImputer with host-built references)."""
    import torch
    from eimp_b200 import synth
    from eimp_b200.bits import W
    from eimp_b200.engine import Context, PBWTImputer, PhaseParams, Phaser
    from eimp_b200.serving import Server, WindowSlot, window_request_bytes
    cfg = synth.CONFIGS["cfg1"]
    panel, _ = synth.generate(cfg)
    reqs = synth.window_requests(cfg, panel, 6, seed=5, max_targets=24, window_mb=(1.0, 3.0))
    dev = torch.device("cuda", 0)
    d_full = torch.from_numpy(panel.sitemajor.view(np.int64)).to(dev)
    d_af = torch.from_numpy(panel.af.astype(np.float32)).to(dev)
    params = PhaseParams(K=512, beamwidth=32)
    nb = lambda r: window_request_bytes(r, panel.nhaps, 512, P=32)  # noqa: E731
    slots = [WindowSlot(0, d_full, d_af, panel.cm, panel.nhaps, params) for _ in range(2)]
    srv = Server(slots, merge=False, mem_budget=3 * max(nb(r) for r in reqs), request_bytes=nb)
    futs = [srv.submit(r) for r in reqs[:3]]
    time.sleep(0.05)
    futs += [srv.submit(r) for r in reqs[3:]]
    mixed = [f.result(timeout=600) for f in futs]
    srv.close()
    alone_slot = WindowSlot(0, d_full, d_af, panel.cm, panel.nhaps, params)
    ctx = Context(0)
    for r, got in zip(reqs, mixed):
        alone = alone_slot.run(r)
        for a, b in zip((got.mats, got.pats, got.bits, got.dosages), alone):
            np.testing.assert_array_equal(a, b)
        # the plain calls on the window's sub-panel, references built on the host
        sub = synth.Panel(panel.nhaps, r.hi - r.lo, panel.pos[r.lo:r.hi], panel.cm[r.lo:r.hi],
                          panel.af[r.lo:r.hi], None, np.ascontiguousarray(panel.sitemajor[r.lo:r.hi]))
        hm, sm, cm = synth.typed_views(sub, r.typed)
        mats, pats, *_ = Phaser(ctx, hm, sm, cm).phase(params, r.gt)
        np.testing.assert_array_equal(got.mats, mats)
        np.testing.assert_array_equal(got.pats, pats)
        ph = np.empty((2 * r.n, W(len(r.typed))), np.uint64)
        ph[0::2], ph[1::2] = mats, pats
        imp = PBWTImputer(ctx, sub.sitemajor, sub.af, r.typed, sm, panel.nhaps)
        imp.prepareImputation(ph, r.gt)
        bits, dos = imp.impute_window(0, r.hi - r.lo)
        np.testing.assert_array_equal(got.bits, bits)
        np.testing.assert_array_equal(got.dosages, dos)
    alone_slot.close()
    ctx.close()
