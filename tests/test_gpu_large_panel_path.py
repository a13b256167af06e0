"""The pieces of the large-panel (cfg4) path, on small sizes: the device bit
transpose with row strides (eimp_transpose_bits_dev) against numpy, the
device panel generator (eimp_b200/synth_device.py: site rows = the transpose
of the mosaics, allele frequencies = popcounts), a DensityGroup whose
references are built on the device from the resident panel giving the same
phased haplotypes, matches and dosages bit for bit as one built from host
typed views, and the prefix-array slices (eimp_imp_prefix_slice) equal to the
full prefix arrays; then the FP64 sample check of the cfg4 leg on cfg1."""
import numpy as np
import pytest

from eimp_b200.bits import W, transpose_bits

pytestmark = pytest.mark.gpu


def test_transpose_bits_dev_strides():
    import torch
    from eimp_b200.engine import Context
    ctx = Context(0)
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(1)
    rows, cols, src_ld = 192, 3000, W(3000) + 3          # source rows longer than their bits
    src = rng.integers(0, 2**63, (rows, src_ld), dtype=np.int64).view(np.uint64)
    src[:, (cols + 63) // 64:] = 0
    last = cols % 64
    src[:, cols // 64] &= np.uint64((1 << last) - 1)
    dst_ld, off = 9, 2                                    # write words 2..4 of rows of 9 words
    d_src = torch.from_numpy(src.view(np.int64)).to(dev)
    d_dst = torch.full((cols, dst_ld), -1, dtype=torch.int64, device=dev)
    ctx.check(ctx.L.eimp_transpose_bits_dev(ctx.h, d_src.data_ptr(), rows, src_ld, d_dst.data_ptr() + off * 8, cols,
                                            dst_ld))
    ctx.synchronize()
    got = d_dst.cpu().numpy().view(np.uint64)
    want = transpose_bits(np.ascontiguousarray(src[:, :W(cols)]), rows, cols)   # (cols, W(rows))
    np.testing.assert_array_equal(got[:, off:off + 3], want[:, :3])
    assert (got[:, :off] == np.uint64(2**64 - 1)).all() and (got[:, off + 3:] == np.uint64(2**64 - 1)).all()
    ctx.close()


def test_device_generator_small():
    import torch
    from eimp_b200 import synth, synth_device
    cfg = synth.SynthConfig("devsmall", nhaps=1280, nsites=9000, segment_mb=3.0, founders=60,
                            groups=(synth.TargetGroup(10, 0.05, 0.01, 0.01),), K=256, beam=32, seed=99)
    P = synth_device.generate(cfg, 0, block=512)
    site = P.d_site.cpu().numpy().view(np.uint64)
    assert site.shape == (cfg.nsites, W(cfg.nhaps))
    hm = transpose_bits(site, cfg.nsites, cfg.nhaps)                   # back to haplotype rows
    dense = np.unpackbits(hm.view(np.uint8), axis=1, bitorder="little")[:, :cfg.nsites]
    np.testing.assert_array_equal(P.d_af.cpu().numpy(), (dense.sum(axis=0) / cfg.nhaps).astype(np.float32))
    # padding haplotype bits are zero; mosaics of few founders: many shared rows
    assert not (np.unpackbits(site.view(np.uint8), axis=1, bitorder="little")[:, cfg.nhaps:]).any()
    assert 0.0 < float(P.d_af.mean()) < 1.0
    typed, gt = synth_device.targets(P, cfg.groups[0], 10, seed=5)
    assert gt.shape == (10, len(typed)) and set(np.unique(gt)) <= {0, 1, 2, 3}
    assert ((gt == 3).sum(axis=1) == int(round(0.01 * len(typed)))).all()
    del P
    torch.cuda.empty_cache()


def test_device_built_references_and_prefix_slices():
    import torch
    from eimp_b200 import synth
    from eimp_b200.batch import DensityGroup
    from eimp_b200.engine import PhaseParams
    from oracle import restate as R
    panel, groups = synth.generate("cfg1")
    tg = groups[0]
    dev = torch.device("cuda", 0)
    d_full = torch.from_numpy(panel.sitemajor.view(np.int64)).to(dev)
    d_af = torch.from_numpy(panel.af.astype(np.float32)).to(dev)
    hm, sm, cm = synth.typed_views(panel, tg.typed)
    gt = tg.gt[:24]
    pp = PhaseParams(K=1024, beamwidth=64)
    host = DensityGroup(0, d_full, d_af, panel.nhaps, tg.typed, hm, sm, cm, gt, pp, batch_targets=24)
    devg = DensityGroup(0, d_full, d_af, panel.nhaps, tg.typed, None, None, cm, gt, pp, batch_targets=24)
    for g in (host, devg):
        g.enqueue()
        g.ctx.synchronize()
    for a, b in ((host.d_mats, devg.d_mats), (host.d_pats, devg.d_pats), (host.d_pdm, devg.d_pdm),
                 (host.d_dos, devg.d_dos), (host.d_bits, devg.d_bits)):
        assert torch.equal(a, b)
    # prefix-array slices against the whole prefix arrays
    M, K = devg.M, panel.nhaps
    ap = np.empty((M + 1, K), np.int32)
    devg.ctx.check(devg.L.eimp_imp_refpbwt(devg.h, None, ap.ctypes.data))
    for site, lo, hi in ((0, 0, K - 1), (M, 17, 17), (M // 2, 100, 2000), (7, K - 5, K - 1)):
        out = np.empty(hi - lo + 1, np.int32)
        devg.ctx.check(devg.L.eimp_imp_prefix_slice(devg.h, site, lo, hi, out.ctypes.data))
        np.testing.assert_array_equal(out, ap[site, lo:hi + 1])
    from eimp_b200._lib import EimpError
    with pytest.raises(EimpError):
        devg.ctx.check(devg.L.eimp_imp_prefix_slice(devg.h, M + 1, 0, 0, np.empty(1, np.int32).ctypes.data))

    # the FP64 check of the cfg4 leg (bench.py cfg4_fp64) on these outputs
    class P:
        pass
    Pp = P()
    Pp.nsites, Pp.nhaps, Pp.d_site, Pp.d_af = panel.nsites, panel.nhaps, d_full, d_af
    import bench
    fp = bench.cfg4_fp64(devg, Pp, tg.typed, nhap_sample=6, frac=0.05)
    assert fp["covered"] > 0 and fp["uncovered_marked_conflict"]
    assert fp["not_equal_to_rounded_fp64"] == 0 and fp["max_abs_err"] <= 3e-8
    # and one haplotype's dosages against the oracle's FP64 pass over all sites
    import ctypes as C
    h = 3
    n = C.c_size_t(0)
    devg.ctx.check(devg.L.eimp_imp_matches(devg.h, h, None, 0, C.byref(n)))
    m = np.zeros((n.value, 4), np.int32)
    devg.ctx.check(devg.L.eimp_imp_matches(devg.h, h, m.ctypes.data, n.value, C.byref(n)))
    phased = devg.d_ph.cpu().numpy().view(np.uint64).reshape(-1, W(devg.M))
    miss = np.flatnonzero(gt[h // 2] == 3).astype(np.int64)
    _, dos, _, d64 = R.impute(m, ap, panel.sitemajor, tg.typed, panel.af, panel.nhaps, miss, phased[h], fp64=True)
    np.testing.assert_array_equal(devg.d_dos[h].cpu().numpy(), dos)
    cov = d64 >= 0
    assert np.abs(dos[cov].astype(np.float64) - d64[cov]).max() <= 3e-8
    for g in (host, devg):
        g.close()
