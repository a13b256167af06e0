"""GPU parity: the output statistics of an imputed bunch
(VCFData::writeVCFImputedBunch, VCFData.cpp:3068-3446) computed on the device
against the reference's own writer (oracle/_ref/libeimp_refwriter.so, the
reference's VCFData.cpp with its records read back) and the oracle
restatement on the same imputed bunch: allele dosages and alleles written,
DS, GP, r2, AF, MAF, AC, AN, filter flags, the conflict count and the
--improveCalls run statistics, all bit-exact (the statistics' double totals,
which the device adds in its own order, within 1e-12 relative), for diploid
and haploid targets, with and without --overwriteCalls / --improveCalls."""
import ctypes as C

import numpy as np
import pytest

from conftest import golden_path
from eimp_b200.bits import W, unpack_rows

pytestmark = pytest.mark.gpu

KEYS = ("ads", "gtbits", "ds", "gp", "r2", "af", "maf", "ac", "an", "passed")
u32 = lambda a: np.ascontiguousarray(a, np.float32).view(np.uint32)  # noqa: E731


def check_writer(got, mref_begin, nsites, phased, dm, dp, gt, typed, Mref, af, overwrite, improve, r2f, maff, bits,
                 dos, haploid):
    """The device's outputs against the reference's own writer on the same bunch."""
    from oracle import refwriter as RW
    w = RW.write_bunch(mref_begin, bits, dos, phased, dm, dp, gt, typed, Mref, af, haploid, overwrite, improve, r2f,
                       maff)
    np.testing.assert_array_equal(got["passed"], w["written"])
    sel = w["written"] == 1
    np.testing.assert_array_equal(u32(got["ads"][:, sel]), u32(w["ads"][:, sel]))
    exp = np.where(w["gtv"] == RW.INT32_VECTOR_END, 0, (w["gtv"] >> 1) - 1)
    np.testing.assert_array_equal(unpack_rows(got["gtbits"], nsites)[:, sel], exp[:, sel])
    for k in ("r2", "af", "maf"):
        np.testing.assert_array_equal(u32(got[k][sel]), u32(w[k][sel]), err_msg=k)
    np.testing.assert_array_equal(got["ac"][sel], w["ac"][sel])
    np.testing.assert_array_equal(got["an"][sel], w["an"][sel])
    # DS and GP where the writer sets them (a haploid target's typed call leaves them unset)
    N = gt.shape[0]
    unset = np.zeros((N, nsites), bool)
    if haploid is not None and not overwrite:
        tix = {int(m): k for k, m in enumerate(typed)}
        for s in range(nsites):
            k = tix.get(mref_begin + s)
            if k is not None:
                unset[:, s] = (np.asarray(haploid) != 0) & (gt[:, k] != 3)
    keep = ~unset & sel[None, :]
    np.testing.assert_array_equal(u32(got["ds"])[keep], u32(w["ds"])[keep])
    np.testing.assert_array_equal(u32(got["gp"])[np.repeat(keep, 3, axis=0)], u32(w["gp"])[np.repeat(keep, 3, axis=0)])
    assert got["conflicts"] == w["conflicts"]
    return w


def check(imp, mref_begin, nsites, phased, dm, dp, gt, typed, Mref, af, overwrite, improve, r2f, maff, haploid=None):
    from oracle import refwriter as RW
    from oracle import restate as R
    bits, dos = imp.impute_window(mref_begin, nsites)
    imp.improveStats(reset=True)
    got = imp.writeImputedBunchStats(mref_begin, nsites, overwrite, improve, r2f, maff, ds=True, gp=True)
    cnt, tot = imp.improveStats(reset=True)
    ref = R.site_stats(mref_begin, bits, dos, phased, dm, dp, gt, typed, Mref, af, overwrite, improve, r2f, maff,
                       want_ds=True, want_gp=True, haploid=haploid)
    for k in KEYS:
        np.testing.assert_array_equal(u32(got[k]) if got[k].dtype == np.float32 else got[k],
                                      u32(ref[k]) if ref[k].dtype == np.float32 else ref[k], err_msg=k)
    assert got["conflicts"] == ref["conflicts"]
    np.testing.assert_array_equal(cnt, ref["improve_counts"])
    np.testing.assert_allclose(tot, ref["improve_totals"], rtol=1e-12, atol=0)
    if RW.available():
        w = check_writer(got, mref_begin, nsites, phased, dm, dp, gt, typed, Mref, af, overwrite, improve, r2f, maff,
                         bits, dos, haploid)
        np.testing.assert_array_equal(cnt, w["improve_counts"])
        np.testing.assert_allclose(tot, w["improve_totals"], rtol=1e-12, atol=0)
    return got


@pytest.mark.parametrize("overwrite,improve", [(False, False), (True, False), (False, True)])
def test_site_stats_golden_panel(ctx, overwrite, improve):
    from eimp_b200.engine import PBWTImputer
    g = np.load(golden_path("golden_tiny.npz"))
    imp = PBWTImputer(ctx, g["sitemajor_full"], g["af_full"], g["typed"], g["sitemajor_typed"], int(g["nhaps"]),
                      imputeCalls=overwrite or improve)
    imp.prepareImputation(g["imp_phased"], g["gt"])
    dm, dp = g["K64_dos_mat"], g["K64_dos_pat"]
    imp.setPhasedDosages(dm, dp)
    Mref = int(g["Mref"])
    for b0, n in [(0, Mref), (100, 1500)]:
        got = check(imp, b0, n, g["imp_phased"], dm, dp, g["gt"], g["typed"], Mref, g["af_full"], overwrite, improve,
                    0.0, 0.0)
        assert got["passed"].all()   # no filter thresholds
        np.testing.assert_array_equal(got["an"], 2 * g["gt"].shape[0])


@pytest.mark.parametrize("overwrite,improve", [(False, False), (False, True)])
def test_site_stats_cfg1_sample(ctx, overwrite, improve):
    """cfg1 panel (5000 haplotypes x 20000 sites, 2000 typed), 20 targets
    phased on the device, the window of all 20000 sites, r2 >= 0.3 and
    MAF >= 0.01 output filters."""
    from eimp_b200 import synth
    from eimp_b200.engine import PBWTImputer, PhaseParams, Phaser
    from eimp_b200.synth import typed_views
    panel, groups = synth.generate("cfg1")
    tg = groups[0]
    nt = 20
    hm, sm, cm = typed_views(panel, tg.typed)
    gt = tg.gt[:nt]
    mats, pats, dm, dp, _, _ = Phaser(ctx, hm, sm, cm).phase(PhaseParams(K=1024, beamwidth=64), gt)
    phased = np.empty((2 * nt, W(len(tg.typed))), np.uint64)
    phased[0::2], phased[1::2] = mats, pats
    imp = PBWTImputer(ctx, panel.sitemajor, panel.af, tg.typed, sm, panel.nhaps, imputeCalls=overwrite or improve)
    imp.prepareImputation(phased, gt)
    imp.setPhasedDosages(dm, dp)
    got = check(imp, 0, panel.nsites, phased, dm, dp, gt, tg.typed, panel.nsites, panel.af, overwrite, improve,
                0.3, 0.01)
    assert 0 < got["passed"].sum() < panel.nsites


@pytest.mark.parametrize("overwrite,improve", [(False, False), (True, False), (False, True)])
def test_site_stats_haploid_targets(ctx, overwrite, improve):
    """The golden haploid panel (every fourth panel sample haploid, 3 of 8
    targets haploid): the haploid targets' first-row dosages and alleles, the
    vector-end second entries, the typed calls that add nothing to AF/r2/AN."""
    from eimp_b200.engine import PBWTImputer
    g = np.load(golden_path("golden_haploid.npz"))
    imp = PBWTImputer(ctx, g["sitemajor_full"], g["af_full"], g["typed"], g["sitemajor_typed"], int(g["nhaps"]),
                      imputeCalls=overwrite or improve, haploid_ref=g["ref_haploid"])
    imp.prepareImputation(g["imp_phased"], g["gt"], haploid_targets=g["tgt_haploid"])
    dm, dp = g["K64_dos_mat"], g["K64_dos_pat"]
    imp.setPhasedDosages(dm, dp)
    Mref = int(g["Mref"])
    assert g["tgt_haploid"].any()
    for b0, n in [(0, Mref), (211, 1400)]:
        got = check(imp, b0, n, g["imp_phased"], dm, dp, g["gt"], g["typed"], Mref, g["af_full"], overwrite, improve,
                    0.0, 0.0, haploid=g["tgt_haploid"])
        assert (got["an"] < 2 * g["gt"].shape[0]).all()


def test_site_stats_dev_in_place(ctx):
    """eimp_imp_site_stats_dev with the allele dosages and alleles written
    over the imputed bunch's own device buffers equals the host call."""
    import torch
    from eimp_b200._lib import EimpSiteStatsOpts, ptr
    from eimp_b200.engine import PBWTImputer
    g = np.load(golden_path("golden_tiny.npz"))
    imp = PBWTImputer(ctx, g["sitemajor_full"], g["af_full"], g["typed"], g["sitemajor_typed"], int(g["nhaps"]))
    imp.prepareImputation(g["imp_phased"], g["gt"])
    imp.setPhasedDosages(g["K64_dos_mat"], g["K64_dos_pat"])
    b0, n = 37, 2000
    want = imp.writeImputedBunchStats(b0, n, r2filter=0.5)
    nh, wb = 2 * g["gt"].shape[0], W(n)
    dev = torch.device("cuda", 0)
    d_bits = torch.zeros(nh * wb, dtype=torch.int64, device=dev)
    d_dos = torch.zeros(nh * n, dtype=torch.float32, device=dev)
    d_pdm = torch.from_numpy(np.ascontiguousarray(g["K64_dos_mat"])).to(dev)
    d_pdp = torch.from_numpy(np.ascontiguousarray(g["K64_dos_pat"])).to(dev)
    site = {k: torch.zeros(n, dtype=t, device=dev) for k, t in
            [("r2", torch.float32), ("af", torch.float32), ("maf", torch.float32), ("ac", torch.int32),
             ("an", torch.int32), ("passed", torch.uint8)]}
    conf = torch.zeros(1, dtype=torch.int64, device=dev)
    torch.cuda.synchronize()
    L, h = ctx.L, ctx.h
    ctx.check(L.eimp_imp_bunch_dev(h, b0, n, ptr(d_bits), wb, ptr(d_dos), n))
    o = EimpSiteStatsOpts(0, 0, 0.5, 0.0)
    ctx.check(L.eimp_imp_site_stats_dev(h, b0, n, ptr(d_bits), wb, ptr(d_dos), n, ptr(d_pdm), ptr(d_pdp),
                                        g["K64_dos_mat"].shape[1], C.byref(o), ptr(d_dos), n, ptr(d_bits), wb, None,
                                        None, ptr(site["r2"]), ptr(site["af"]), ptr(site["maf"]), ptr(site["ac"]),
                                        ptr(site["an"]), ptr(site["passed"]), ptr(conf)))
    ctx.check(L.eimp_synchronize(h))
    np.testing.assert_array_equal(d_dos.cpu().numpy().reshape(nh, n), want["ads"])
    np.testing.assert_array_equal(d_bits.cpu().numpy().view(np.uint64).reshape(nh, wb), want["gtbits"])
    for k in site:
        np.testing.assert_array_equal(site[k].cpu().numpy(), want[k], err_msg=k)
    assert int(conf.item()) == want["conflicts"]
